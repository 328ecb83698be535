"""B200-native (sm_100a) matrix-free Pauli-Hamiltonian MVP.

A drop-in for TenCirPauli's ``PauliOperator.native_mvp_plan()`` / ``.mvp()``
path: canonical Pauli operators are compiled into device plans and applied by
hand-written CUDA kernels in ``libtcpmvp.so`` (C ABI: ``include/tcp_mvp.h``).
"""

from ._native_mvp import DEFAULT_MAX_BYTES, MIN_ENFORCED_MAX_BYTES
from .pauli import NativeMVPPlan, PauliOperator, PauliTerm, PauliWord

__version__ = "0.1.0"

__all__ = [
    "DEFAULT_MAX_BYTES",
    "MIN_ENFORCED_MAX_BYTES",
    "NativeMVPPlan",
    "PauliOperator",
    "PauliTerm",
    "PauliWord",
    "__version__",
]
