"""B200-native (sm_100a) matrix-free Pauli-Hamiltonian MVP.

A drop-in for TenCirPauli's ``PauliOperator.native_mvp_plan()`` / ``.mvp()``
path: canonical Pauli operators are compiled into device plans and applied by
hand-written CUDA kernels in ``libtcpmvp.so`` (C ABI: ``include/tcp_mvp.h``).
"""

from ._native_mvp import DEFAULT_MAX_BYTES, MIN_ENFORCED_MAX_BYTES
from ._native_mvp import COOMatrix, CSRMatrix
from .pauli import NativeMVPPlan, PauliOperator, PauliTerm, PauliWord
from .symmetry import U1MvpPlan, U1RestrictedOperator, U1Sector

__version__ = "0.1.0"

__all__ = [
    "COOMatrix",
    "CSRMatrix",
    "U1MvpPlan",
    "U1RestrictedOperator",
    "U1Sector",
    "DEFAULT_MAX_BYTES",
    "MIN_ENFORCED_MAX_BYTES",
    "NativeMVPPlan",
    "PauliOperator",
    "PauliTerm",
    "PauliWord",
    "__version__",
]
