"""Versioned pure-array MVP plan whose executor runs on the device.

Mirrors the reference's ``BackendMVPPlan`` for Pauli operators
(``python/tencirpauli/hamiltonian.py:345-603``, built from
``PauliOperator::backend_mvp_plan``, ``crates/tencir-pauli-core/src/hamiltonian.rs:501-524``):
read-only packed ``x_words`` / ``z_words`` (canonical order) and complex128
``coefficients``, schema version 1, ``qubit0_msb_matrix`` ordering and the
``T * (16 W + 16)`` byte estimate.  Where the reference runs an independent
NumPy executor, this plan applies through the device kernels, and
``device_callable()`` returns a function on device arrays (any DLPack
producer: torch, CuPy, JAX on GPU) that never copies the state to the host
-- the role of the reference's backend MVP callable
(``python/tencirpauli/integrations/tensorcircuit.py:231``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Optional, Tuple

import numpy as np

from ._native_mvp import DEFAULT_MAX_BYTES, check_allocation, validate_max_bytes

_FACTORY = object()


def _is_capsule(value: Any) -> bool:
    """A bare DLPack capsule (``PyCapsule`` named "dltensor")."""
    return type(value).__name__ == "PyCapsule"


@dataclass(frozen=True)
class BackendMVPPlan:
    schema_version: int
    nqubits: int
    word_count: int
    x_words: np.ndarray
    z_words: np.ndarray
    coefficients: np.ndarray
    ordering: str = "qubit0_msb_matrix"
    integer_width: int = 64
    required_operations: Tuple[str, ...] = ("xor", "phase", "scatter_add")
    local_dimensions: Tuple[int, ...] = ()
    basis_ordering: str = "qubit0_msb_matrix"
    estimated_bytes: int = 0
    plan_kind: str = "pauli"
    target: str = "backend_mvp"
    _factory_token: object = field(default=None, repr=False, compare=False)
    _device_plan: Any = field(default=None, repr=False, compare=False)

    def __post_init__(self) -> None:
        if self._factory_token is not _FACTORY:
            raise TypeError("BackendMVPPlan instances must be created by a plan factory")
        for name, dtype in (("x_words", np.uint64), ("z_words", np.uint64), ("coefficients", np.complex128)):
            values = np.ascontiguousarray(getattr(self, name), dtype=dtype)
            values.setflags(write=False)
            object.__setattr__(self, name, values)
        if self.word_count != (self.nqubits + 63) // 64:
            raise ValueError("Pauli word_count does not match nqubits")
        shape = (len(self.coefficients), self.word_count)
        if self.x_words.shape != shape or self.z_words.shape != shape:
            raise ValueError("Pauli word arrays must match plan term and word counts")
        if not np.isfinite(self.coefficients).all():
            raise ValueError("backend plan coefficients must be finite")

    @classmethod
    def from_operator(cls, op: Any, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> "BackendMVPPlan":
        validate_max_bytes(max_bytes)
        width = (op.nqubits + 63) // 64
        nbytes = op.term_count * (width * 16 + 16)
        check_allocation(nbytes, max_bytes, "backend MVP plan")
        return cls(
            schema_version=1,
            nqubits=op.nqubits,
            word_count=width,
            x_words=op.x_words.reshape(op.term_count, width),
            z_words=op.z_words.reshape(op.term_count, width),
            coefficients=op.coefficients,
            local_dimensions=(2,) * op.nqubits,
            estimated_bytes=nbytes,
            _factory_token=_FACTORY,
        )

    @property
    def dimension(self) -> int:
        return 1 << self.nqubits

    @property
    def term_count(self) -> int:
        return int(self.coefficients.shape[0])

    def _plan(self) -> Any:
        if self._device_plan is None:
            from . import _native

            plan = _native.NativeMvpPlan(self.nqubits, self.x_words, self.z_words, self.coefficients)
            object.__setattr__(self, "_device_plan", plan)
        return self._device_plan

    def apply(self, state: Any, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        """H @ state.  NumPy input -> NumPy complex128 output (host copies);
        a device array -> a device array of the same dtype, no host copy."""
        validate_max_bytes(max_bytes)
        if _is_capsule(state):
            return self.device_callable()(state)
        if isinstance(state, np.ndarray) or not hasattr(state, "__dlpack__"):
            values = np.ascontiguousarray(np.asarray(state, dtype=np.complex128))
            if values.shape != (self.dimension,):
                raise ValueError(f"state must have shape ({self.dimension},), got {values.shape}")
            return self._plan().apply(values, 2**63 - 1)
        return self.device_callable()(state)

    def __call__(self, state: Any) -> Any:
        return self.apply(state)

    def device_callable(self):
        """f(x) -> H x for device arrays (complex128 or complex64, shape (2^n,)
        or (k, 2^n)) from any DLPack producer -- an object with ``__dlpack__``
        or a bare DLPack capsule; returns a torch CUDA tensor."""
        import torch

        plan = self._plan()

        def apply(x: Any) -> Any:
            if isinstance(x, torch.Tensor):
                t = x
            elif _is_capsule(x):
                t = torch.utils.dlpack.from_dlpack(x)
            else:
                t = torch.from_dlpack(x)
            if t.device.type != "cuda":
                raise ValueError("device_callable needs a device array")
            t = t.contiguous()
            y = torch.empty_like(t)
            plan.apply_device(t, y)
            return y

        return apply
