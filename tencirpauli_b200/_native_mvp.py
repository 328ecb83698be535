"""Public-call contract of native MVP plans.

Behaviour mirrors the reference facade ``python/tencirpauli/_native_mvp.py``:
the advisory ``max_bytes`` policy (16 GiB default, 1 GiB enforcement floor,
``:19-57``), the strict zero-copy ``apply_into`` buffer protocol (``:61-81``),
the shared metadata record (``:84-221``) and ``apply`` / ``apply_into`` /
``__call__`` (``:272-311``).
"""

from __future__ import annotations

import sys
from dataclasses import dataclass
from typing import Any, Literal, Optional, Sequence, Tuple

import numpy as np

DEFAULT_MAX_BYTES = 16 * 1024 * 1024 * 1024
MIN_ENFORCED_MAX_BYTES = 1024 * 1024 * 1024


def validate_max_bytes(max_bytes: Optional[int]) -> None:
    if max_bytes is not None and (
        not isinstance(max_bytes, int) or isinstance(max_bytes, bool) or max_bytes < 0
    ):
        raise ValueError("max_bytes must be a non-negative integer or None")


def enforced_max_bytes(max_bytes: Optional[int]) -> Optional[int]:
    """The limit actually enforced: values below 1 GiB (and None) are advisory."""
    validate_max_bytes(max_bytes)
    if max_bytes is None or max_bytes < MIN_ENFORCED_MAX_BYTES:
        return None
    return max_bytes


def effective_max_bytes(max_bytes: Optional[int]) -> int:
    limit = enforced_max_bytes(max_bytes)
    return sys.maxsize if limit is None else limit


def check_allocation(requested: int, limit: Optional[int], context: str) -> None:
    enforced = enforced_max_bytes(limit)
    if enforced is not None and requested > enforced:
        raise MemoryError(
            f"{context} requires approximately {requested} bytes, exceeding max_bytes={enforced}"
        )


def validate_apply_into_buffers(input_state: object, output_state: object, dimension: int) -> None:
    """The strict buffer protocol of ``apply_into``: ndarrays, complex128,
    shape ``(dimension,)``, C-contiguous, writable output, no overlap."""
    if not isinstance(input_state, np.ndarray) or not isinstance(output_state, np.ndarray):
        raise TypeError("apply_into input and output must be NumPy arrays")
    expected = np.dtype(np.complex128)
    if input_state.dtype != expected or output_state.dtype != expected:
        raise TypeError("apply_into input and output must have dtype complex128")
    for name, value in (("input", input_state), ("output", output_state)):
        if value.ndim != 1 or value.shape != (dimension,):
            raise ValueError(f"apply_into {name} must have shape ({dimension},)")
        if not value.flags.c_contiguous:
            raise ValueError(f"apply_into {name} must be C-contiguous")
    if not output_state.flags.writeable:
        raise ValueError("apply_into output must be writable")
    if np.shares_memory(input_state, output_state):
        raise ValueError("apply_into input and output must not overlap")


@dataclass(frozen=True)
class NativePlanMetadata:
    dimension: int
    term_count: int
    storage: Literal["lazy", "eager"]
    basis_ordering: str
    target: Literal["native_mvp"]
    execution_family: str
    native_variant: str
    retained_format: str
    source_term_count: int
    schedule_count: int
    estimated_retained_bytes: int
    estimated_construction_peak_bytes: int
    transition_count: Optional[int]

    def __post_init__(self) -> None:
        for name in (
            "dimension",
            "term_count",
            "source_term_count",
            "schedule_count",
            "estimated_retained_bytes",
            "estimated_construction_peak_bytes",
        ):
            value = getattr(self, name)
            if not isinstance(value, int) or isinstance(value, bool) or value < 0:
                raise ValueError(f"{name} must be a non-negative integer")
        if self.storage not in ("lazy", "eager"):
            raise ValueError("storage must be either 'eager' or 'lazy'")
        if self.target != "native_mvp":
            raise ValueError("native MVP plans must have target='native_mvp'")
        if self.transition_count is not None and (
            not isinstance(self.transition_count, int) or self.transition_count < 0
        ):
            raise ValueError("transition_count must be a non-negative integer or None")


class NativeMvpFacade:
    """Mixin implementing the shared native-plan call contract."""

    _execution: Any
    _metadata: NativePlanMetadata

    @property
    def dimension(self) -> int:
        return self._metadata.dimension

    @property
    def term_count(self) -> int:
        return self._metadata.term_count

    @property
    def storage(self) -> str:
        return self._metadata.storage

    @property
    def basis_ordering(self) -> str:
        return self._metadata.basis_ordering

    @property
    def target(self) -> str:
        return self._metadata.target

    @property
    def execution_family(self) -> str:
        return self._metadata.execution_family

    @property
    def native_variant(self) -> str:
        return self._metadata.native_variant

    @property
    def retained_format(self) -> str:
        return self._metadata.retained_format

    @property
    def source_term_count(self) -> int:
        return self._metadata.source_term_count

    @property
    def schedule_count(self) -> int:
        return self._metadata.schedule_count

    @property
    def estimated_retained_bytes(self) -> int:
        return self._metadata.estimated_retained_bytes

    @property
    def estimated_construction_peak_bytes(self) -> int:
        return self._metadata.estimated_construction_peak_bytes

    @property
    def estimated_bytes(self) -> int:
        return self._metadata.estimated_retained_bytes

    @property
    def transition_count(self) -> Optional[int]:
        return self._metadata.transition_count

    def apply(
        self, state: Sequence[complex], *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES
    ) -> np.ndarray:
        """Apply the plan through one coarse native call; returns an owned array."""
        validate_max_bytes(max_bytes)
        values = np.asarray(state, dtype=np.complex128)
        if values.ndim != 1 or values.shape[0] != self.dimension:
            raise ValueError(f"state must have shape ({self.dimension},), got {values.shape}")
        check_allocation(self.dimension * 16, max_bytes, "requested native MVP output")
        return np.asarray(
            self._execution.apply(np.ascontiguousarray(values), effective_max_bytes(max_bytes)),
            dtype=np.complex128,
            order="C",
        )

    def apply_into(
        self,
        input_state: np.ndarray,
        output_state: np.ndarray,
        *,
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> None:
        """Apply into strict caller-owned buffers without a Python state copy."""
        validate_apply_into_buffers(input_state, output_state, self.dimension)
        self._execution.apply_into(input_state, output_state, effective_max_bytes(max_bytes))

    def __call__(self, state: Sequence[complex]) -> np.ndarray:
        return self.apply(state)

    def to_scipy_linear_operator(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        from .integrations.scipy import to_scipy_linear_operator

        return to_scipy_linear_operator(self, max_bytes=max_bytes)


@dataclass(frozen=True)
class COOMatrix:
    """Coordinate arrays of a materialised operator (``hamiltonian.py:109-132``
    of the reference): ``row``, ``column``, ``data`` of equal length in the
    producing operator's order, and the logical ``shape``."""

    row: np.ndarray
    column: np.ndarray
    data: np.ndarray
    shape: Tuple[int, int]

    @property
    def value(self) -> np.ndarray:
        return self.data

    def to_scipy(self) -> Any:
        from scipy.sparse import coo_matrix

        return coo_matrix((self.data, (self.row, self.column)), shape=self.shape)


@dataclass(frozen=True)
class CSRMatrix:
    """Compressed-sparse-row arrays (``hamiltonian.py:135-158`` of the
    reference): ``indptr``, ``indices``, ``data`` and ``shape``."""

    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray
    shape: Tuple[int, int]

    @property
    def value(self) -> np.ndarray:
        return self.data

    def to_scipy(self) -> Any:
        from scipy.sparse import csr_matrix

        return csr_matrix((self.data, self.indices, self.indptr), shape=self.shape)
