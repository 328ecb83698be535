"""Fixed-particle-number (U(1)) sectors and restricted device MVP plans.

Mirrors the U(1) part of the reference's ``python/tencirpauli/symmetry.py``
(``U1Sector`` ``:140-260``, ``U1RestrictedOperator`` ``:263-537``,
``U1MvpPlan`` ``:540-592``, ``_restrict_u1`` ``:655-706``) on top of the
sector plans of ``libtcpmvp.so`` (``include/tcp_sector.h``).  A sector keeps
the computational basis states with exactly ``particle_number`` ones, in
ascending TensorCircuit integer order; restricted states have length
``C(nqubits, particle_number)``.  Every apply runs the CUDA sector kernel.
"""

from __future__ import annotations

import math
import threading
import warnings
from dataclasses import dataclass
from typing import Any, Literal, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from ._native_mvp import (
    DEFAULT_MAX_BYTES,
    COOMatrix,
    CSRMatrix,
    NativeMvpFacade,
    NativePlanMetadata,
    check_allocation,
    effective_max_bytes,
    enforced_max_bytes,
    validate_apply_into_buffers,
    validate_max_bytes,
)

U1Storage = Literal["lazy", "eager"]


def _coerce_bitstring(nqubits: int, bitstring: Union[int, Sequence[int]]) -> int:
    if isinstance(bitstring, bool):
        raise TypeError("bitstring must be an integer or a sequence of bits")
    if isinstance(bitstring, (int, np.integer)):
        value = int(bitstring)
    else:
        bits = tuple(bitstring)
        if len(bits) != nqubits or any(bit not in (0, 1) for bit in bits):
            raise ValueError("bitstring must contain exactly nqubits binary values")
        value = 0
        for bit in bits:
            value = (value << 1) | int(bit)
    if value < 0 or value.bit_length() > nqubits:
        raise ValueError("bitstring is outside the computational basis")
    return value


@dataclass(frozen=True)
class U1Sector:
    """Fixed-Hamming-weight basis with TensorCircuit integer ordering."""

    nqubits: int
    particle_number: int

    def __post_init__(self) -> None:
        if not isinstance(self.nqubits, int) or isinstance(self.nqubits, bool) or self.nqubits < 0:
            raise ValueError("nqubits must be a non-negative integer")
        if (
            not isinstance(self.particle_number, int)
            or isinstance(self.particle_number, bool)
            or not 0 <= self.particle_number <= self.nqubits
        ):
            raise ValueError("particle_number must be between 0 and nqubits")
        dimension = math.comb(self.nqubits, self.particle_number)
        if dimension > np.iinfo(np.uint64).max:
            raise OverflowError("U1 sector dimension exceeds uint64 restricted indices")
        if dimension > np.iinfo(np.intp).max:
            raise OverflowError("U1 sector dimension exceeds platform indices")

    @property
    def dimension(self) -> int:
        """``C(nqubits, particle_number)``."""
        return math.comb(self.nqubits, self.particle_number)

    def rank(self, bitstring: Union[int, Sequence[int]]) -> int:
        """Position of a basis state in the sector order (no basis materialised)."""
        value = _coerce_bitstring(self.nqubits, bitstring)
        if bin(value).count("1") != self.particle_number:
            raise ValueError("bitstring has the wrong Hamming weight")
        # Scan qubits from 0 (the most significant bit): each set qubit counts
        # the states that agree before it, leave it clear and put every
        # remaining one after it.
        rank, left = 0, self.particle_number
        for qubit in range(self.nqubits):
            if (value >> (self.nqubits - 1 - qubit)) & 1:
                rank += math.comb(self.nqubits - qubit - 1, left)
                left -= 1
        return rank

    def unrank(self, index: int) -> Tuple[int, ...]:
        """Occupation bits (qubit 0 first) of the state at a restricted index."""
        if not isinstance(index, (int, np.integer)) or isinstance(index, bool) or not 0 <= int(index) < self.dimension:
            raise IndexError("restricted basis index is out of range")
        rest, left = int(index), self.particle_number
        bits = []
        for qubit in range(self.nqubits):
            clear = math.comb(self.nqubits - qubit - 1, left)
            if rest >= clear:
                rest -= clear
                left -= 1
                bits.append(1)
            else:
                bits.append(0)
        return tuple(bits)

    def basis_states(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """Read-only ``uint8`` rows (qubit 0 first) in sector order."""
        validate_max_bytes(max_bytes)
        check_allocation(self.dimension * self.nqubits, max_bytes, "U1 basis states")
        if self.nqubits == 0:
            result = np.zeros((self.dimension, 0), dtype=np.uint8)
        else:
            _, width, words = _native.u1_basis_words(self.nqubits, self.particle_number, effective_max_bytes(max_bytes))
            words = words.reshape(self.dimension, width)
            if self.nqubits <= 64:
                shifts = np.arange(self.nqubits - 1, -1, -1, dtype=np.uint64)
                result = ((words[:, :1] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)
            else:
                q = np.arange(self.nqubits)
                result = ((words[:, q // 64] >> (q % 64).astype(np.uint64)) & np.uint64(1)).astype(np.uint8)
        result.flags.writeable = False
        return result

    def basis_words_packed(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """Read-only ``uint64`` basis: TensorCircuit integers for n <= 64, else
        packed occupation words (qubit q at word q // 64, bit q % 64)."""
        validate_max_bytes(max_bytes)
        dimension, width, words = _native.u1_basis_words(
            self.nqubits, self.particle_number, effective_max_bytes(max_bytes)
        )
        result = np.asarray(words, dtype=np.uint64).reshape((dimension, width))
        result.flags.writeable = False
        return result


def _materialization_bytes(dimension: int, transition_count: int, target: str) -> int:
    if target == "dense":
        return dimension * dimension * 16
    if target == "coo":
        return transition_count * 32
    if target == "csr":
        return (dimension + 1) * 8 + transition_count * 24
    raise ValueError(f"unsupported U1 materialization target: {target}")


class U1RestrictedOperator:
    """A number-conserving Pauli operator restricted to one U(1) sector.

    ``storage="lazy"`` keeps the compiled groups only; ``"eager"`` also scans
    every source for leakage and counts the restricted matrix's entries.  Both
    apply through the same device kernel.
    """

    def __init__(self, sector: U1Sector, operator: Any, *, storage: U1Storage = "lazy",
                 native_plan: Optional[_native.NativeU1Plan] = None) -> None:
        if storage not in ("lazy", "eager"):
            raise ValueError("storage must be either 'eager' or 'lazy'")
        self.sector = sector
        self.dimension = sector.dimension
        self.term_count = operator.term_count
        self.storage = storage
        self._operator = operator
        self._lock = threading.Lock()
        self._plans: dict = {}
        if native_plan is not None:
            self._plans[native_plan.storage] = native_plan

    def _plan(self, storage: str, max_bytes: Optional[int]) -> _native.NativeU1Plan:
        with self._lock:
            plan = self._plans.get(storage)
            if plan is None:
                op = self._operator
                plan = _native.NativeU1Plan(
                    self.sector.nqubits,
                    self.sector.particle_number,
                    op._x_words,
                    op._z_words,
                    op._coefficients,
                    storage=storage,
                    max_bytes=effective_max_bytes(max_bytes),
                )
                self._plans[storage] = plan
            return plan

    @property
    def _native_plan(self) -> _native.NativeU1Plan:
        return self._plan(self.storage, None)

    @property
    def estimated_bytes(self) -> int:
        plan = self._native_plan
        if plan.transition_count is not None:
            return plan.estimated_bytes + plan.transition_count * 32
        return plan.estimated_bytes

    def apply(self, state: Sequence[complex], *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """Apply to a restricted state (length ``dimension``)."""
        validate_max_bytes(max_bytes)
        values = np.asarray(state, dtype=np.complex128)
        if values.ndim != 1 or values.shape[0] != self.dimension:
            raise ValueError(f"state must have shape ({self.dimension},), got {values.shape}")
        return self._native_plan.apply(np.ascontiguousarray(values), effective_max_bytes(max_bytes))

    def apply_into(self, input_state: np.ndarray, output_state: np.ndarray, *,
                   max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> None:
        validate_apply_into_buffers(input_state, output_state, self.dimension)
        self._native_plan.apply_into(input_state, output_state, effective_max_bytes(max_bytes))

    def mvp_plan(self, *, storage: U1Storage = "lazy", max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> "U1MvpPlan":
        """A reusable restricted matrix-free plan."""
        validate_max_bytes(max_bytes)
        if storage not in ("lazy", "eager"):
            raise ValueError("storage must be either 'eager' or 'lazy'")
        plan = self._plan(storage, max_bytes)
        if storage == "lazy":
            check_allocation(plan.estimated_bytes, max_bytes, "U1 MVP plan")
        return U1MvpPlan._create(self.sector, plan, self.term_count, storage)

    def _csr_arrays(self, max_bytes: Optional[int], target: str):
        plan = self._plan("eager", max_bytes)
        check_allocation(
            _materialization_bytes(self.dimension, int(plan.transition_count or 0), target), max_bytes,
            f"U1 {target} materialization",
        )
        return plan.csr(effective_max_bytes(max_bytes))

    def dense(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """Dense restricted matrix (rows: destinations, sector order)."""
        validate_max_bytes(max_bytes)
        check_allocation(self.dimension * self.dimension * 16, max_bytes, "U1 dense materialization")
        dim, indptr, cols, vals = self._csr_arrays(max_bytes, "dense")
        out = np.zeros((dim, dim), dtype=np.complex128)
        rows = np.repeat(np.arange(dim, dtype=np.int64), np.diff(indptr.astype(np.int64)))
        out[rows, cols.astype(np.int64)] = vals
        return out

    def coo(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> COOMatrix:
        validate_max_bytes(max_bytes)
        dim, indptr, cols, vals = self._csr_arrays(max_bytes, "coo")
        rows = np.repeat(np.arange(dim, dtype=np.uint64), np.diff(indptr.astype(np.int64)))
        return COOMatrix(rows, cols.astype(np.uint64), vals, (dim, dim))

    def csr(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> CSRMatrix:
        validate_max_bytes(max_bytes)
        dim, indptr, cols, vals = self._csr_arrays(max_bytes, "csr")
        return CSRMatrix(indptr, cols.astype(np.uint64), vals, (dim, dim))

    def compile(self, target: str, *, storage: U1Storage = "lazy",
                max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        """``dense`` / ``coo`` / ``csr`` / ``native_mvp`` (``symmetry.py:505-537``)."""
        if target == "dense":
            return self.dense(max_bytes=max_bytes)
        if target == "coo":
            return self.coo(max_bytes=max_bytes)
        if target == "csr":
            return self.csr(max_bytes=max_bytes)
        if target == "native_mvp":
            return self.mvp_plan(storage=storage, max_bytes=max_bytes)
        raise ValueError("target must be one of 'dense', 'coo', 'csr', or 'native_mvp'")


_U1_FACTORY_TOKEN = object()


class U1MvpPlan(NativeMvpFacade):
    """Reusable device matrix-free plan over a fixed-particle-number basis."""

    def __init__(self, *args: Any, _factory_token: object = None, **kwargs: Any) -> None:
        if _factory_token is not _U1_FACTORY_TOKEN:
            raise TypeError("U1MvpPlan instances must be created by U1RestrictedOperator.mvp_plan")
        self._init(*args, **kwargs)

    def _init(self, sector: U1Sector, execution: _native.NativeU1Plan, term_count: int, storage: str) -> None:
        self.sector = sector
        self._execution = execution
        dimension = execution.dimension
        transitions = execution.transition_count if storage == "eager" else None
        retained = (
            execution.estimated_bytes
            if storage == "lazy"
            else dimension * 16 + (dimension + 1) * 8 + int(transitions or 0) * 32
        )
        self._metadata = NativePlanMetadata(
            dimension=dimension,
            term_count=int(term_count),
            storage=storage,  # type: ignore[arg-type]
            basis_ordering="qubit0_msb_matrix",
            target="native_mvp",
            execution_family="product",
            native_variant=execution.native_variant,
            retained_format="compiled_actions",
            source_term_count=int(term_count),
            schedule_count=int(term_count),
            estimated_retained_bytes=int(retained),
            estimated_construction_peak_bytes=int(retained),
            transition_count=transitions,
        )

    @classmethod
    def _create(cls, sector: U1Sector, execution: _native.NativeU1Plan, term_count: int, storage: str) -> "U1MvpPlan":
        return cls(sector, execution, term_count, storage, _factory_token=_U1_FACTORY_TOKEN)

    @property
    def _native_plan(self) -> _native.NativeU1Plan:
        return self._execution

    @property
    def nqubits(self) -> int:
        return self.sector.nqubits

    def apply_device(self, x: Any, y: Any, stream: Any = None) -> None:
        """y <- H x on torch CUDA tensors of restricted length."""
        self._execution.apply_device(x, y, stream)

    def diagonal_device(self, out: Any, stream: Any = None) -> None:
        self._execution.diagonal_device(out, stream)


def restrict_u1(operator: Any, sector: U1Sector, *, storage: U1Storage = "lazy",
                max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> U1RestrictedOperator:
    """``_restrict_u1`` (``symmetry.py:655-706``): lazy restriction requires an
    exactly number-conserving operator ([H, N] = 0 by the reference's selection
    rule); eager restriction scans the sector's sources for leakage instead."""
    validate_max_bytes(max_bytes)
    if storage not in ("lazy", "eager"):
        raise ValueError("storage must be either 'eager' or 'lazy'")
    if not isinstance(sector, U1Sector):
        raise TypeError(f"expected U1Sector, got {type(sector).__name__}")
    if sector.nqubits != operator.nqubits:
        raise ValueError(f"expected sector for {operator.nqubits} qubits, got {sector.nqubits}")
    if storage == "lazy":
        nonzero = _native.number_commutator(operator.nqubits, operator._x_words, operator._z_words,
                                            operator._coefficients)
        if nonzero:
            raise ValueError(
                "selected U1 sector requires an exactly conserved operator; "
                "nonzero U(1) sector leakage was detected"
            )
    restricted = U1RestrictedOperator(sector, operator, storage=storage)
    restricted._plan(storage, max_bytes)  # build (and, eager, validate) now
    return restricted


def deprecated_restrict_u1(operator: Any, sector: U1Sector, storage: U1Storage,
                           max_bytes: Optional[int]) -> U1RestrictedOperator:
    warnings.warn(
        "PauliOperator.restrict_u1() is deprecated; use restrict_charge(U1Sector(...)) instead",
        DeprecationWarning,
        stacklevel=3,
    )
    return restrict_u1(operator, sector, storage=storage, max_bytes=max_bytes)


__all__ = ["U1Sector", "U1RestrictedOperator", "U1MvpPlan", "restrict_u1"]
