"""``PauliOperator`` and ``NativeMVPPlan``: the Python plan/apply API of the MVP path.

Mirrors the reference's ``PauliOperator`` construction and MVP entry points
(``python/tencirpauli/pauli.py:306-560,931-1072``) and ``NativeMVPPlan``
(``python/tencirpauli/hamiltonian.py:161-342``).  Canonicalization and the
plan build run in ``libtcpmvp.so``; application runs on the GPU.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Iterable, Literal, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from ._native_mvp import (
    DEFAULT_MAX_BYTES,
    NativeMvpFacade,
    NativePlanMetadata,
    effective_max_bytes,
    validate_max_bytes,
)

_LETTERS = "IXYZ"


@dataclass(frozen=True)
class PauliWord:
    """Phase-free Pauli word held as external I/X/Y/Z codes (qubit order)."""

    codes: Tuple[int, ...]

    @property
    def nqubits(self) -> int:
        return len(self.codes)

    def to_codes(self) -> Tuple[int, ...]:
        return self.codes

    def to_string(self) -> str:
        return "".join(_LETTERS[c] for c in self.codes)


@dataclass(frozen=True)
class PauliTerm:
    word: PauliWord
    coefficient: complex


PauliInput = Union[str, Sequence[int], PauliWord]


def _word_codes(nqubits: int, word: PauliInput) -> Tuple[int, ...]:
    if isinstance(word, PauliWord):
        codes = word.codes
    elif isinstance(word, str):
        try:
            codes = tuple(_LETTERS.index(ch) for ch in word.upper())
        except ValueError:
            raise ValueError(f"Pauli strings may only contain I, X, Y, Z; got {word!r}") from None
    else:
        codes = tuple(int(c) for c in word)
    if len(codes) != nqubits:
        raise ValueError(f"expected structure length {nqubits}, got {len(codes)}")
    for index, code in enumerate(codes):
        if code < 0 or code > 3:
            raise ValueError(f"invalid Pauli code {code} at index {index}; expected 0..=3")
    return codes


def _words_to_codes(nqubits: int, x_words: np.ndarray, z_words: np.ndarray) -> np.ndarray:
    count = x_words.shape[0]
    codes = np.zeros((count, nqubits), dtype=np.uint8)
    for q in range(nqubits):
        x = (x_words[:, q // 64] >> np.uint64(q % 64)) & np.uint64(1)
        z = (z_words[:, q // 64] >> np.uint64(q % 64)) & np.uint64(1)
        codes[:, q] = np.where(x == 1, np.where(z == 1, 2, 1), np.where(z == 1, 3, 0))
    return codes


class PauliOperator:
    """Deterministic sparse Pauli operator (canonical on construction).

    Duplicate words are aggregated in IEEE-bit order, exact zeros removed and
    terms sorted by their code tuple, as ``PauliOperator::from_terms``
    (``crates/tencir-pauli-core/src/operator.rs:117-155``).
    """

    def __init__(
        self,
        nqubits: int,
        terms: Iterable[Tuple[PauliInput, complex]] = (),
        *,
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> None:
        validate_max_bytes(max_bytes)
        if not isinstance(nqubits, int) or isinstance(nqubits, bool) or nqubits < 0:
            raise ValueError("nqubits must be a non-negative integer")
        items = tuple(terms)
        codes = np.zeros((len(items), nqubits), dtype=np.uint8)
        coefficients = np.zeros(len(items), dtype=np.complex128)
        for index, (word, coefficient) in enumerate(items):
            codes[index] = _word_codes(nqubits, word)
            coefficients[index] = complex(coefficient)
        self._init_from_arrays(nqubits, codes, coefficients)

    def _init_from_arrays(self, nqubits: int, codes: np.ndarray, coefficients: np.ndarray) -> None:
        self.nqubits = int(nqubits)
        x, z, c = _native.canonicalize(nqubits, codes, coefficients)
        for array in (x, z, c):
            array.setflags(write=False)
        self._x_words, self._z_words, self._coefficients = x, z, c
        self._terms: Optional[Tuple[PauliTerm, ...]] = None

    # -- constructors -----------------------------------------------------
    @classmethod
    def from_terms(
        cls,
        nqubits: int,
        terms: Iterable[Tuple[PauliInput, complex]],
        *,
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> "PauliOperator":
        return cls(nqubits, terms, max_bytes=max_bytes)

    @classmethod
    def from_code_arrays(
        cls,
        structures: Sequence[Sequence[int]],
        coefficients: Sequence[complex],
        *,
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> "PauliOperator":
        """Array constructor: one coarse native canonicalization call."""
        validate_max_bytes(max_bytes)
        codes = np.asarray(structures)
        if codes.ndim != 2:
            raise ValueError("structures must be a two-dimensional code array")
        values = np.asarray(coefficients, dtype=np.complex128).reshape(-1)
        if values.shape[0] != codes.shape[0]:
            raise ValueError("coefficients must provide one value per structure")
        if codes.size and (codes.min() < 0 or codes.max() > 3):
            raise ValueError("Pauli codes must lie in the half-open range 0..4")
        instance = object.__new__(cls)
        instance._init_from_arrays(int(codes.shape[1]), codes.astype(np.uint8), values)
        return instance

    @classmethod
    def from_strings(
        cls, terms: Iterable[Tuple[str, complex]], *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES
    ) -> "PauliOperator":
        items = tuple(terms)
        if not items:
            raise ValueError("cannot infer nqubits from an empty term sequence")
        return cls(len(items[0][0]), items, max_bytes=max_bytes)

    @classmethod
    def empty(cls, nqubits: int) -> "PauliOperator":
        return cls(nqubits, ())

    # -- canonical content --------------------------------------------------
    @property
    def term_count(self) -> int:
        return int(self._coefficients.shape[0])

    @property
    def x_words(self) -> np.ndarray:
        return self._x_words

    @property
    def z_words(self) -> np.ndarray:
        return self._z_words

    @property
    def coefficients(self) -> np.ndarray:
        return self._coefficients

    @property
    def codes(self) -> np.ndarray:
        return _words_to_codes(self.nqubits, self._x_words, self._z_words)

    @property
    def terms(self) -> Tuple[PauliTerm, ...]:
        if self._terms is None:
            codes = self.codes
            self._terms = tuple(
                PauliTerm(PauliWord(tuple(int(c) for c in codes[i])), complex(self._coefficients[i]))
                for i in range(self.term_count)
            )
        return self._terms

    def __repr__(self) -> str:
        return f"PauliOperator(nqubits={self.nqubits}, term_count={self.term_count})"

    # -- MVP entry points -----------------------------------------------------
    def native_mvp_plan(
        self,
        *,
        storage: Literal["lazy", "eager"] = "lazy",
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> "NativeMVPPlan":
        """Compile a reusable device MVP plan (``pauli.py:985-1036`` contract)."""
        validate_max_bytes(max_bytes)
        if storage not in ("lazy", "eager"):
            raise ValueError("invalid sector: storage must be either 'eager' or 'lazy'")
        execution = _native.NativeMvpPlan(
            self.nqubits,
            self._x_words,
            self._z_words,
            self._coefficients,
            storage=storage,
            max_bytes=effective_max_bytes(max_bytes),
        )
        if execution.nqubits != self.nqubits:
            raise RuntimeError("native MVP plan has incompatible qubit count")
        if execution.term_count != self.term_count:
            raise RuntimeError("native MVP plan has incompatible term count")
        word_count = (self.nqubits + 63) // 64
        term_bytes = self.term_count * (word_count * 16 + 16)
        estimated = term_bytes
        if storage == "eager":
            estimated += execution.group_count * (1 << self.nqubits) * 16
        return NativeMVPPlan._create(self.nqubits, execution, storage, estimated)

    def mvp(self, state: Sequence[complex], *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """One-shot MVP (``PauliOperator::mvp``, hamiltonian.rs:481-483)."""
        validate_max_bytes(max_bytes)
        values = np.asarray(state, dtype=np.complex128)
        if values.ndim != 1:
            raise ValueError(f"state must be one-dimensional, got shape {values.shape}")
        execution = _native.NativeMvpPlan(
            self.nqubits, self._x_words, self._z_words, self._coefficients, storage="lazy"
        )
        return execution.apply(np.ascontiguousarray(values), effective_max_bytes(max_bytes))

    def compile(
        self,
        target: str,
        *,
        storage: Literal["lazy", "eager"] = "lazy",
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> Any:
        """Compile one named target (``pauli.py:1047-1072`` of the reference):
        ``dense``, ``coo``, ``csr``, ``native_mvp`` or ``backend_mvp``."""
        if target == "dense":
            return self.dense(max_bytes=max_bytes)
        if target == "coo":
            return self.coo(max_bytes=max_bytes)
        if target == "csr":
            return self.csr(max_bytes=max_bytes)
        if target == "native_mvp":
            return self.native_mvp_plan(storage=storage, max_bytes=max_bytes)
        if target == "backend_mvp":
            from .backend import BackendMVPPlan

            return BackendMVPPlan.from_operator(self, max_bytes=max_bytes)
        raise ValueError("target must be one of 'dense', 'coo', 'csr', 'native_mvp', or 'backend_mvp'")

    # -- materialisation (``pauli.py:866-930`` of the reference) ----------------
    def _matrix_plan(self) -> Any:
        return _native.NativeMvpPlan(self.nqubits, self._x_words, self._z_words, self._coefficients, storage="lazy")

    def dense(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> np.ndarray:
        """Bounded complex128 dense matrix, qubit 0 the most significant bit."""
        validate_max_bytes(max_bytes)
        return self._matrix_plan().dense(effective_max_bytes(max_bytes))

    def coo(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        """Deterministic, duplicate-aggregated COO arrays (rows ascending, columns
        ascending inside a row, exact zeros skipped)."""
        from ._native_mvp import COOMatrix

        validate_max_bytes(max_bytes)
        indptr, cols, vals = self._matrix_plan().sparse("coo", effective_max_bytes(max_bytes))
        dim = 1 << self.nqubits
        rows = np.repeat(np.arange(dim, dtype=np.uint64), np.diff(indptr.astype(np.int64)))
        return COOMatrix(rows, cols, vals, (dim, dim))

    def csr(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        """Deterministic CSR arrays from the canonical COO stream."""
        from ._native_mvp import CSRMatrix

        validate_max_bytes(max_bytes)
        indptr, cols, vals = self._matrix_plan().sparse("csr", effective_max_bytes(max_bytes))
        dim = 1 << self.nqubits
        return CSRMatrix(indptr, cols, vals, (dim, dim))

    def backend_mvp_plan(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        """Versioned pure-array plan (``pauli.py:953-983`` of the reference)
        whose executor runs on the device."""
        from .backend import BackendMVPPlan

        return BackendMVPPlan.from_operator(self, max_bytes=max_bytes)

    def to_scipy_linear_operator(self, *, max_bytes: Optional[int] = DEFAULT_MAX_BYTES) -> Any:
        from .integrations.scipy import to_scipy_linear_operator

        return to_scipy_linear_operator(self.native_mvp_plan(max_bytes=max_bytes), max_bytes=max_bytes)

    # -- U(1) sectors (``pauli.py:705-736,803-828`` of the reference) ----------
    def conserves_particle_number(self) -> bool:
        """[H, N] == 0 by the reference's selection rule for qubit levels (0, 1)."""
        return _native.number_commutator(self.nqubits, self._x_words, self._z_words, self._coefficients) == 0

    def restrict_charge(
        self,
        sector: Any,
        *,
        storage: Literal["lazy", "eager"] = "lazy",
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> Any:
        """Restrict a number-conserving operator to a ``U1Sector``.

        Only qubit-number sectors are part of this build; general additive
        charge sectors are not."""
        from .symmetry import U1Sector, restrict_u1

        if not isinstance(sector, U1Sector):
            raise TypeError(f"expected U1Sector, got {type(sector).__name__}")
        return restrict_u1(self, sector, storage=storage, max_bytes=max_bytes)

    def restrict_u1(
        self,
        sector: Any,
        *,
        storage: Literal["lazy", "eager"] = "lazy",
        max_bytes: Optional[int] = DEFAULT_MAX_BYTES,
    ) -> Any:
        """Deprecated alias of :meth:`restrict_charge` with a ``U1Sector``."""
        from .symmetry import U1Sector, deprecated_restrict_u1

        validate_max_bytes(max_bytes)
        if not isinstance(sector, U1Sector):
            raise TypeError(f"expected U1Sector, got {type(sector).__name__}")
        return deprecated_restrict_u1(self, sector, storage, max_bytes)


_PLAN_FACTORY_TOKEN = object()


class NativeMVPPlan(NativeMvpFacade):
    """Reusable device matrix-free MVP plan (``hamiltonian.py:161-342`` contract)."""

    def __init__(self, *args: Any, _factory_token: object = None, **kwargs: Any) -> None:
        if _factory_token is not _PLAN_FACTORY_TOKEN:
            raise TypeError("NativeMVPPlan instances must be created by a plan factory")
        self._init(*args, **kwargs)

    def _init(self, nqubits: int, execution: Any, storage: str, estimated: int) -> None:
        self.nqubits = nqubits
        self._execution = execution
        self.local_dimensions = (2,) * nqubits
        self.schema_version = 1
        self._metadata = NativePlanMetadata(
            dimension=1 << nqubits,
            term_count=execution.term_count,
            storage=storage,  # type: ignore[arg-type]
            basis_ordering="qubit0_msb_matrix",
            target="native_mvp",
            execution_family="pauli",
            native_variant=execution.native_variant,
            retained_format="compact_graph" if storage == "eager" else "compiled_actions",
            source_term_count=execution.term_count,
            schedule_count=execution.term_count,
            estimated_retained_bytes=int(estimated),
            estimated_construction_peak_bytes=int(estimated),
            transition_count=execution.transition_count if storage == "eager" else None,
        )

    @classmethod
    def _create(cls, nqubits: int, execution: Any, storage: str, estimated: int) -> "NativeMVPPlan":
        return cls(nqubits, execution, storage, estimated, _factory_token=_PLAN_FACTORY_TOKEN)

    @property
    def _native_plan(self) -> Any:
        return self._execution

    @property
    def group_count(self) -> int:
        return int(self._execution.group_count)

    # -- device-resident extensions (no host copies) ----------------------------
    def apply_device(self, x: Any, y: Any, stream: Any = None, accumulate: bool = False) -> None:
        """y <- H x (or y += H x with ``accumulate``) for torch CUDA tensors
        (complex128: FP64, complex64: FP32 Kahan)."""
        self._execution.apply_device(x, y, stream, accumulate)

    def diagonal_device(self, out: Any, stream: Any = None) -> None:
        self._execution.diagonal_device(out, stream)
