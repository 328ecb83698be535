"""The MVP entries of the reference's PyO3 module ``tencirpauli._native``,
served by ``libtcpmvp.so``.

TenCirPauli's own Python facade reaches its matrix-free MVP through four
names of its compiled extension (``python/tencirpauli/_native.pyi:98-127,
536-552`` of the reference):

* ``pauli_operator_native_array(nqubits, structures, coefficients, max_bytes)``
  and ``pauli_operator_native(nqubits, structures, re, im, max_bytes)`` ->
  ``NativePauliOperatorHandle`` (canonical operator; PyO3 code at
  ``crates/tencirpauli-native/src/operator.rs:166-270``),
* ``pauli_mvp_plan_handle(handle, max_bytes, storage="lazy")`` ->
  ``NativeMvpPlan`` (``crates/tencirpauli-native/src/hamiltonian.rs:98-116``),
* ``pauli_mvp_handle(handle, state, max_bytes)`` -> one-shot ``H @ state``
  (``hamiltonian.rs:83-96``), and
* the handle's ``nqubits``, ``term_count``, ``distinct_x_mask_count()`` and
  ``materialize()``.

A maintainer who routes the reference's facade onto the GPU binds these in
place of the PyO3 ones (for example by assigning them onto the imported
``tencirpauli._native`` module); ``PauliOperator.from_code_arrays``,
``.native_mvp_plan()``, ``.mvp()`` and ``NativeMVPPlan.apply`` /
``apply_into`` then run on the device kernels unchanged.  Canonicalization
runs in the library's host code (``tcp_pauli_canonicalize``); plans are
``tencirpauli_b200._native.NativeMvpPlan`` objects.  Error types follow the
reference's ``map_error`` (``crates/tencirpauli-native/src/convert.rs:35-42``):
MemoryLimit -> MemoryError, Overflow -> OverflowError, the rest ValueError.
"""

from __future__ import annotations

import sys
from typing import Any, Tuple

import numpy as np

from .. import _native

U64_MAX = (1 << 64) - 1


class NativePauliOperatorHandle:
    """Canonical operator handle: packed words and coefficients in the
    reference's canonical order (``operator.rs:117-155``)."""

    __slots__ = ("_nqubits", "_x", "_z", "_coefficients")

    def __init__(self, nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray) -> None:
        self._nqubits = int(nqubits)
        self._x = np.ascontiguousarray(x_words, dtype=np.uint64)
        self._z = np.ascontiguousarray(z_words, dtype=np.uint64)
        self._coefficients = np.ascontiguousarray(coefficients, dtype=np.complex128)

    @property
    def nqubits(self) -> int:
        return self._nqubits

    @property
    def term_count(self) -> int:
        return int(self._coefficients.shape[0])

    @property
    def word_count(self) -> int:
        return self._nqubits // 64 + (self._nqubits % 64 != 0)

    def distinct_x_mask_count(self) -> int:
        if self.term_count == 0:
            return 0
        return int(np.unique(self._x.reshape(self.term_count, -1), axis=0).shape[0])

    def materialize(self) -> Tuple[int, int, np.ndarray, np.ndarray, np.ndarray]:
        """(term_count, word_count, x_words, z_words, coefficients), flat words."""
        return (self.term_count, self.word_count, self._x.reshape(-1).copy(), self._z.reshape(-1).copy(),
                self._coefficients.copy())


def _check_operator_limit(term_count: int, nqubits: int, max_bytes: int) -> None:
    # operator.rs:244-266: T * (16 W + 16) bytes against max_bytes
    requested = term_count * ((nqubits + 63) // 64 * 16 + 16)
    if requested > max_bytes:
        raise MemoryError(
            f"native Pauli operator requires approximately {requested} bytes, exceeding max_bytes={max_bytes}"
        )


def pauli_operator_native_array(nqubits: int, structures: Any, coefficients: Any, max_bytes: int) -> NativePauliOperatorHandle:
    codes = np.asarray(structures)
    values = np.asarray(coefficients)
    if codes.ndim != 2 or codes.shape[1] != nqubits:
        raise ValueError(f"expected structure width {nqubits}, got {codes.shape[1] if codes.ndim == 2 else codes.shape}")
    if codes.shape[0] != values.shape[0]:
        raise ValueError(f"expected {codes.shape[0]} coefficients, got {values.shape[0]}")
    if not codes.flags.c_contiguous:
        raise ValueError("structures must be C-contiguous")
    if not values.flags.c_contiguous:
        raise ValueError("coefficients must be C-contiguous")
    x, z, c = _native.canonicalize(nqubits, codes.astype(np.uint8, copy=False), values.astype(np.complex128, copy=False))
    _check_operator_limit(int(c.shape[0]), nqubits, int(max_bytes))
    return NativePauliOperatorHandle(nqubits, x, z, c)


def pauli_operator_native(nqubits: int, structures: Any, coefficients_re: Any, coefficients_im: Any,
                          max_bytes: int) -> NativePauliOperatorHandle:
    """Code rows as sequences (``PauliOperator.from_terms``), coefficients as
    separate real and imaginary parts."""
    codes = np.zeros((len(structures), nqubits), dtype=np.uint8)
    for row, value in enumerate(structures):
        if len(value) != nqubits:
            raise ValueError(f"expected structure width {nqubits}, got {len(value)}")
        codes[row] = np.asarray(value, dtype=np.int64)
    values = np.asarray(coefficients_re, dtype=np.float64) + 1j * np.asarray(coefficients_im, dtype=np.float64)
    return pauli_operator_native_array(nqubits, codes, np.ascontiguousarray(values), max_bytes)


def pauli_mvp_plan_handle(handle: NativePauliOperatorHandle, max_bytes: int, storage: str = "lazy") -> "_native.NativeMvpPlan":
    count, width, x, z, c = handle.materialize()
    return _native.NativeMvpPlan(handle.nqubits, x.reshape(count, width), z.reshape(count, width), c,
                                 storage=storage, max_bytes=min(int(max_bytes), U64_MAX))


def pauli_mvp_handle(handle: NativePauliOperatorHandle, state: np.ndarray, max_bytes: int) -> np.ndarray:
    """``PauliOperator::mvp``: a one-shot lazy plan applied once (hamiltonian.rs:481-483)."""
    values = np.asarray(state)
    if not values.flags.c_contiguous:
        raise ValueError("state must be C-contiguous")
    plan = pauli_mvp_plan_handle(handle, sys.maxsize, "lazy")
    return plan.apply(values, max_bytes)


__all__ = [
    "NativePauliOperatorHandle",
    "pauli_mvp_handle",
    "pauli_mvp_plan_handle",
    "pauli_operator_native",
    "pauli_operator_native_array",
]
