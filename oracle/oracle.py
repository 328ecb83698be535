"""CPU oracle bindings -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper over ``oracle/_build/libmvp_oracle.so`` (the plain-C
restatement of TenCirPauli's Rust MVP in ``oracle/mvp_oracle.c``).  Only the
test-suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference arms may import this module, and only as the checker or as the timed
CPU baseline; the product library never calls it.

Every function restates one reference item (paths inside the reference
project ``crates/tencir-pauli-core/src``):

* :func:`encode_codes`       -- ``word.rs:94-110`` (``PauliWord::from_codes``)
* :func:`canonicalize`       -- ``operator.rs:117-155`` (``PauliOperator::from_terms``)
* :func:`matrix_terms`       -- ``pauli_action.rs:24-88`` + ``hamiltonian.rs:564-571``
* :func:`apply_term_direct`  -- ``hamiltonian.rs:204-270`` (TermDirect, lazy plan)
* :func:`apply_xmask_diagonal` -- ``hamiltonian.rs:79-147,233-235`` (eager plan)
* :func:`transition_count`   -- ``hamiltonian.rs:166-179``
* :func:`apply_rows`         -- the TermDirect row loop on selected rows only
* :func:`dense`              -- ``hamiltonian.rs:313-355`` (``dense_matrix``)
* :func:`csr`                -- ``hamiltonian.rs:584-752`` (sparse rows, sorted columns)

U(1) sector items (``oracle/u1_oracle.c``, paths in ``sector.rs``):

* :func:`u1_dimension` / :func:`u1_rank` / :func:`u1_unrank` -- ``:79-238,310-341``
* :func:`u1_apply`           -- ``U1LazyMvpPlan::apply_into`` (``:579-643``)
* :func:`u1_csr`             -- ``U1RestrictedOperator::new`` / ``csr`` (``:345-431``)
* :func:`number_commutator`  -- ``operator.rs:396-444`` with levels (0, 1)
* :func:`u1_apply_rows`      -- selected rows of the restricted MVP (CPU baseline sample)
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libmvp_oracle.so")
_lib: Optional[ctypes.CDLL] = None

_u8p = ctypes.POINTER(ctypes.c_uint8)
_u64p = ctypes.POINTER(ctypes.c_uint64)
_f64p = ctypes.POINTER(ctypes.c_double)


def build() -> str:
    """Compile the oracle library with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        lib.oracle_encode_codes.argtypes = [u32, u64, _u8p, _u64p, _u64p]
        lib.oracle_canonicalize.argtypes = [u32, u64, _u8p, _f64p, _u64p, _u64p, _f64p, _u64p, _u64p]
        lib.oracle_matrix_terms.argtypes = [u32, u64, _u64p, _u64p, _f64p, _u64p, _u64p, _f64p]
        lib.oracle_apply_term_direct.argtypes = [u32, u64, _u64p, _u64p, _f64p, _f64p, _f64p, i32]
        lib.oracle_apply_rows.argtypes = [u32, u64, _u64p, _u64p, _f64p, _f64p, u64, _u64p, _f64p, i32]
        lib.oracle_apply_xmask_diagonal.argtypes = [u32, u64, _u64p, _u64p, _f64p, _f64p, _f64p, _u64p, i32]
        lib.oracle_transition_count.argtypes = [u32, u64, _u64p, _u64p, _f64p, _u64p, i32]
        lib.oracle_group_count.argtypes = [u64, _u64p]
        lib.oracle_group_count.restype = u64
        lib.oracle_packed_word_count.argtypes = [u32]
        lib.oracle_packed_word_count.restype = u32
        lib.oracle_max_threads.restype = i32
        lib.oracle_dense.argtypes = [u32, u64, _u64p, _u64p, _f64p, _f64p]
        lib.oracle_csr.argtypes = [u32, u64, _u64p, _u64p, _f64p, _u64p, _u64p, _f64p, u64, _u64p]
        lib.oracle_dense.restype = i32
        lib.oracle_csr.restype = i32
        lib.oracle_u1_dimension.argtypes = [u32, u32, _u64p]
        lib.oracle_u1_rank.argtypes = [u32, u32, _u64p, _u64p]
        lib.oracle_u1_unrank.argtypes = [u32, u32, u64, _u64p]
        lib.oracle_u1_apply.argtypes = [u32, u32, u64, _u64p, _u64p, _f64p, _f64p, _f64p, _u64p, _u64p]
        lib.oracle_u1_csr.argtypes = [u32, u32, u64, _u64p, _u64p, _f64p, _u64p, _u64p, _f64p, u64, _u64p, _u64p, _u64p]
        lib.oracle_number_commutator.argtypes = [u32, u64, _u64p, _u64p, _f64p, _u64p]
        lib.oracle_u1_apply_rows.argtypes = [u32, u32, u64, _u64p, _u64p, _f64p, _f64p, u64, _u64p, _f64p, i32]
        for name in ("oracle_u1_dimension", "oracle_u1_rank", "oracle_u1_unrank", "oracle_u1_apply",
                     "oracle_u1_csr", "oracle_number_commutator", "oracle_u1_apply_rows"):
            getattr(lib, name).restype = i32
        for name in (
            "oracle_encode_codes",
            "oracle_canonicalize",
            "oracle_matrix_terms",
            "oracle_apply_term_direct",
            "oracle_apply_rows",
            "oracle_apply_xmask_diagonal",
            "oracle_transition_count",
        ):
            getattr(lib, name).restype = i32
        _lib = lib
    return _lib


def _p(array: np.ndarray, ptype):  # type: ignore[no-untyped-def]
    return array.ctypes.data_as(ptype)


class OracleError(RuntimeError):
    def __init__(self, status: int, detail: str = "") -> None:
        super().__init__(f"oracle status {status} {detail}".strip())
        self.status = status


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def packed_word_count(nqubits: int) -> int:
    return int(_load().oracle_packed_word_count(nqubits))


def encode_codes(nqubits: int, codes: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    codes = np.ascontiguousarray(codes, dtype=np.uint8).reshape(-1, nqubits) if nqubits else np.zeros((len(codes), 0), np.uint8)
    count = codes.shape[0]
    width = packed_word_count(nqubits)
    x = np.zeros((count, width), dtype=np.uint64)
    z = np.zeros((count, width), dtype=np.uint64)
    status = _load().oracle_encode_codes(nqubits, count, _p(codes, _u8p), _p(x, _u64p), _p(z, _u64p))
    if status:
        raise OracleError(status)
    return x, z


def canonicalize(
    nqubits: int, codes: np.ndarray, coefficients: np.ndarray
) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Return canonical (x_words[T,W], z_words[T,W], coefficients[T])."""
    count = len(coefficients)
    codes = np.ascontiguousarray(np.asarray(codes, dtype=np.uint8).reshape(count, nqubits))
    coeffs = np.ascontiguousarray(np.asarray(coefficients, dtype=np.complex128))
    width = packed_word_count(nqubits)
    x = np.zeros((max(count, 1), width), dtype=np.uint64)
    z = np.zeros((max(count, 1), width), dtype=np.uint64)
    out = np.zeros(max(count, 1), dtype=np.complex128)
    n_out = np.zeros(1, dtype=np.uint64)
    bad = np.zeros(1, dtype=np.uint64)
    status = _load().oracle_canonicalize(
        nqubits,
        count,
        _p(codes, _u8p),
        _p(coeffs.view(np.float64), _f64p),
        _p(x, _u64p),
        _p(z, _u64p),
        _p(out.view(np.float64), _f64p),
        _p(n_out, _u64p),
        _p(bad, _u64p),
    )
    if status:
        raise OracleError(status, f"index {int(bad[0])}")
    t = int(n_out[0])
    return x[:t].copy(), z[:t].copy(), out[:t].copy()


def matrix_terms(
    nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray
) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Return (x_mask, z_mask, weighted_phase) in the MSB matrix index space."""
    count = len(coefficients)
    xw = np.ascontiguousarray(x_words, dtype=np.uint64)
    zw = np.ascontiguousarray(z_words, dtype=np.uint64)
    coeffs = np.ascontiguousarray(coefficients, dtype=np.complex128)
    xm = np.zeros(max(count, 1), dtype=np.uint64)
    zm = np.zeros(max(count, 1), dtype=np.uint64)
    wp = np.zeros(max(count, 1), dtype=np.complex128)
    status = _load().oracle_matrix_terms(
        nqubits,
        count,
        _p(xw, _u64p),
        _p(zw, _u64p),
        _p(coeffs.view(np.float64), _f64p),
        _p(xm, _u64p),
        _p(zm, _u64p),
        _p(wp.view(np.float64), _f64p),
    )
    if status:
        raise OracleError(status)
    return xm[:count].copy(), zm[:count].copy(), wp[:count].copy()


def apply_term_direct(
    nqubits: int,
    x_mask: np.ndarray,
    z_mask: np.ndarray,
    weighted: np.ndarray,
    state: np.ndarray,
    threads: int = 0,
) -> np.ndarray:
    state = np.ascontiguousarray(state, dtype=np.complex128)
    if state.shape != (1 << nqubits,):
        raise ValueError("state length must be 2**nqubits")
    out = np.empty_like(state)
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    wp = np.ascontiguousarray(weighted, dtype=np.complex128)
    status = _load().oracle_apply_term_direct(
        nqubits,
        len(wp),
        _p(xm, _u64p),
        _p(zm, _u64p),
        _p(wp.view(np.float64), _f64p),
        _p(state.view(np.float64), _f64p),
        _p(out.view(np.float64), _f64p),
        threads,
    )
    if status:
        raise OracleError(status)
    return out


def apply_rows(
    nqubits: int,
    x_mask: np.ndarray,
    z_mask: np.ndarray,
    weighted: np.ndarray,
    state: np.ndarray,
    rows: np.ndarray,
    threads: int = 0,
) -> np.ndarray:
    state = np.ascontiguousarray(state, dtype=np.complex128)
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    if rows.size and int(rows.max()) >= (1 << nqubits):
        raise ValueError("row index out of range")
    out = np.empty(len(rows), dtype=np.complex128)
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    wp = np.ascontiguousarray(weighted, dtype=np.complex128)
    status = _load().oracle_apply_rows(
        nqubits,
        len(wp),
        _p(xm, _u64p),
        _p(zm, _u64p),
        _p(wp.view(np.float64), _f64p),
        _p(state.view(np.float64), _f64p),
        len(rows),
        _p(rows, _u64p),
        _p(out.view(np.float64), _f64p),
        threads,
    )
    if status:
        raise OracleError(status)
    return out


def apply_xmask_diagonal(
    nqubits: int,
    x_mask: np.ndarray,
    z_mask: np.ndarray,
    weighted: np.ndarray,
    state: np.ndarray,
    threads: int = 0,
) -> Tuple[np.ndarray, int]:
    state = np.ascontiguousarray(state, dtype=np.complex128)
    out = np.empty_like(state)
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    wp = np.ascontiguousarray(weighted, dtype=np.complex128)
    transitions = np.zeros(1, dtype=np.uint64)
    status = _load().oracle_apply_xmask_diagonal(
        nqubits,
        len(wp),
        _p(xm, _u64p),
        _p(zm, _u64p),
        _p(wp.view(np.float64), _f64p),
        _p(state.view(np.float64), _f64p),
        _p(out.view(np.float64), _f64p),
        _p(transitions, _u64p),
        threads,
    )
    if status:
        raise OracleError(status)
    return out, int(transitions[0])


def transition_count(
    nqubits: int, x_mask: np.ndarray, z_mask: np.ndarray, weighted: np.ndarray, threads: int = 0
) -> int:
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    wp = np.ascontiguousarray(weighted, dtype=np.complex128)
    out = np.zeros(1, dtype=np.uint64)
    status = _load().oracle_transition_count(
        nqubits, len(wp), _p(xm, _u64p), _p(zm, _u64p), _p(wp.view(np.float64), _f64p), _p(out, _u64p), threads
    )
    if status:
        raise OracleError(status)
    return int(out[0])


def group_count(x_mask: np.ndarray) -> int:
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    return int(_load().oracle_group_count(len(xm), _p(xm, _u64p)))


def mvp(nqubits: int, codes: np.ndarray, coefficients: np.ndarray, state: np.ndarray, threads: int = 0) -> np.ndarray:
    """One-shot ``PauliOperator::mvp`` (hamiltonian.rs:481-483): canonicalize, compile, apply."""
    xw, zw, c = canonicalize(nqubits, codes, coefficients)
    xm, zm, wp = matrix_terms(nqubits, xw, zw, c)
    return apply_term_direct(nqubits, xm, zm, wp, state, threads)


# --------------------------- U(1) sector oracle ------------------------------
class OracleLeakage(OracleError):
    """``PauliError::SectorLeakage``: the lowest leaking source and its weight."""

    def __init__(self, source: int, weight: int) -> None:
        super().__init__(11, f"leakage from source {source} to weight {weight}")
        self.source = source
        self.weight = weight


def u1_dimension(nqubits: int, particle_number: int) -> int:
    out = np.zeros(1, np.uint64)
    status = _load().oracle_u1_dimension(nqubits, particle_number, _p(out, _u64p))
    if status:
        raise OracleError(status)
    return int(out[0])


def u1_rank(nqubits: int, particle_number: int, words: np.ndarray) -> int:
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
    if w.size == 0:
        w = np.zeros(1, np.uint64)
    out = np.zeros(1, np.uint64)
    status = _load().oracle_u1_rank(nqubits, particle_number, _p(w, _u64p), _p(out, _u64p))
    if status:
        raise OracleError(status)
    return int(out[0])


def u1_unrank(nqubits: int, particle_number: int, index: int) -> np.ndarray:
    out = np.zeros(max(packed_word_count(nqubits), 1), np.uint64)
    status = _load().oracle_u1_unrank(nqubits, particle_number, index, _p(out, _u64p))
    if status:
        raise OracleError(status)
    return out[: packed_word_count(nqubits)]


def _u1_terms(nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray):
    count = int(len(coefficients))
    width = max(packed_word_count(nqubits), 1)
    xw = np.zeros((max(count, 1), width), np.uint64)
    zw = np.zeros((max(count, 1), width), np.uint64)
    if count and packed_word_count(nqubits):
        xw[:count] = np.asarray(x_words, np.uint64).reshape(count, -1)
        zw[:count] = np.asarray(z_words, np.uint64).reshape(count, -1)
    if packed_word_count(nqubits) == 0:  # n = 0: no words at all
        xw = np.zeros(1, np.uint64)
        zw = np.zeros(1, np.uint64)
    c = np.zeros(max(count, 1), np.complex128)
    c[:count] = coefficients
    return count, np.ascontiguousarray(xw), np.ascontiguousarray(zw), c


def u1_apply(nqubits: int, particle_number: int, x_words: np.ndarray, z_words: np.ndarray,
             coefficients: np.ndarray, state: np.ndarray) -> np.ndarray:
    """Restricted MVP of the canonical operator (packed x/z words, coefficients)."""
    count, xw, zw, c = _u1_terms(nqubits, x_words, z_words, coefficients)
    dim = u1_dimension(nqubits, particle_number)
    x = np.ascontiguousarray(state, dtype=np.complex128)
    if x.shape != (dim,):
        raise ValueError(f"state must have shape ({dim},)")
    out = np.zeros(dim, np.complex128)
    ls = np.zeros(1, np.uint64)
    lw = np.zeros(1, np.uint64)
    status = _load().oracle_u1_apply(nqubits, particle_number, count, _p(xw, _u64p), _p(zw, _u64p),
                                     _p(c.view(np.float64), _f64p), _p(x.view(np.float64), _f64p),
                                     _p(out.view(np.float64), _f64p), _p(ls, _u64p), _p(lw, _u64p))
    if status == 11:
        raise OracleLeakage(int(ls[0]), int(lw[0]))
    if status:
        raise OracleError(status)
    return out


def u1_csr(nqubits: int, particle_number: int, x_words: np.ndarray, z_words: np.ndarray,
           coefficients: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Destination-major CSR (indptr, columns, values) of the restricted operator."""
    count, xw, zw, c = _u1_terms(nqubits, x_words, z_words, coefficients)
    dim = u1_dimension(nqubits, particle_number)
    lib = _load()
    indptr = np.zeros(dim + 1, np.uint64)
    nnz = np.zeros(1, np.uint64)
    ls = np.zeros(1, np.uint64)
    lw = np.zeros(1, np.uint64)
    one = np.zeros(1, np.uint64)
    onev = np.zeros(2, np.float64)
    args = (nqubits, particle_number, count, _p(xw, _u64p), _p(zw, _u64p), _p(c.view(np.float64), _f64p))
    status = lib.oracle_u1_csr(*args, _p(indptr, _u64p), _p(one, _u64p), _p(onev, _f64p), 0, _p(nnz, _u64p),
                               _p(ls, _u64p), _p(lw, _u64p))
    if status == 11:
        raise OracleLeakage(int(ls[0]), int(lw[0]))
    if status:
        raise OracleError(status)
    m = int(nnz[0])
    cols = np.zeros(max(m, 1), np.uint64)
    vals = np.zeros(max(m, 1), np.complex128)
    status = lib.oracle_u1_csr(*args, _p(indptr, _u64p), _p(cols, _u64p), _p(vals.view(np.float64), _f64p), m,
                               _p(nnz, _u64p), _p(ls, _u64p), _p(lw, _u64p))
    if status:
        raise OracleError(status)
    return indptr, cols[:m], vals[:m]


def number_commutator(nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray) -> int:
    """Nonzero commutator words of [H, N] (0 iff H conserves the particle number)."""
    count, xw, zw, c = _u1_terms(nqubits, x_words, z_words, coefficients)
    out = np.zeros(1, np.uint64)
    status = _load().oracle_number_commutator(nqubits, count, _p(xw, _u64p), _p(zw, _u64p),
                                              _p(c.view(np.float64), _f64p), _p(out, _u64p))
    if status:
        raise OracleError(status)
    return int(out[0])


def u1_apply_rows(nqubits: int, particle_number: int, x_words: np.ndarray, z_words: np.ndarray,
                  coefficients: np.ndarray, state: np.ndarray, rows: np.ndarray, threads: int = 0) -> np.ndarray:
    """Rows ``rows`` (restricted indices) of the restricted MVP, pulled from their sources."""
    count, xw, zw, c = _u1_terms(nqubits, x_words, z_words, coefficients)
    x = np.ascontiguousarray(state, dtype=np.complex128)
    r = np.ascontiguousarray(rows, dtype=np.uint64)
    out = np.zeros(max(len(r), 1), np.complex128)
    status = _load().oracle_u1_apply_rows(nqubits, particle_number, count, _p(xw, _u64p), _p(zw, _u64p),
                                          _p(c.view(np.float64), _f64p), _p(x.view(np.float64), _f64p), len(r),
                                          _p(r if len(r) else np.zeros(1, np.uint64), _u64p),
                                          _p(out.view(np.float64), _f64p), threads or max_threads())
    if status:
        raise OracleError(status)
    return out[: len(r)]


def dense(nqubits: int, x_mask: np.ndarray, z_mask: np.ndarray, weighted: np.ndarray) -> np.ndarray:
    """Dense row-major matrix (``PauliOperator::dense_matrix``)."""
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    w = np.ascontiguousarray(weighted, dtype=np.complex128)
    dim = 1 << nqubits
    out = np.zeros((dim, dim), np.complex128)
    status = _load().oracle_dense(nqubits, len(xm), _p(xm if len(xm) else np.zeros(1, np.uint64), _u64p),
                                  _p(zm if len(zm) else np.zeros(1, np.uint64), _u64p),
                                  _p((w if len(w) else np.zeros(1, np.complex128)).view(np.float64), _f64p),
                                  _p(out.view(np.float64), _f64p))
    if status:
        raise OracleError(status)
    return out


def csr(nqubits: int, x_mask: np.ndarray, z_mask: np.ndarray, weighted: np.ndarray):
    """(indptr, columns, values) of the sparse rows (``sparse_entries``)."""
    xm = np.ascontiguousarray(x_mask, dtype=np.uint64)
    zm = np.ascontiguousarray(z_mask, dtype=np.uint64)
    w = np.ascontiguousarray(weighted, dtype=np.complex128)
    if len(xm) == 0:
        xm = np.zeros(1, np.uint64); zm = np.zeros(1, np.uint64); w = np.zeros(1, np.complex128)
        count = 0
    else:
        count = len(xm)
    dim = 1 << nqubits
    indptr = np.zeros(dim + 1, np.uint64)
    nnz = np.zeros(1, np.uint64)
    lib = _load()
    one_c, one_v = np.zeros(1, np.uint64), np.zeros(2, np.float64)
    lib.oracle_csr(nqubits, count, _p(xm, _u64p), _p(zm, _u64p), _p(w.view(np.float64), _f64p), _p(indptr, _u64p),
                   _p(one_c, _u64p), _p(one_v, _f64p), 0, _p(nnz, _u64p))
    m = int(nnz[0])
    cols = np.zeros(max(m, 1), np.uint64)
    vals = np.zeros(max(m, 1), np.complex128)
    lib.oracle_csr(nqubits, count, _p(xm, _u64p), _p(zm, _u64p), _p(w.view(np.float64), _f64p), _p(indptr, _u64p),
                   _p(cols, _u64p), _p(vals.view(np.float64), _f64p), m, _p(nnz, _u64p))
    return indptr, cols[:m], vals[:m]
