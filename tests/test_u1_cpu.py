"""CPU checks of the U(1) sector row: the oracle (``oracle/u1_oracle.c``)
against the reference's own known answers and against an independent dense
projection, and the host-side entry points of ``include/tcp_sector.h``
(rank, unrank, basis, number-commutator rule) against the oracle.  No kernel
is launched here.

Known answers come from the reference's tests: the explicit sector orders of
``tests/test_symmetry.py:159-182`` and the wide-sector orders built from
``itertools.combinations`` in ``tests/test_u1.py:13-27,84-122``.
"""

from __future__ import annotations

import math
from itertools import combinations

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)
from oracle import oracle
from tencirpauli_b200 import PauliOperator, U1Sector, _native


def _basis_values(n: int, k: int) -> list:
    return sorted(sum(1 << (n - 1 - q) for q in occ) for occ in combinations(range(n), k))


def _packed(value: int, n: int) -> np.ndarray:
    words = [0] * ((n + 63) // 64)
    for q in range(n):
        if (value >> (n - 1 - q)) & 1:
            words[q // 64] |= 1 << (q % 64)
    return np.asarray(words, dtype=np.uint64)


def _local(n: int, code: str, *qubits: int) -> str:
    s = ["I"] * n
    for q in qubits:
        s[q] = code
    return "".join(s)


def _hopping(n: int, coefficient: complex = 0.5) -> list:
    terms = []
    for q in range(n - 1):
        terms += [(_local(n, "X", q, q + 1), coefficient), (_local(n, "Y", q, q + 1), coefficient)]
    return terms


# ------------------------------ oracle pins ----------------------------------
@pytest.mark.parametrize(
    "n,k,expected",
    [(0, 0, [0]), (3, 0, [0]), (3, 1, [1, 2, 4]), (3, 2, [3, 5, 6]), (3, 3, [7])],
)
def test_oracle_basis_order_matches_reference_known_answers(n: int, k: int, expected: list) -> None:
    assert oracle.u1_dimension(n, k) == len(expected)
    for index, value in enumerate(expected):
        words = oracle.u1_unrank(n, k, index)
        np.testing.assert_array_equal(words, _packed(value, n))
        assert oracle.u1_rank(n, k, _packed(value, n)) == index


@pytest.mark.parametrize("n,k", [(63, 1), (64, 2), (65, 1), (65, 63), (127, 2), (128, 1), (129, 2), (256, 2)])
def test_oracle_wide_sector_order(n: int, k: int) -> None:
    expected = _basis_values(n, k)
    assert oracle.u1_dimension(n, k) == len(expected)
    rng = np.random.default_rng(n * 1000 + k)
    picks = {0, len(expected) - 1, *map(int, rng.integers(0, len(expected), size=40))}
    for index in sorted(picks):
        np.testing.assert_array_equal(oracle.u1_unrank(n, k, index), _packed(expected[index], n))
        assert oracle.u1_rank(n, k, _packed(expected[index], n)) == index


def _dense_full(op: PauliOperator) -> np.ndarray:
    n = op.nqubits
    xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
    dim = 1 << n
    out = np.zeros((dim, dim), np.complex128)
    eye = np.eye(dim, dtype=np.complex128)
    for c in range(dim):
        out[:, c] = oracle.apply_term_direct(n, xm, zm, wp, eye[c])
    return out


def _random_conserving(n: int, rng: np.random.Generator) -> list:
    """Identity + XX/YY hopping (shared coefficients) + Z fields + ZZ, complex
    coefficients (the shape of tests/test_symmetry.py:237-278)."""
    terms = [("I" * n, complex(rng.normal(), rng.normal()))]
    for q in range(n - 1):
        h = complex(rng.normal(), rng.normal())
        terms += [(_local(n, "X", q, q + 1), h), (_local(n, "Y", q, q + 1), h)]
    for q in range(n):
        terms.append((_local(n, "Z", q), complex(rng.normal(), rng.normal())))
    if n > 2:
        terms.append((_local(n, "Z", 0, n - 1), complex(rng.normal(), 0.0)))
        # a longer-range exchange whose Y factors sit between the XY pair
        terms += [("X" + "Z" * (n - 2) + "X", 0.3), ("Y" + "Z" * (n - 2) + "Y", 0.3)]
    return terms


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6])
def test_oracle_apply_is_the_projection_of_the_full_operator(n: int) -> None:
    rng = np.random.default_rng(20260802 + n)
    op = PauliOperator.from_terms(n, _random_conserving(n, rng))
    full = _dense_full(op)
    for k in range(n + 1):
        basis = np.asarray(_basis_values(n, k))
        expected = full[np.ix_(basis, basis)]
        state = rng.normal(size=len(basis)) + 1j * rng.normal(size=len(basis))
        got = oracle.u1_apply(n, k, op.x_words, op.z_words, op.coefficients, state)
        np.testing.assert_allclose(got, expected @ state, rtol=1e-12, atol=1e-12)
        indptr, cols, vals = oracle.u1_csr(n, k, op.x_words, op.z_words, op.coefficients)
        dense = np.zeros_like(expected)
        for r in range(len(basis)):
            row_cols = cols[indptr[r] : indptr[r + 1]]
            assert np.all(np.diff(row_cols.astype(np.int64)) > 0)  # ascending sources
            dense[r, row_cols.astype(np.int64)] = vals[indptr[r] : indptr[r + 1]]
        np.testing.assert_allclose(dense, expected, rtol=1e-12, atol=1e-12)


def test_oracle_reference_projection_case_and_leakage() -> None:
    # tests/test_symmetry.py:185-206 and :229-234 of the reference
    op = PauliOperator.from_terms(3, [("XXI", 0.5), ("YYI", 0.5), ("IZZ", -0.25), ("ZII", 0.1)])
    full = _dense_full(op)
    basis = np.asarray([1, 2, 4])
    state = np.asarray([1.0, 2.0, 3.0], np.complex128)
    got = oracle.u1_apply(3, 1, op.x_words, op.z_words, op.coefficients, state)
    np.testing.assert_allclose(got, full[np.ix_(basis, basis)] @ state, rtol=1e-12, atol=1e-15)
    hop = PauliOperator.from_terms(3, [("XXI", 1.0), ("YYI", 1.0)])
    oracle.u1_apply(3, 1, hop.x_words, hop.z_words, hop.coefficients, state)  # aggregated: no leak
    leak = PauliOperator.from_terms(3, [("XII", 1.0)])
    with pytest.raises(oracle.OracleLeakage) as info:
        oracle.u1_apply(3, 1, leak.x_words, leak.z_words, leak.coefficients, state)
    assert info.value.source == 0 and info.value.weight == 2  # |001> -> |101>


def test_oracle_number_commutator_matches_dense_commutator() -> None:
    rng = np.random.default_rng(7)
    for n in (2, 3, 4):
        number = np.diag([bin(i).count("1") for i in range(1 << n)]).astype(np.complex128)
        for trial in range(12):
            if trial % 3 == 0:
                terms = _random_conserving(n, rng)
            else:
                letters = "IXYZ"
                terms = [("".join(letters[int(c)] for c in rng.integers(0, 4, size=n)), complex(rng.normal(), 0.0))
                         for _ in range(int(rng.integers(1, 6)))]
            op = PauliOperator.from_terms(n, terms)
            h = _dense_full(op)
            conserved = np.allclose(h @ number - number @ h, 0.0, atol=1e-12)
            nonzero = oracle.number_commutator(n, op.x_words, op.z_words, op.coefficients)
            assert (nonzero == 0) == conserved, (n, terms)


# ------------------------- host entry points vs oracle ----------------------------
@pytest.mark.parametrize("n,k", [(0, 0), (1, 1), (5, 2), (10, 7), (20, 10), (33, 3), (63, 1), (64, 2), (64, 0),
                                 (65, 63), (129, 2), (256, 2)])
def test_host_rank_unrank_match_oracle(n: int, k: int) -> None:
    dim = _native.u1_dimension(n, k)
    assert dim == math.comb(n, k) == oracle.u1_dimension(n, k)
    rng = np.random.default_rng(n + 17 * k)
    picks = {0, dim - 1, *map(int, rng.integers(0, dim, size=30))}
    for index in sorted(picks):
        words = _native.u1_unrank_words(n, k, index)
        np.testing.assert_array_equal(words, oracle.u1_unrank(n, k, index))
        if n:
            assert _native.u1_rank_words(n, k, words) == index
    sector = U1Sector(n, k)
    if dim <= 64 and n <= 64:
        values = _basis_values(n, k)
        assert [sector.rank(v) for v in values] == list(range(dim))
        assert [sector.unrank(i) for i in range(dim)] == [
            tuple((v >> (n - 1 - q)) & 1 for q in range(n)) for v in values
        ]


@pytest.mark.parametrize("n,k", [(3, 1), (3, 2), (8, 4), (63, 1), (64, 2), (65, 1), (127, 2), (128, 1), (129, 2), (256, 2)])
def test_basis_words_packed_matches_reference_layout(n: int, k: int) -> None:
    # tests/test_u1.py:84-122: TensorCircuit integers for n <= 64, packed words beyond
    sector = U1Sector(n, k)
    expected = _basis_values(n, k)
    basis = sector.basis_words_packed()
    assert basis.flags.writeable is False
    if n <= 64:
        assert basis.shape == (len(expected), 1)
        np.testing.assert_array_equal(basis[:, 0], np.asarray(expected, dtype=np.uint64))
    else:
        assert basis.shape == (len(expected), (n + 63) // 64)
        np.testing.assert_array_equal(basis[:32], np.asarray([_packed(v, n) for v in expected[:32]]))
        if n % 64:
            assert np.all(basis[:, -1] < (1 << (n % 64)))
    if n <= 8:
        states = sector.basis_states()
        np.testing.assert_array_equal(
            states, np.asarray([[(v >> (n - 1 - q)) & 1 for q in range(n)] for v in expected], np.uint8)
        )


def test_host_errors_mirror_the_reference() -> None:
    with pytest.raises(ValueError):
        U1Sector(2, 3)
    with pytest.raises((ValueError, IndexError)):
        U1Sector(2, 1).unrank(2)
    with pytest.raises(ValueError, match="invalid sector"):
        _native.u1_dimension(2, 3)
    with pytest.raises(ValueError, match="wrong Hamming weight"):
        _native.u1_rank_words(3, 1, np.asarray([3], np.uint64))
    with pytest.raises(ValueError, match="padding bits"):
        _native.u1_rank_words(3, 1, np.asarray([8], np.uint64))
    with pytest.raises(ValueError, match="out of range"):
        _native.u1_unrank_words(3, 1, 3)
    with pytest.raises(OverflowError):
        _native.u1_dimension(200, 100)
    with pytest.raises(ValueError, match="bitstring has the wrong Hamming weight"):
        U1Sector(3, 1).rank(3)


@pytest.mark.parametrize("seed", range(8))
def test_number_commutator_matches_oracle(seed: int) -> None:
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 80))
    count = int(rng.integers(0, 60))
    letters = "IXYZ"
    terms = []
    for _ in range(count):
        if rng.random() < 0.5 and n > 1:
            a, b = sorted(rng.choice(n, size=2, replace=False))
            h = complex(rng.normal(), rng.normal())
            terms += [(_local(n, "X", a, b), h), (_local(n, "Y", a, b), h)]
        else:
            terms.append(("".join(letters[int(c)] for c in rng.integers(0, 4, size=n)), complex(rng.normal(), 0.0)))
    op = PauliOperator.from_terms(n, terms) if terms else PauliOperator.empty(n)
    got = _native.number_commutator(n, op.x_words, op.z_words, op.coefficients)
    assert got == oracle.number_commutator(n, op.x_words, op.z_words, op.coefficients)


def test_lazy_restriction_rejects_a_non_conserving_operator_before_any_device_work() -> None:
    sector = U1Sector(3, 1)
    with pytest.raises(ValueError, match=r"U\(1\) sector leakage"):
        PauliOperator.from_terms(3, [("XII", 1.0)]).restrict_charge(sector)
    with pytest.raises(TypeError):
        PauliOperator.from_terms(3, [("ZII", 1.0)]).restrict_charge(object())
    with pytest.raises(ValueError, match="expected sector for 3 qubits"):
        PauliOperator.from_terms(3, [("ZII", 1.0)]).restrict_charge(U1Sector(4, 1))
