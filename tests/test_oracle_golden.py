"""Pin the CPU oracle (test infrastructure) to the reference's golden vectors.

The fixtures in ``tests/golden`` hold outputs of the reference's independent
dense Kronecker oracle (``tests/reference.py`` in the reference project) and
the fixed vectors written in its tests; see ``tests/golden/make_golden.py``.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_mvp_names, load_golden
from oracle import oracle


@pytest.mark.parametrize("name", golden_mvp_names())
def test_term_direct_matches_golden(name: str) -> None:
    g = load_golden(name)
    n = int(g["nqubits"])
    y = oracle.mvp(n, g["codes"], g["coefficients"], g["state"])
    # tests/test_hamiltonian.py:51-68,126-147 use rtol = atol = 1e-12
    np.testing.assert_allclose(y, g["expected"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("name", golden_mvp_names())
def test_xmask_diagonal_matches_golden_and_term_direct(name: str) -> None:
    g = load_golden(name)
    n = int(g["nqubits"])
    xw, zw, c = oracle.canonicalize(n, g["codes"], g["coefficients"])
    xm, zm, wp = oracle.matrix_terms(n, xw, zw, c)
    y_eager, transitions = oracle.apply_xmask_diagonal(n, xm, zm, wp, g["state"])
    np.testing.assert_allclose(y_eager, g["expected"], rtol=1e-12, atol=1e-12)
    assert transitions == oracle.transition_count(n, xm, zm, wp)
    assert transitions <= oracle.group_count(xm) * (1 << n)


def test_abi_fixed_vector_is_exact() -> None:
    g = load_golden("abi_fixed")
    y = oracle.mvp(1, g["codes"], g["coefficients"], g["state"])
    np.testing.assert_array_equal(y, np.asarray([3.0, -2.0], dtype=np.complex128))


def test_canonicalization_known_answers() -> None:
    k = load_golden("canonical_known_answers")
    for prefix in ("a", "b"):
        codes = k[f"{prefix}_codes"]
        n = codes.shape[1]
        xw, zw, c = oracle.canonicalize(n, codes, k[f"{prefix}_coefficients"])
        ex, ez = oracle.encode_codes(n, k[f"{prefix}_expected_codes"])
        np.testing.assert_array_equal(xw, ex)
        np.testing.assert_array_equal(zw, ez)
        np.testing.assert_array_equal(c, k[f"{prefix}_expected_coefficients"])


def test_rows_sampler_matches_full_apply() -> None:
    g = load_golden("rust_fixture_10_64")
    n = int(g["nqubits"])
    xw, zw, c = oracle.canonicalize(n, g["codes"], g["coefficients"])
    xm, zm, wp = oracle.matrix_terms(n, xw, zw, c)
    full = oracle.apply_term_direct(n, xm, zm, wp, g["state"])
    rows = np.asarray([0, 1, 17, 512, 1023], dtype=np.uint64)
    np.testing.assert_array_equal(oracle.apply_rows(n, xm, zm, wp, g["state"], rows), full[rows])


def test_planted_sign_error_is_detected() -> None:
    """A mistake planted in the oracle's inputs (Y phase dropped) must fail parity."""
    g = load_golden("random_differential_4")
    n = int(g["nqubits"])
    xw, zw, c = oracle.canonicalize(n, g["codes"], g["coefficients"])
    xm, zm, wp = oracle.matrix_terms(n, xw, zw, c)
    wrong = c.copy()  # coefficient without the i^{#Y} phase
    y = oracle.apply_term_direct(n, xm, zm, wrong, g["state"])
    assert not np.allclose(y, g["expected"], rtol=1e-12, atol=1e-12)


def test_empty_operator_and_zero_qubits() -> None:
    y = oracle.mvp(3, np.zeros((0, 3), np.uint8), np.zeros(0, np.complex128), np.ones(8, np.complex128))
    np.testing.assert_array_equal(y, np.zeros(8, np.complex128))
    y0 = oracle.mvp(0, np.zeros((1, 0), np.uint8), np.asarray([2.5 - 1j]), np.asarray([2.0 + 0j]))
    np.testing.assert_array_equal(y0, np.asarray([5.0 - 2.0j]))


def test_invalid_inputs_report_status() -> None:
    with pytest.raises(oracle.OracleError) as err:
        oracle.canonicalize(2, np.asarray([[1, 4]], np.uint8), np.asarray([1.0 + 0j]))
    assert err.value.status == 1
    with pytest.raises(oracle.OracleError) as err:
        oracle.canonicalize(1, np.asarray([[1]], np.uint8), np.asarray([np.nan + 0j]))
    assert err.value.status == 5
