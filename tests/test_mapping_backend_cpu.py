"""Host-side rows next to the MVP: the Jordan-Wigner integral mapping (against
a dense construction from ladder matrices) and the pure-array backend plan."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle
from tencirpauli_b200 import PauliOperator
from tencirpauli_b200.backend import BackendMVPPlan
from tencirpauli_b200.mapping import chemistry_integrals, jordan_wigner_integrals


def _dense_from_op(op: PauliOperator) -> np.ndarray:
    n = op.nqubits
    xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
    dim = 1 << n
    H = np.zeros((dim, dim), dtype=np.complex128)
    for col in range(dim):
        e = np.zeros(dim, dtype=np.complex128)
        e[col] = 1.0
        H[:, col] = oracle.apply_term_direct(n, xm, zm, wp, e)
    return H


def _ladder_dense(n: int, p: int) -> np.ndarray:
    """a_p with qubit 0 as the most significant Kronecker factor and Z on modes < p."""
    Z = np.diag([1.0, -1.0]).astype(np.complex128)
    lower = np.array([[0, 1], [0, 0]], dtype=np.complex128)  # (X + iY)/2
    out = np.array([[1.0 + 0j]])
    for q in range(n):
        f = Z if q < p else (lower if q == p else np.eye(2, dtype=np.complex128))
        out = np.kron(out, f)
    return out


@pytest.mark.parametrize("n,seed", [(3, 1), (4, 2)])
def test_jordan_wigner_matches_dense_ladder_construction(n: int, seed: int) -> None:
    h, g = chemistry_integrals(n, seed=seed)
    codes, coeffs = jordan_wigner_integrals(h, g)
    op = PauliOperator.from_code_arrays(codes, coeffs)
    a = [_ladder_dense(n, p) for p in range(n)]
    ad = [m.conj().T for m in a]
    dim = 1 << n
    H = np.zeros((dim, dim), dtype=np.complex128)
    for p in range(n):
        for q in range(n):
            H += h[p, q] * ad[p] @ a[q]
    for p in range(n):
        for q in range(n):
            for r in range(n):
                for s in range(n):
                    H += 0.5 * g[p, q, r, s] * ad[p] @ ad[q] @ a[s] @ a[r]
    np.testing.assert_allclose(_dense_from_op(op), H, rtol=1e-12, atol=1e-13)
    assert np.allclose(H, H.conj().T)  # Hermitian with the 8-fold symmetric integrals


def test_integral_known_answer_of_the_reference() -> None:
    """The reference's integral convention (tests/test_integral_ingestion.py:11-38
    of the reference): the mapped operator equals the listed fermionic terms --
    1/2 on the two-body sum, a+_p a+_q a_s a_r index order, constant kept."""
    k = load_golden("integral_known_answer")
    h, g, constant = k["one_body"], k["two_body"], complex(k["constant"])
    codes, coeffs = jordan_wigner_integrals(h, g, constant=constant)
    op = PauliOperator.from_code_arrays(codes, coeffs)
    n = h.shape[0]
    a = [_ladder_dense(n, p) for p in range(n)]
    expected = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    for ops, c in zip(k["term_ops"], k["term_coefficients"]):
        m = np.eye(1 << n, dtype=np.complex128)
        for mode, action in ops:
            if mode < 0:
                break
            m = m @ (a[mode].conj().T if action == 1 else a[mode])
        expected += c * m
    np.testing.assert_allclose(_dense_from_op(op), expected, rtol=0, atol=1e-15)
    # without the constant the operator moves by exactly -constant * I
    codes0, coeffs0 = jordan_wigner_integrals(h, g)
    dense0 = _dense_from_op(PauliOperator.from_code_arrays(codes0, coeffs0))
    np.testing.assert_allclose(dense0 + constant * np.eye(1 << n), expected, rtol=0, atol=1e-15)


def test_integral_symmetries() -> None:
    h, g = chemistry_integrals(5, seed=3)
    np.testing.assert_array_equal(h, h.T)
    # g_pqrs = (pr|qs) with the 8-fold symmetry of real orbitals
    np.testing.assert_array_equal(g, g.transpose(1, 0, 3, 2))
    np.testing.assert_array_equal(g, g.transpose(2, 3, 0, 1))
    mags = np.abs(g[g != 0])
    assert mags.max() <= 1.0


def test_backend_plan_arrays_are_versioned_and_read_only() -> None:
    op = PauliOperator.from_terms(3, [("XZI", 1.0), ("IYY", -0.5j)])
    plan = op.compile("backend_mvp")
    assert isinstance(plan, BackendMVPPlan)
    assert plan.schema_version == 1 and plan.ordering == "qubit0_msb_matrix"
    assert plan.x_words.dtype == np.uint64 and plan.coefficients.dtype == np.complex128
    assert plan.estimated_bytes == 2 * (16 + 16)
    with pytest.raises(ValueError, match="read-only"):
        plan.x_words[0, 0] = 0
    with pytest.raises(TypeError, match="plan factory"):
        BackendMVPPlan(1, 3, 1, plan.x_words, plan.z_words, plan.coefficients)
