"""GPU tests of the dense / COO / CSR targets (``include/tcp_matrix.h``).

Pins: the reference's own dense matrices (``tests/golden``, made from
``tests/reference.py`` of the reference by ``tests/golden/make_golden.py``) at
the reference's tolerance rtol = atol = 1e-12
(``tests/test_hamiltonian.py:51-68``).  Against the oracle
(``oracle/mvp_oracle.c``: ``dense_matrix`` and ``sparse_entries`` restated),
which sums every value in the same order, the dense matrix and the CSR
arrays are compared exactly.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden_mvp_names, load_golden
from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, workloads  # noqa: E402


def _oracle_parts(op: PauliOperator):
    return oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)


def _check_against_oracle(op: PauliOperator) -> None:
    xm, zm, wp = _oracle_parts(op)
    n = op.nqubits
    dense = op.dense()
    np.testing.assert_array_equal(dense, oracle.dense(n, xm, zm, wp))
    indptr, cols, vals = oracle.csr(n, xm, zm, wp)
    csr = op.csr()
    np.testing.assert_array_equal(csr.indptr, indptr)
    np.testing.assert_array_equal(csr.indices, cols)
    assert csr.data.tobytes() == vals.tobytes()
    coo = op.coo()
    np.testing.assert_array_equal(coo.row, np.repeat(np.arange(1 << n, dtype=np.uint64), np.diff(indptr.astype(np.int64))))
    np.testing.assert_array_equal(coo.column, cols)
    assert coo.data.tobytes() == vals.tobytes()
    assert coo.shape == csr.shape == (1 << n, 1 << n)


@pytest.mark.parametrize("name", [n for n in golden_mvp_names() if "dense" in load_golden(n)])
def test_dense_coo_csr_match_the_reference_dense_oracle(name: str) -> None:
    g = load_golden(name)
    n = int(g["nqubits"])
    op = PauliOperator.from_code_arrays(g["codes"].reshape(len(g["coefficients"]), n), g["coefficients"])
    expected = g["dense"]
    np.testing.assert_allclose(op.dense(), expected, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(op.compile("coo").to_scipy().toarray(), expected, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(op.compile("csr").to_scipy().toarray(), expected, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(op.compile("dense"), expected, rtol=1e-12, atol=1e-12)
    _check_against_oracle(op)


@pytest.mark.parametrize("n,words,seed", [(6, 40, 1), (9, 150, 2), (11, 300, 3), (12, 64, 4)])
def test_random_operators_match_the_oracle_exactly(n: int, words: int, seed: int) -> None:
    codes, coeffs = workloads.random_k_local(n=n, words=words, seed=seed)
    op = PauliOperator.from_code_arrays(codes, coeffs * (1.0 + 0.5j) if seed % 2 else coeffs)
    _check_against_oracle(op)


def test_exact_cancellations_are_skipped_by_the_sparse_targets_only() -> None:
    # IZ + ZZ: the diagonal group sums to zero on half of the columns
    op = PauliOperator.from_terms(2, [("IZ", 1.0), ("ZZ", 1.0), ("XX", 0.5), ("YY", 0.5)])
    dense = op.dense()
    assert np.count_nonzero(dense == 0) > 0
    csr = op.csr()
    assert len(csr.data) == np.count_nonzero(dense)
    np.testing.assert_array_equal(csr.to_scipy().toarray(), dense)
    _check_against_oracle(op)


def test_heisenberg_chain_n14_csr_matches_oracle_and_mvp() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(14))
    _xm, _zm, _wp = _oracle_parts(op)
    indptr, cols, vals = oracle.csr(14, _xm, _zm, _wp)
    csr = op.csr()
    np.testing.assert_array_equal(csr.indptr, indptr)
    np.testing.assert_array_equal(csr.indices, cols)
    assert csr.data.tobytes() == vals.tobytes()
    state = workloads.random_state(14, seed=5)
    np.testing.assert_allclose(csr.to_scipy() @ state, op.mvp(state), rtol=1e-12, atol=1e-12)
    assert len(cols) == op.native_mvp_plan(storage="eager").transition_count


def test_budgets_raise_memory_error_before_any_allocation() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(16))
    with pytest.raises(MemoryError, match="exceeds memory limit"):
        op.dense(max_bytes=2 * 1024**3)  # 2^32 * 16 bytes needed
    big = PauliOperator.from_code_arrays(*workloads.random_k_local(n=22, words=400, seed=1))
    with pytest.raises(MemoryError, match="exceeds memory limit"):
        big.csr(max_bytes=1024**3 + 1)
    with pytest.raises(MemoryError, match="exceeds memory limit"):
        big.coo(max_bytes=1024**3 + 1)
    with pytest.raises(ValueError, match="target must be one of"):
        op.compile("sparse")
