"""Host-side API behaviour that needs no GPU: operator construction, the
max_bytes policy and the strict apply_into buffer protocol."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle
from tencirpauli_b200 import DEFAULT_MAX_BYTES, NativeMVPPlan, PauliOperator
from tencirpauli_b200 import _native_mvp as facade
from tencirpauli_b200 import workloads


def test_from_terms_canonical_order_and_exact_cancellation() -> None:
    # tests/test_pauli_operator.py:23-30 of the reference
    op = PauliOperator.from_terms(2, (("ZX", 1.0), ("II", 2.0), ("ZX", -0.25j), ("II", -2.0)))
    assert tuple(t.word.to_string() for t in op.terms) == ("ZX",)
    assert op.terms[0].coefficient == 1.0 - 0.25j
    assert PauliOperator.empty(2).terms == ()


def test_code_array_constructor_and_validation() -> None:
    op = PauliOperator.from_code_arrays(np.array([[3, 1], [0, 0], [3, 1]]), [1.0, 2.0, -0.25j])
    assert tuple((t.word.to_string(), t.coefficient) for t in op.terms) == (("II", 2.0), ("ZX", 1.0 - 0.25j))
    with pytest.raises(ValueError, match=r"half-open range 0\.\.4"):
        PauliOperator.from_code_arrays([[4]], [1.0])
    with pytest.raises(ValueError, match="one value per structure"):
        PauliOperator.from_code_arrays([[1], [2]], [1.0])
    with pytest.raises(ValueError, match="expected structure length"):
        PauliOperator.from_terms(3, (("XX", 1.0),))
    with pytest.raises(ValueError):
        PauliOperator.from_terms(1, (("Q", 1.0),))
    with pytest.raises(ValueError, match="not finite"):
        PauliOperator.from_terms(1, (("X", float("nan")),))


def test_operator_terms_match_oracle_canonicalization() -> None:
    codes, coeffs = workloads.random_k_local(n=12, words=300, seed=5)
    op = PauliOperator.from_code_arrays(codes, coeffs)
    ox, oz, oc = oracle.canonicalize(12, codes, coeffs)
    np.testing.assert_array_equal(op.x_words, ox)
    np.testing.assert_array_equal(op.z_words, oz)
    np.testing.assert_array_equal(op.coefficients, oc)
    assert not op.x_words.flags.writeable


def test_workload_sizes() -> None:
    chain = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(20))
    assert chain.term_count == 80
    xm, _, _ = oracle.matrix_terms(20, chain.x_words, chain.z_words, chain.coefficients)
    assert oracle.group_count(xm) == 21
    j1j2 = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(4, 6))
    assert j1j2.term_count == 288
    xm, _, _ = oracle.matrix_terms(24, j1j2.x_words, j1j2.z_words, j1j2.coefficients)
    assert oracle.group_count(xm) == 97
    a = workloads.random_k_local(n=28, words=2000)
    b = workloads.random_k_local(n=28, words=2000)
    np.testing.assert_array_equal(a[0], b[0])
    assert workloads.lattice_shape(24) == (4, 6)
    assert workloads.lattice_shape(17) == (1, 17)


def test_max_bytes_policy() -> None:
    assert DEFAULT_MAX_BYTES == 16 * 1024**3
    facade.check_allocation(facade.MIN_ENFORCED_MAX_BYTES, 0, "advisory allocation")
    with pytest.raises(MemoryError, match="exceeding max_bytes"):
        facade.check_allocation(facade.MIN_ENFORCED_MAX_BYTES + 1, facade.MIN_ENFORCED_MAX_BYTES, "major")
    with pytest.raises(ValueError, match="max_bytes"):
        facade.validate_max_bytes(-1)
    with pytest.raises(ValueError, match="max_bytes"):
        facade.validate_max_bytes(True)  # type: ignore[arg-type]


def test_apply_into_buffer_protocol() -> None:
    dim = 8
    state = np.arange(dim, dtype=np.complex128)
    readonly = np.empty_like(state)
    readonly.flags.writeable = False
    with pytest.raises(ValueError, match="writable"):
        facade.validate_apply_into_buffers(state, readonly, dim)
    with pytest.raises(ValueError, match="C-contiguous"):
        facade.validate_apply_into_buffers(state, np.empty(2 * dim, np.complex128)[::2], dim)
    overlapping = np.empty(dim + 1, dtype=np.complex128)
    with pytest.raises(ValueError, match="overlap"):
        facade.validate_apply_into_buffers(overlapping[:-1], overlapping[1:], dim)
    with pytest.raises(ValueError, match="shape"):
        facade.validate_apply_into_buffers(state, np.empty(dim + 1, np.complex128), dim)
    with pytest.raises(TypeError, match="complex128"):
        facade.validate_apply_into_buffers(state.astype(np.complex64), np.empty_like(state), dim)
    with pytest.raises(TypeError, match="NumPy arrays"):
        facade.validate_apply_into_buffers(list(state), np.empty_like(state), dim)


def test_eager_plan_over_budget_raises_memory_error_without_device() -> None:
    op = PauliOperator.from_terms(30, (("X" + "I" * 29, 1.0),))
    with pytest.raises(MemoryError, match="exceeds memory limit"):
        op.native_mvp_plan(storage="eager", max_bytes=2 * 1024**3)


def test_plan_factory_token_is_required() -> None:
    with pytest.raises(TypeError, match="plan factory"):
        NativeMVPPlan(1, None, "lazy", 0)


def test_storage_label_is_validated() -> None:
    with pytest.raises(ValueError, match="storage"):
        PauliOperator.from_terms(1, (("X", 1.0),)).native_mvp_plan(storage="dense")  # type: ignore[arg-type]
