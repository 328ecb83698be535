"""GPU parity tests: the CUDA path (through the C ABI) against the oracle.

Tolerances: FP64 results must match the reference MVP to 1e-12 -- the
reference's own ``rtol = atol = 1e-12`` for the small fixtures
(``tests/test_hamiltonian.py:51-68,126-147`` of the reference), and at larger
sizes ``allclose(rtol=1e-12, atol=1e-12 * max|y_ref|)`` plus a norm-relative
error <= 1e-12.  complex64 (FP32 + Kahan) results are compared with the FP64
oracle at a norm-relative 2e-6.
"""

from __future__ import annotations

import threading

import numpy as np
import pytest

from conftest import golden_mvp_names, load_golden
from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, workloads  # noqa: E402
from tencirpauli_b200._native import NativeDeviceError  # noqa: E402

FP64_RTOL = 1e-12
C64_NORM_RTOL = 2e-6


def _oracle_terms(op: PauliOperator):
    return oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)


def _assert_fp64_close(y: np.ndarray, ref: np.ndarray) -> None:
    scale = float(np.max(np.abs(ref))) if ref.size else 0.0
    np.testing.assert_allclose(y, ref, rtol=FP64_RTOL, atol=FP64_RTOL * max(scale, 1e-300))
    denom = float(np.linalg.norm(ref))
    if denom > 0:
        assert float(np.linalg.norm(y - ref)) / denom <= FP64_RTOL


@pytest.mark.parametrize("name", golden_mvp_names())
@pytest.mark.parametrize("storage", ["lazy", "eager"])
def test_golden_vectors(name: str, storage: str) -> None:
    g = load_golden(name)
    n = int(g["nqubits"])
    op = PauliOperator.from_code_arrays(g["codes"].reshape(len(g["coefficients"]), n), g["coefficients"])
    plan = op.native_mvp_plan(storage=storage)
    y = plan.apply(g["state"])
    np.testing.assert_allclose(y, g["expected"], rtol=1e-12, atol=1e-12)
    out = np.full_like(y, 9.0 + 4.0j)
    plan.apply_into(np.ascontiguousarray(g["state"], dtype=np.complex128), out)
    np.testing.assert_array_equal(out, y)
    np.testing.assert_allclose(op.mvp(g["state"]), g["expected"], rtol=1e-12, atol=1e-12)
    if storage == "eager":
        xm, zm, wp = _oracle_terms(op)
        assert plan.transition_count == oracle.transition_count(n, xm, zm, wp)
        assert plan.retained_format == "compact_graph"
    else:
        assert plan.transition_count is None
        assert plan.retained_format == "compiled_actions"


def test_abi_fixed_vector_exact() -> None:
    # tests/test_native_abi.py:84-120 of the reference: H = 2Z + I, [1, 2] -> [3, -2]
    plan = PauliOperator.from_terms(1, [("Z", 2.0), ("I", 1.0)]).compile("native_mvp")
    out = plan._native_plan.apply(np.asarray([1.0 + 0j, 2.0 + 0j]), 2**63 - 1)
    np.testing.assert_array_equal(out, [3.0, -2.0])
    assert out.dtype == np.complex128 and out.flags.c_contiguous and out.flags.writeable


@pytest.mark.parametrize("n,words,seed", [(8, 50, 1), (12, 120, 2), (13, 200, 3), (14, 300, 4), (16, 400, 5), (17, 64, 6)])
def test_random_k_local_tiled_and_rowwise_paths(n: int, words: int, seed: int) -> None:
    codes, coeffs = workloads.random_k_local(n=n, words=words, seed=seed)
    coeffs = coeffs * (1.0 + 0.3j) if seed % 2 else coeffs  # exercise complex weights too
    op = PauliOperator.from_code_arrays(codes, coeffs)
    state = workloads.random_state(n, seed=seed)
    xm, zm, wp = _oracle_terms(op)
    ref = oracle.apply_term_direct(n, xm, zm, wp, state)
    plan = op.native_mvp_plan()
    _assert_fp64_close(plan.apply(state), ref)
    y64 = plan._native_plan.apply_c64(state.astype(np.complex64)).astype(np.complex128)
    assert np.linalg.norm(y64 - ref) / np.linalg.norm(ref) <= C64_NORM_RTOL


def test_heisenberg_chain_n20_matches_oracle() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(20))
    state = workloads.random_state(20)
    xm, zm, wp = _oracle_terms(op)
    ref = oracle.apply_term_direct(20, xm, zm, wp, state)
    plan = op.native_mvp_plan()
    _assert_fp64_close(plan.apply(state), ref)
    eager = op.native_mvp_plan(storage="eager")
    _assert_fp64_close(eager.apply(state), ref)
    assert eager.transition_count == oracle.transition_count(20, xm, zm, wp)


def test_overwrite_and_concurrent_apply_into() -> None:
    # tests/test_native_mvp_resources.py:180-207,276-311 of the reference
    op = PauliOperator.from_code_arrays(*workloads.random_k_local(n=14, words=100, seed=9))
    plan = op.native_mvp_plan()
    state = workloads.random_state(14, seed=3)
    original = state.copy()
    expected = plan.apply(state)
    outs = [np.full(plan.dimension, 9.0 + 3.0j), np.full(plan.dimension, -4.0 + 2.0j)]
    errors = []

    def work(out: np.ndarray) -> None:
        try:
            for _ in range(5):
                plan.apply_into(state, out, max_bytes=0)
        except Exception as exc:  # pragma: no cover - reported below
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(o,)) for o in outs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors
    np.testing.assert_array_equal(state, original)
    for o in outs:
        np.testing.assert_array_equal(o, expected)
    with pytest.raises(ValueError, match="overlap"):
        plan.apply_into(state, state)
    with pytest.raises(TypeError, match="complex128"):
        plan.apply_into(state.astype(np.complex64), np.empty_like(state))


def test_length_errors_and_empty_operator() -> None:
    with pytest.raises(ValueError, match="expected structure length"):
        PauliOperator.empty(2).mvp(np.ones(3, dtype=np.complex128))
    op = PauliOperator.empty(20)
    state = np.zeros(1 << 20, dtype=np.complex128)
    np.testing.assert_array_equal(op.mvp(state, max_bytes=1), state)
    plan = op.native_mvp_plan(max_bytes=1)
    np.testing.assert_array_equal(plan.apply(np.ones(1 << 20, np.complex128), max_bytes=1), state)


def test_device_apply_multi_rhs_matches_host() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_2d_open(16, seed=7))
    plan = op.native_mvp_plan()
    xs = torch.stack([workloads.random_state_device(16, seed=s) for s in range(3)])
    ys = torch.empty_like(xs)
    plan.apply_device(xs, ys)
    torch.cuda.synchronize()
    for v in range(3):
        ref = plan.apply(xs[v].cpu().numpy())
        np.testing.assert_array_equal(ys[v].cpu().numpy(), ref)
    xs64 = xs.to(torch.complex64)
    ys64 = torch.empty_like(xs64)
    plan.apply_device(xs64, ys64)
    torch.cuda.synchronize()
    rel = torch.linalg.vector_norm(ys64.to(torch.complex128) - ys) / torch.linalg.vector_norm(ys)
    assert float(rel) <= C64_NORM_RTOL
    plan._native_plan.device_status()


def test_diagonal_matches_oracle() -> None:
    op = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(3, 4))
    plan = op.native_mvp_plan()
    n = op.nqubits
    diag = torch.empty(1 << n, dtype=torch.complex128, device="cuda")
    plan.diagonal_device(diag)
    xm, zm, wp = _oracle_terms(op)
    keep = xm == 0
    ones = np.ones(1 << n, dtype=np.complex128)
    ref = oracle.apply_term_direct(n, xm[keep], zm[keep], wp[keep], ones)
    np.testing.assert_array_equal(diag.cpu().numpy(), ref)


def test_random_k_local_n28_full_size_sampled_rows_and_hermiticity() -> None:
    """The n = 28, 2000-word workload at full size: exact rows against the
    oracle on a random row sample, plus size-independent properties."""
    codes, coeffs = workloads.random_k_local(n=28, words=2000)
    op = PauliOperator.from_code_arrays(codes, coeffs)
    plan = op.native_mvp_plan()
    x = workloads.random_state_device(28, seed=11)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    torch.cuda.synchronize()
    plan._native_plan.device_status()
    rng = np.random.default_rng(0)
    rows = np.sort(rng.choice(1 << 28, size=4096, replace=False)).astype(np.uint64)
    xh = x.cpu().numpy()
    xm, zm, wp = _oracle_terms(op)
    ref_rows = oracle.apply_rows(28, xm, zm, wp, xh, rows)
    got = y[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy()
    _assert_fp64_close(got, ref_rows)
    # Hermiticity: <a, H b> == <H a, b> (real coefficients -> H Hermitian)
    a = workloads.random_state_device(28, seed=12)
    ha = torch.empty_like(a)
    plan.apply_device(a, ha)
    lhs = torch.vdot(a, y)
    rhs = torch.vdot(ha, x)
    torch.cuda.synchronize()
    assert abs(complex(lhs) - complex(rhs)) <= 1e-12 * max(1.0, abs(complex(lhs)))
    del x, y, a, ha
    torch.cuda.empty_cache()


def test_wrong_device_or_bad_tensor_rejected() -> None:
    plan = PauliOperator.from_terms(2, [("XX", 1.0)]).native_mvp_plan()
    x = torch.zeros(4, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError):
        plan.apply_device(x, torch.zeros(8, dtype=torch.complex128, device="cuda"))
    with pytest.raises(TypeError):
        plan.apply_device(x, torch.zeros(4, dtype=torch.complex64, device="cuda"))
    assert isinstance(NativeDeviceError("x", 33), RuntimeError)


def test_host_apply_of_a_large_state_streams_output_chunks_and_matches_device_path() -> None:
    """n = 25: the host entry point copies the state in quarters and runs one
    pass of the tiled kernel per quarter (the steps whose source tiles lie in
    it, adding to y after the first), then splits the last pass into chunks
    of output tiles whose copies overlap the next chunk.  Only the grouping
    of the FP64 sums differs from the single-pass device apply; pageable and
    pinned host buffers give the same bits."""
    codes, coeffs = workloads.random_k_local(n=25, words=64, seed=21)
    # X or Y letters on the two top row bits (qubits 0 and 1) put steps into
    # more than one pass
    assert np.isin(codes[:, 0], (1, 2)).any() and np.isin(codes[:, 1], (1, 2)).any()
    op = PauliOperator.from_code_arrays(codes, coeffs)
    plan = op.native_mvp_plan()
    x = workloads.random_state_device(25, seed=4)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    torch.cuda.synchronize()
    host_x = x.cpu().numpy()
    out = np.full(1 << 25, np.nan, dtype=np.complex128)
    plan.apply_into(host_x, out)
    dev = y.cpu().numpy()
    assert np.linalg.norm(out - dev) <= 1e-14 * np.linalg.norm(dev)
    rows = np.random.default_rng(5).choice(1 << 25, 256, replace=False).astype(np.uint64)
    xm, zm, wp = oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)
    expect = oracle.apply_rows(25, xm, zm, wp, host_x, rows)
    np.testing.assert_allclose(out[rows.astype(np.int64)], expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())
    pinned_x = torch.from_numpy(host_x).pin_memory()
    pinned_y = torch.empty_like(pinned_x).pin_memory()
    plan._native_plan.apply_into(pinned_x.numpy(), pinned_y.numpy(), 2**63 - 1)
    np.testing.assert_array_equal(pinned_y.numpy(), out)
    # complex64 host buffers take the same passes with Kahan-compensated sums
    out64 = np.empty(1 << 25, dtype=np.complex64)
    plan._native_plan.apply_c64_into(host_x.astype(np.complex64), out64)
    assert np.linalg.norm(out64 - dev) <= 2e-6 * np.linalg.norm(dev)
    del x, y
    torch.cuda.empty_cache()
