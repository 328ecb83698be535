"""GPU tests of the batched MVP (many Hamiltonians x RHS blocks, one persistent
graph-launched kernel) against the oracle and the single-plan path."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, workloads  # noqa: E402
from tencirpauli_b200.batch import BatchedMVP  # noqa: E402

FP64_RTOL = 1e-12
C64_NORM_RTOL = 2e-6


def _members():
    ops = [PauliOperator.from_code_arrays(*workloads.heisenberg_2d_open(n, seed=100 + n)) for n in (10, 12, 13, 14, 16)]
    codes, coeffs = workloads.random_k_local(n=12, words=150, seed=8)
    ops.append(PauliOperator.from_code_arrays(codes, coeffs * (0.5 - 0.25j)))
    ops.append(PauliOperator.empty(10))
    return ops


def _blocks(ops, nrhs, dtype):
    xs = [workloads.random_state_device(op.nqubits, seed=7 + i, dtype=dtype, nrhs=nrhs) for i, op in enumerate(ops)]
    ys = [torch.full_like(x, float("nan")) for x in xs]
    return xs, ys


def _oracle_apply(op, x: np.ndarray) -> np.ndarray:
    xm, zm, wp = oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)
    return oracle.apply_term_direct(op.nqubits, xm, zm, wp, x)


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_batch_matches_oracle_for_every_member_and_rhs(dtype: str) -> None:
    ops = _members()
    plans = [op.native_mvp_plan() for op in ops]
    tdt = torch.complex128 if dtype == "complex128" else torch.complex64
    nrhs = 4
    xs, ys = _blocks(ops, nrhs, tdt)
    batch = BatchedMVP(plans, nrhs=nrhs, dtype=dtype)
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    batch.device_status()
    for op, x, y in zip(ops, xs, ys):
        for v in range(nrhs):
            ref = _oracle_apply(op, x[v].cpu().numpy().astype(np.complex128))
            got = y[v].cpu().numpy().astype(np.complex128)
            if not np.any(ref):
                np.testing.assert_array_equal(got, ref)
                continue
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= (FP64_RTOL if dtype == "complex128" else C64_NORM_RTOL), (op.nqubits, v, err)


def test_every_variant_gives_the_same_result_and_graph_replays() -> None:
    ops = _members()[:5]
    plans = [op.native_mvp_plan() for op in ops]
    nrhs = 4
    xs, ys = _blocks(ops, nrhs, torch.complex128)
    batch = BatchedMVP(plans, nrhs=nrhs, dtype="complex128")
    batch.configure(9, 4)
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    ref = [y.clone() for y in ys]
    for logt in (8, 9, 10):
        for rb in (1, 2, 4):
            batch.configure(logt, rb)
            for y in ys:
                y.fill_(float("nan"))
            batch.apply(xs, ys)
            batch.apply(xs, ys)  # graph replay
            torch.cuda.synchronize()
            for y, r in zip(ys, ref):
                rel = torch.linalg.vector_norm(y - r) / torch.linalg.vector_norm(r)
                assert float(rel) <= 1e-13, (logt, rb, float(rel))
    # new buffers: the descriptor table is refreshed, the graph is reused
    xs2, ys2 = _blocks(ops, nrhs, torch.complex128)
    batch.apply(xs2, ys2)
    torch.cuda.synchronize()
    for op, x, y in zip(ops, xs2, ys2):
        ref0 = _oracle_apply(op, x[0].cpu().numpy())
        assert np.linalg.norm(y[0].cpu().numpy() - ref0) / np.linalg.norm(ref0) <= FP64_RTOL
    batch.device_status()


@pytest.mark.parametrize("dtype", ["complex128", "complex64"])
def test_ring_configuration_matches_the_persistent_kernel(dtype: str) -> None:
    # (12, 1): one ring-kernel launch per member over all tiles and RHS
    ops = _members()[1:6] + [PauliOperator.empty(12)]
    plans = [op.native_mvp_plan() for op in ops]
    tdt = torch.complex128 if dtype == "complex128" else torch.complex64
    nrhs = 3
    xs, ys = _blocks(ops, nrhs, tdt)
    batch = BatchedMVP(plans, nrhs=nrhs, dtype=dtype)
    batch.configure(9, 1)
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    ref = [y.clone() for y in ys]
    batch.configure(12, 1)
    info = batch.info()
    assert info["tile_rows_log2"] == 12 and info["rhs_block"] == 1 and info["grid"] == len(ops) - 1
    for y in ys:
        y.fill_(float("nan"))
    batch.apply(xs, ys)
    batch.apply(xs, ys)  # graph replay
    torch.cuda.synchronize()
    batch.device_status()
    tol = 1e-13 if dtype == "complex128" else C64_NORM_RTOL
    for op, x, y, r in zip(ops, xs, ys, ref):
        if op.term_count == 0:
            assert not torch.any(y != 0)
            continue
        rel = torch.linalg.vector_norm(y - r) / torch.linalg.vector_norm(r)
        assert float(rel) <= tol, (op.nqubits, float(rel))
    # new buffers: the captured launches are rebuilt around them
    xs2, ys2 = _blocks(ops, nrhs, tdt)
    batch.apply(xs2, ys2)
    torch.cuda.synchronize()
    for op, x, y in zip(ops, xs2, ys2):
        if op.term_count == 0:
            continue
        for v in range(nrhs):
            want = _oracle_apply(op, x[v].cpu().numpy().astype(np.complex128))
            got = y[v].cpu().numpy().astype(np.complex128)
            err = np.linalg.norm(got - want) / np.linalg.norm(want)
            assert err <= (FP64_RTOL if dtype == "complex128" else C64_NORM_RTOL), (op.nqubits, v, err)
    # a member below 12 qubits has no ring schedule
    small = BatchedMVP([op.native_mvp_plan() for op in _members()[:2]], nrhs=1, dtype=dtype)
    with pytest.raises(ValueError, match="ring schedule"):
        small.configure(12, 1)


def test_autotune_picks_a_variant_and_caches_it(tmp_path) -> None:
    ops = _members()[1:5]
    plans = [op.native_mvp_plan() for op in ops]
    xs, ys = _blocks(ops, 8, torch.complex64)
    batch = BatchedMVP(plans, nrhs=8, dtype="complex64")
    cache = tmp_path / "autotune.txt"
    info = batch.autotune(xs, ys, cache_path=str(cache), repeats=2)
    assert info["tile_rows_log2"] in (8, 9, 10, 12) and 8 % info["rhs_block"] == 0
    text = cache.read_text().split()
    assert len(text) == 3 and int(text[1]) == info["tile_rows_log2"] and int(text[2]) == info["rhs_block"]
    again = BatchedMVP(plans, nrhs=8, dtype="complex64").autotune(xs, ys, cache_path=str(cache))
    assert again == info
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    for op, x, y in zip(ops, xs, ys):
        ref = _oracle_apply(op, x[3].cpu().numpy().astype(np.complex128))
        assert np.linalg.norm(y[3].cpu().numpy() - ref) / np.linalg.norm(ref) <= C64_NORM_RTOL


def test_batch_argument_errors() -> None:
    plans = [PauliOperator.from_code_arrays(*workloads.heisenberg_2d_open(10, seed=1)).native_mvp_plan()]
    with pytest.raises(ValueError):
        BatchedMVP(plans, nrhs=0)
    small = [PauliOperator.from_terms(4, [("XXII", 1.0)]).native_mvp_plan()]
    with pytest.raises(ValueError, match="at least 8 qubits"):
        BatchedMVP(small, nrhs=1)
    batch = BatchedMVP(plans, nrhs=2)
    with pytest.raises(ValueError, match="RHS block"):
        batch.configure(9, 4)
    x = torch.zeros(2, 1 << 10, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError):
        batch.apply([x], [x.clone()])  # complex128 buffers for a complex64 batch
