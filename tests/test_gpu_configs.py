"""Parity at the benchmark configurations, at full size, through the C ABI.

* random 2000-word 2..4-local Hamiltonian, n = 28 (the bench workload):
  complex128 and complex64 on 2^18 random rows against the oracle's row loop,
  plus the host entry point against the device entry point;
* the same generator at n = 24: the full vector against the full oracle, for
  both dtypes and through both the host and the device entries;
* the batched set: 64 open 2D Heisenberg lattices (n uniform in 16..26),
  8 complex64 right-hand sides each, one autotuned graph-launched batch, every
  member x RHS checked on 1024 rows;
* the Jordan-Wigner chemistry-like operator: n = 28 (347,513 terms) on a row
  sample, and the full vector at n = 20 for both dtypes.

Tolerances follow the reference's own MVP tests
(``tests/test_hamiltonian.py:51-68,126-147``: rtol = atol = 1e-12): FP64 rows
satisfy ``allclose(rtol=1e-12, atol=1e-12 * max|y_ref|)`` and a norm-relative
error <= 1e-12; complex64 (FP32 products, Kahan-compensated sums) is held to a
norm-relative 2e-6 of the FP64 oracle, and the measured error is printed.
"""

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
from tencirpauli_b200.mapping import chemistry_integrals, jordan_wigner_integrals  # noqa: E402

FP64_RTOL = 1e-12
C64_NORM_RTOL = 2e-6


def _terms(op: PauliOperator):
    return oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)


def _fp64_close(got: np.ndarray, ref: np.ndarray) -> float:
    scale = float(np.abs(ref).max())
    np.testing.assert_allclose(got, ref, rtol=FP64_RTOL, atol=FP64_RTOL * scale)
    rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    assert rel <= FP64_RTOL
    return rel


def _c64_close(got: np.ndarray, ref: np.ndarray, label: str) -> float:
    rel = float(np.linalg.norm(got.astype(np.complex128) - ref) / np.linalg.norm(ref))
    print(f"{label}: complex64 norm-relative error vs FP64 oracle {rel:.3e}")
    assert rel <= C64_NORM_RTOL
    return rel


def _rows(dim: int, count: int, seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(dim, size=count, replace=False)).astype(np.uint64)


def _take(y, rows: np.ndarray) -> np.ndarray:
    return y[torch.from_numpy(rows.astype(np.int64)).to(y.device)].cpu().numpy()


def test_random_2000_words_n28_sampled_rows_both_dtypes_and_host_entry() -> None:
    n = 28
    op = PauliOperator.from_code_arrays(*workloads.random_k_local(n=n, words=2000))
    plan = op.native_mvp_plan()
    xm, zm, wp = _terms(op)
    rows = _rows(1 << n, 1 << 18, seed=28)

    x = workloads.random_state_device(n, seed=31)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    torch.cuda.synchronize()
    plan._native_plan.device_status()
    xh = x.cpu().numpy()
    ref = oracle.apply_rows(n, xm, zm, wp, xh, rows)
    _fp64_close(_take(y, rows), ref)

    # the host entry point (state in four parts, passes of the tiled kernel,
    # chunked copies) against the single-pass device result
    out = np.empty_like(xh)
    plan.apply_into(xh, out)
    yd = y.cpu().numpy()
    assert np.linalg.norm(out - yd) <= 1e-14 * np.linalg.norm(yd)
    _fp64_close(out[rows.astype(np.int64)], ref)
    del y, out, yd
    torch.cuda.empty_cache()

    # complex64 storage of the same state
    x64 = x.to(torch.complex64)
    del x
    y64 = torch.empty_like(x64)
    plan.apply_device(x64, y64)
    torch.cuda.synchronize()
    plan._native_plan.device_status()
    ref64 = oracle.apply_rows(n, xm, zm, wp, x64.cpu().numpy().astype(np.complex128), rows)
    _c64_close(_take(y64, rows), ref64, "random 2000 words n=28 (2^18 rows)")
    del x64, y64
    torch.cuda.empty_cache()


def test_random_2000_words_n24_full_vector_host_and_device_entries() -> None:
    n = 24
    op = PauliOperator.from_code_arrays(*workloads.random_k_local(n=n, words=2000))
    plan = op.native_mvp_plan()
    state = workloads.random_state(n, seed=24)
    xm, zm, wp = _terms(op)
    ref = oracle.apply_term_direct(n, xm, zm, wp, state)

    _fp64_close(plan.apply(state), ref)  # host entry, complex128
    x = torch.from_numpy(state).cuda()
    y = torch.empty_like(x)
    plan.apply_device(x, y)  # device entry, complex128
    torch.cuda.synchronize()
    _fp64_close(y.cpu().numpy(), ref)

    s64 = state.astype(np.complex64)
    ref64 = oracle.apply_term_direct(n, xm, zm, wp, s64.astype(np.complex128))
    _c64_close(plan._native_plan.apply_c64(s64), ref64, "random 2000 words n=24 host entry")
    x64 = torch.from_numpy(s64).cuda()
    y64 = torch.empty_like(x64)
    plan.apply_device(x64, y64)
    torch.cuda.synchronize()
    plan._native_plan.device_status()
    _c64_close(y64.cpu().numpy(), ref64, "random 2000 words n=24 device entry")


def test_batched_64_lattices_every_member_and_rhs() -> None:
    members = workloads.batched_heisenberg_set(64)
    ops = [PauliOperator.from_code_arrays(c, w) for _, c, w in members]
    assert sorted({op.nqubits for op in ops})[0] >= 16 and max(op.nqubits for op in ops) <= 26
    plans = [op.native_mvp_plan() for op in ops]
    nrhs = 8
    xs = [workloads.random_state_device(op.nqubits, seed=900 + i, dtype=torch.complex64, nrhs=nrhs)
          for i, op in enumerate(ops)]
    ys = [torch.full_like(x, float("nan")) for x in xs]
    batch = BatchedMVP(plans, nrhs=nrhs, dtype="complex64")
    batch.autotune(xs, ys, cache_path=None, repeats=1)
    for y in ys:
        y.fill_(float("nan"))
    batch.apply(xs, ys)  # graph replay with the tuned shape
    torch.cuda.synchronize()
    batch.device_status()
    worst = 0.0
    for i, (op, x, y) in enumerate(zip(ops, xs, ys)):
        xm, zm, wp = _terms(op)
        rows = _rows(1 << op.nqubits, 1024, seed=i)
        idx = torch.from_numpy(rows.astype(np.int64)).cuda()
        for v in range(nrhs):
            ref = oracle.apply_rows(op.nqubits, xm, zm, wp, x[v].cpu().numpy().astype(np.complex128), rows)
            got = y[v][idx].cpu().numpy().astype(np.complex128)
            rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            assert rel <= C64_NORM_RTOL, (i, op.nqubits, v, rel)
            worst = max(worst, rel)
    print(f"batched 64 lattices x 8 RHS: worst complex64 norm-relative row error {worst:.3e}")


def test_jordan_wigner_n28_rows_and_n20_full_vector() -> None:
    h, g = chemistry_integrals(28, seed=20261203)
    op = PauliOperator.from_code_arrays(*jordan_wigner_integrals(h, g))
    assert op.term_count == 347513
    plan = op.native_mvp_plan()
    x = workloads.random_state_device(28, seed=5)
    y = torch.empty_like(x)
    plan.apply_device(x, y)
    torch.cuda.synchronize()
    plan._native_plan.device_status()
    rows = _rows(1 << 28, 2048, seed=5)
    xm, zm, wp = _terms(op)
    _fp64_close(_take(y, rows), oracle.apply_rows(28, xm, zm, wp, x.cpu().numpy(), rows))
    del x, y, plan
    torch.cuda.empty_cache()

    h, g = chemistry_integrals(20, seed=20261203)
    op = PauliOperator.from_code_arrays(*jordan_wigner_integrals(h, g))
    plan = op.native_mvp_plan()
    state = workloads.random_state(20, seed=6)
    xm, zm, wp = _terms(op)
    ref = oracle.apply_term_direct(20, xm, zm, wp, state)
    _fp64_close(plan.apply(state), ref)
    s64 = state.astype(np.complex64)
    ref64 = oracle.apply_term_direct(20, xm, zm, wp, s64.astype(np.complex128))
    _c64_close(plan._native_plan.apply_c64(s64), ref64, "Jordan-Wigner n=20 full vector")
