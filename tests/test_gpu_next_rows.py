"""GPU checks of the rows next to the MVP: the backend plan's device callable
(no host copies) and the Jordan-Wigner chemistry workload through the MVP,
against the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, workloads  # noqa: E402
from tencirpauli_b200.mapping import chemistry_integrals, jordan_wigner_integrals  # noqa: E402


def _oracle(op, state):
    xm, zm, wp = oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)
    return oracle.apply_term_direct(op.nqubits, xm, zm, wp, state)


def test_backend_plan_host_and_device_paths() -> None:
    codes, coeffs = workloads.random_k_local(n=13, words=90, seed=21)
    op = PauliOperator.from_code_arrays(codes, coeffs * (1 - 0.5j))
    plan = op.backend_mvp_plan() if hasattr(op, "backend_mvp_plan") else op.compile("backend_mvp")
    state = workloads.random_state(13, seed=4)
    ref = _oracle(op, state)
    np.testing.assert_allclose(plan.apply(state), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    f = plan.device_callable()
    x = torch.from_numpy(state).cuda()
    y = f(x)
    assert y.device.type == "cuda" and y.dtype == torch.complex128
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    # DLPack from another producer: an object that only speaks the protocol
    # (as CuPy or JAX arrays do), and a bare capsule, take the same path
    class Foreign:
        def __init__(self, t):
            self._t = t

        def __dlpack__(self, *args, **kwargs):
            return self._t.__dlpack__(*args, **kwargs)

        def __dlpack_device__(self):
            return self._t.__dlpack_device__()

    y2 = plan.apply(Foreign(x))
    assert isinstance(y2, torch.Tensor) and torch.equal(y2, y)
    y3 = f(torch.utils.dlpack.to_dlpack(x.clone()))
    assert torch.equal(y3, y)
    block = torch.stack([x, 2 * x]).to(torch.complex64)
    yb = f(block)
    assert yb.shape == block.shape and yb.dtype == torch.complex64
    rel = np.linalg.norm(yb[1].cpu().numpy() - 2 * ref) / np.linalg.norm(2 * ref)
    assert rel <= 2e-6


def test_jordan_wigner_chemistry_mvp_matches_oracle() -> None:
    n = 12
    h, g = chemistry_integrals(n, seed=5)
    op = PauliOperator.from_code_arrays(*jordan_wigner_integrals(h, g))
    assert op.term_count > 1000
    state = workloads.random_state(n, seed=6)
    ref = _oracle(op, state)
    y = op.native_mvp_plan().apply(state)
    scale = np.abs(ref).max()
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12 * scale)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-12
