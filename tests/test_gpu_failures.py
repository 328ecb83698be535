"""Failure detection on the GPU without faulting it: host-side allocation
failure injection, and a bounded device wait that runs out on purpose and
comes back as a status (the context stays usable)."""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, _native, workloads  # noqa: E402


def test_injected_allocation_failure_raises_memory_error_and_recovers() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(12))
    os.environ["TCP_FAIL_ALLOC_AFTER"] = "0"
    try:
        with pytest.raises(MemoryError, match="device allocation"):
            op.native_mvp_plan()
    finally:
        del os.environ["TCP_FAIL_ALLOC_AFTER"]
    plan = op.native_mvp_plan()
    state = workloads.random_state(12, seed=2)
    assert np.isfinite(plan.apply(state)).all()


def test_bounded_wait_expires_into_a_status_and_the_context_survives() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(12))
    plan = op.native_mvp_plan()
    lib = _native.load_library()
    status = lib.tcp_selftest_bounded_wait(plan._native_plan.handle, 1_000_000)  # 1 ms
    assert status == _native.TCP_ERR_DEVICE_TIMEOUT
    assert "bounded device-side wait expired" in _native.last_error()
    # the status word was cleared and the device still works
    plan._native_plan.device_status()
    state = workloads.random_state(12, seed=3)
    y = plan.apply(state)
    plan2 = op.native_mvp_plan()
    np.testing.assert_array_equal(plan2.apply(state), y)
