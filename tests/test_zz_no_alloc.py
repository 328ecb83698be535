"""The allocation-free host apply, ``tcp_mvp_apply_into_host_noalloc``.

Some callers must not allocate device memory while they apply an operator:
their own allocator owns the GPU's memory, or every allocation is reserved at
start-up.  This entry point stages the state and the result through a fixed
device array that belongs to the library (at most 2^20 amplitudes), instead of
the workspace that ``tcp_mvp_apply_into_host`` allocates.  These tests call it
through the C ABI and compare it with the existing host entry point at the
FP64 tolerance used by the other parity tests (rtol = 1e-12, atol = 1e-12 *
max|y|), on two calls in a row.  The file sorts last so a run that stops at
the first failure has already run every other test.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("CUDA device required", allow_module_level=True)

from tencirpauli_b200 import PauliOperator, _native, workloads  # noqa: E402

FP64_RTOL = 1e-12


def _noalloc(plan, state: np.ndarray, out: np.ndarray) -> int:
    lib = _native.load_library()
    dp = ctypes.POINTER(ctypes.c_double)
    return lib.tcp_mvp_apply_into_host_noalloc(
        plan._native_plan.handle,
        state.view(np.float64).ctypes.data_as(dp),
        state.shape[0],
        out.view(np.float64).ctypes.data_as(dp),
        out.shape[0],
        None,
    )


@pytest.mark.parametrize(
    "codes_coeffs",
    [
        workloads.heisenberg_chain(16),  # tiled kernel (n >= 12)
        workloads.random_k_local(n=10, words=40, seed=4),  # row kernel (n < 12)
        workloads.heisenberg_chain(20),  # the largest size the static scratch holds
    ],
    ids=["chain16", "random10", "chain20"],
)
def test_noalloc_matches_existing_entry_on_two_calls_in_a_row(codes_coeffs) -> None:
    op = PauliOperator.from_code_arrays(*codes_coeffs)
    plan = op.native_mvp_plan()
    n = op.nqubits
    for call, seed in enumerate((101, 202)):
        state = workloads.random_state(n, seed=seed)
        expected = np.empty_like(state)
        plan.apply_into(state, expected)  # existing entry point, tcp_mvp_apply_into_host
        out = np.full_like(state, np.nan)
        # The allocation-injection hook makes any allocation through the
        # library's allocator fail; this entry point must not reach it.
        os.environ["TCP_FAIL_ALLOC_AFTER"] = "0"
        try:
            status = _noalloc(plan, state, out)
        finally:
            del os.environ["TCP_FAIL_ALLOC_AFTER"]
        assert status == _native.TCP_OK, _native.last_error()
        scale = float(np.max(np.abs(expected)))
        np.testing.assert_allclose(out, expected, rtol=FP64_RTOL, atol=FP64_RTOL * scale, err_msg=f"call {call}")


def test_noalloc_rejects_sizes_beyond_the_static_maximum() -> None:
    op = PauliOperator.from_code_arrays(*workloads.heisenberg_chain(21))
    plan = op.native_mvp_plan()
    state = np.zeros(1 << 21, dtype=np.complex128)
    out = np.zeros_like(state)
    status = _noalloc(plan, state, out)
    assert status == _native.TCP_ERR_MEMORY_LIMIT
    assert "at most 20 qubits" in _native.last_error()
    short = np.zeros(8, dtype=np.complex128)
    small = PauliOperator.from_terms(2, [("XZ", 1.0)]).native_mvp_plan()
    assert _noalloc(small, short, np.zeros(4, np.complex128)) == _native.TCP_ERR_INVALID_STRUCTURE_LENGTH
