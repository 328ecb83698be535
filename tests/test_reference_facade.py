"""The reference's own Python facade driven through this library's shim.

``python/tencirpauli/pauli.py``, ``hamiltonian.py`` and ``_native_mvp.py`` of
the reference checkout are imported as the package ``tencirpauli`` whose
compiled extension ``_native`` is replaced by
``tencirpauli_b200.integrations.reference_native`` -- the binding a
maintainer would install.  ``PauliOperator.from_code_arrays``,
``.native_mvp_plan()``, ``.mvp()`` and ``NativeMVPPlan.apply`` /
``apply_into`` then run the reference's facade code over this library's
``NativeMvpPlan`` class (argument marshalling, strict-buffer checks, error
mapping) and its host canonicalization.

These tests run where the reference checkout exists, which is a machine
without a GPU: there, the plan's four device-side C-ABI calls (plan create,
info, host apply, destroy) are answered by a CPU stand-in that computes with
the oracle, while every other call (canonicalization, error text, error
fields) goes to ``libtcpmvp.so`` itself, and plan creation still runs the
library's own argument and budget checks first.  On a GPU machine the same
class calls the library for all of them; the GPU suite covers that half.
"""

from __future__ import annotations

import ctypes
import importlib
import os
import sys
import threading
import types

import numpy as np
import pytest

from conftest import golden_mvp_names, load_golden
from oracle import oracle
from tencirpauli_b200 import _native
from tencirpauli_b200.integrations import reference_native

REFERENCE = os.environ.get("TCP_REFERENCE_CHECKOUT", "/root/reference")
FACADE = os.path.join(REFERENCE, "python", "tencirpauli")

pytestmark = pytest.mark.skipif(
    not os.path.exists(os.path.join(FACADE, "pauli.py")),
    reason="the reference checkout (python/tencirpauli) is not on this machine",
)


class _DeviceStandIn:
    """libtcpmvp.so with its device-side plan entries computed on the CPU by
    the oracle (this machine has no GPU); every other symbol is the library's."""

    def __init__(self, real: ctypes.CDLL) -> None:
        self._real = real
        self._plans = {}
        self._next = 1
        self._message = None

    def __getattr__(self, name: str):
        return getattr(self._real, name)

    def _fail(self, status: int, message: str) -> int:
        self._message = message
        return status

    def tcp_last_error(self, buf, cap):
        if self._message is None:
            return self._real.tcp_last_error(buf, cap)
        data = self._message.encode()[: max(0, int(cap) - 1)] + b"\0"
        ctypes.memmove(buf, data, len(data))
        return len(self._message)

    def tcp_mvp_plan_create(self, n, count, width, xp, zp, cp, storage, max_bytes, out):
        self._message = None
        # the library's own host checks (word length, finiteness, storage
        # label, eager budget) come first; without a device it then stops at
        # the device query
        probe = ctypes.c_void_p(None)
        status = self._real.tcp_mvp_plan_create(n, count, width, xp, zp, cp, storage, max_bytes, ctypes.byref(probe))
        if status not in (_native.TCP_OK, _native.TCP_ERR_CUDA):
            return status
        k = max(int(count), 1)
        x = np.ctypeslib.as_array(xp, shape=(k * width,)).copy().reshape(k, width)[: int(count)]
        z = np.ctypeslib.as_array(zp, shape=(k * width,)).copy().reshape(k, width)[: int(count)]
        c = np.ctypeslib.as_array(cp, shape=(2 * k,)).copy().view(np.complex128)[: int(count)]
        xm, zm, wp = oracle.matrix_terms(int(n), x, z, c)
        plan = {"n": int(n), "terms": (xm, zm, wp), "count": int(count),
                "groups": oracle.group_count(xm) if int(count) else 0,
                "transitions": oracle.transition_count(int(n), xm, zm, wp) if storage == _native.TCP_STORAGE_EAGER else -1}
        handle = self._next
        self._next += 1
        self._plans[handle] = plan
        out._obj.value = handle
        return _native.TCP_OK

    def tcp_mvp_plan_info(self, handle, info_ref):
        plan = self._plans[handle.value]
        info = info_ref._obj
        info.nqubits = plan["n"]
        info.word_count = plan["n"] // 64 + (plan["n"] % 64 != 0)
        info.dimension = 1 << plan["n"]
        info.term_count = plan["count"]
        info.group_count = plan["groups"]
        info.transition_count = plan["transitions"]
        return _native.TCP_OK

    def tcp_mvp_apply_into_host(self, handle, sp, slen, op, olen, max_bytes):
        self._message = None
        plan = self._plans[handle.value]
        dim = 1 << plan["n"]
        for length in (int(slen), int(olen)):
            if length != dim:
                return self._fail(_native.TCP_ERR_INVALID_STRUCTURE_LENGTH, f"expected structure length {dim}, got {length}")
        state = np.ctypeslib.as_array(sp, shape=(2 * dim,)).view(np.complex128)
        out = np.ctypeslib.as_array(op, shape=(2 * dim,)).view(np.complex128)
        xm, zm, wp = plan["terms"]
        out[:] = oracle.apply_term_direct(plan["n"], xm, zm, wp, state) if plan["count"] else 0
        return _native.TCP_OK

    def tcp_mvp_plan_destroy(self, handle):
        self._plans.pop(handle.value, None)
        return _native.TCP_OK


@pytest.fixture(scope="module")
def facade():
    real = _native.load_library()
    saved_lib = _native._lib
    saved_modules = {k: v for k, v in sys.modules.items() if k == "tencirpauli" or k.startswith("tencirpauli.")}
    for k in saved_modules:
        del sys.modules[k]
    _native._lib = _DeviceStandIn(real)
    package = types.ModuleType("tencirpauli")
    package.__path__ = [FACADE]
    extension = types.ModuleType("tencirpauli._native")
    for name in reference_native.__all__:
        setattr(extension, name, getattr(reference_native, name))
    extension.NativeMvpPlan = _native.NativeMvpPlan
    sys.modules["tencirpauli"] = package
    sys.modules["tencirpauli._native"] = extension
    package._native = extension
    try:
        pauli = importlib.import_module("tencirpauli.pauli")
        yield pauli
    finally:
        _native._lib = saved_lib
        for k in [k for k in sys.modules if k == "tencirpauli" or k.startswith("tencirpauli.")]:
            del sys.modules[k]
        sys.modules.update(saved_modules)


@pytest.mark.parametrize("name", golden_mvp_names())
@pytest.mark.parametrize("storage", ["lazy", "eager"])
def test_golden_vectors_through_the_reference_facade(facade, name: str, storage: str) -> None:
    g = load_golden(name)
    n = int(g["nqubits"])
    op = facade.PauliOperator.from_code_arrays(g["codes"].reshape(len(g["coefficients"]), n), g["coefficients"])
    plan = op.native_mvp_plan(storage=storage)
    assert isinstance(plan._execution, _native.NativeMvpPlan)
    np.testing.assert_allclose(plan.apply(g["state"]), g["expected"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(op.mvp(g["state"]), g["expected"], rtol=1e-12, atol=1e-12)
    out = np.full(1 << n, 7.0 - 3.0j)
    plan.apply_into(np.ascontiguousarray(g["state"], dtype=np.complex128), out)
    np.testing.assert_allclose(out, g["expected"], rtol=1e-12, atol=1e-12)
    assert plan.retained_format == ("compact_graph" if storage == "eager" else "compiled_actions")
    if storage == "eager":
        xm, zm, wp = oracle.matrix_terms(n, op._native_handle._x, op._native_handle._z, op._native_handle._coefficients)
        assert plan.transition_count == oracle.transition_count(n, xm, zm, wp)
    else:
        assert plan.transition_count is None


def test_abi_fixed_vector_and_metadata(facade) -> None:
    # tests/test_native_abi.py:84-120 of the reference: H = 2Z + I, [1, 2] -> [3, -2]
    op = facade.PauliOperator.from_terms(1, [("Z", 2.0), ("I", 1.0)])
    plan = op.native_mvp_plan()
    np.testing.assert_array_equal(plan.apply([1.0, 2.0]), [3.0, -2.0])
    assert plan.nqubits == 1 and plan.term_count == 2
    assert plan._execution.native_variant == "pauli"


def test_overwrite_concurrency_and_buffer_contract(facade) -> None:
    # tests/test_native_mvp_resources.py:173-311 of the reference
    g = load_golden("random_differential_6")
    op = facade.PauliOperator.from_code_arrays(g["codes"], g["coefficients"])
    plan = op.native_mvp_plan()
    state = np.ascontiguousarray(g["state"], dtype=np.complex128)
    original = state.copy()
    expected = plan.apply(state)
    outs = [np.full(64, 9.0 + 3.0j), np.full(64, -4.0 + 2.0j)]
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
    with pytest.raises(ValueError):
        plan.apply_into(state, state)  # overlapping buffers
    with pytest.raises(TypeError):
        plan.apply_into(state.astype(np.complex64), np.empty_like(state))
    with pytest.raises(ValueError, match="expected structure length 64, got 3"):
        plan._execution.apply(np.ones(3, np.complex128), 0)


def test_errors_keep_the_reference_exception_types(facade) -> None:
    with pytest.raises(ValueError, match="storage must be either 'eager' or 'lazy'"):
        facade.PauliOperator.from_terms(1, [("Z", 1.0)]).native_mvp_plan(storage="dense")
    # eager budget: MemoryLimit -> MemoryError (convert.rs:35-42); limits
    # below the facade's 1 GiB floor are advisory, so the operator is sized
    # past it (one group of 2^27 complex128 diagonal entries = 2 GiB)
    op = facade.PauliOperator.from_terms(27, [("X" + "I" * 26, 1.0)])
    with pytest.raises(MemoryError):
        op.native_mvp_plan(storage="eager", max_bytes=1 << 30)
    assert _native.last_error_fields()[0] == _native.TCP_ERR_MEMORY_LIMIT
