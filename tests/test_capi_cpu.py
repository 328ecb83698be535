"""CPU-only checks of the C-ABI library: it loads, exports every declared
symbol, and its host-side entry points (canonicalization, plan-budget errors)
behave as the reference's.  No kernel is launched here."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden
from oracle import oracle
from tencirpauli_b200 import _native


def _declared_functions(name: str = "tcp_mvp.h") -> list:
    header = open(os.path.join(ROOT, "include", name)).read()
    header = re.sub(r"/\*.*?\*/", "", header, flags=re.S)
    return sorted(set(re.findall(r"\b(tcp_[a-z0-9_]+)\s*\(", header)))


def test_library_loads_and_exports_every_declared_symbol() -> None:
    lib = _native.load_library()
    declared = _declared_functions()
    assert declared, "no functions parsed from include/tcp_mvp.h"
    assert set(declared) == set(_native.EXPORTED_SYMBOLS)
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.tcp_abi_version() == 1
    solver = _declared_functions("tcp_solver.h")
    assert set(solver) == set(_native.SOLVER_SYMBOLS)
    for name in solver:
        assert hasattr(lib, name), name
    matrix = _declared_functions("tcp_matrix.h")
    assert set(matrix) == set(_native.MATRIX_SYMBOLS)
    for name in matrix:
        assert hasattr(lib, name), name
    probe = _declared_functions("tcp_probe.h")
    assert set(probe) == set(_native.PROBE_SYMBOLS)
    for name in probe:
        assert hasattr(lib, name), name
    sector = _declared_functions("tcp_sector.h")
    assert set(sector) == set(_native.SECTOR_SYMBOLS)
    for name in sector:
        assert hasattr(lib, name), name
    assert lib.tcp_mlp_train_work_bytes() == 296 * 434 * 4
    assert lib.tcp_gram_work_bytes(4, 3) == 296 * 12 * 16


def test_canonicalize_matches_reference_known_answers() -> None:
    k = load_golden("canonical_known_answers")
    for prefix in ("a", "b"):
        codes = k[f"{prefix}_codes"]
        n = codes.shape[1]
        x, z, c = _native.canonicalize(n, codes, k[f"{prefix}_coefficients"])
        ex, ez = oracle.encode_codes(n, k[f"{prefix}_expected_codes"])
        np.testing.assert_array_equal(x, ex)
        np.testing.assert_array_equal(z, ez)
        np.testing.assert_array_equal(c, k[f"{prefix}_expected_coefficients"])


@pytest.mark.parametrize("seed", range(6))
def test_canonicalize_matches_oracle_bitwise(seed: int) -> None:
    rng = np.random.default_rng(seed)
    n = int(rng.integers(0, 70))
    count = int(rng.integers(0, 200))
    # few distinct words so that duplicates (and exact cancellations) occur
    base = rng.integers(0, 4, size=(max(1, count // 3), n)).astype(np.uint8)
    codes = base[rng.integers(0, base.shape[0], size=count)] if count else np.zeros((0, n), np.uint8)
    coeffs = rng.normal(size=count) + 1j * rng.normal(size=count)
    if count > 4:
        codes[1] = codes[0]
        coeffs[1] = -coeffs[0]
        coeffs[2] = 0.0
        coeffs[3] = -0.0 + 0.0j
    x, z, c = _native.canonicalize(n, codes, coeffs)
    ox, oz, oc = oracle.canonicalize(n, codes, coeffs)
    np.testing.assert_array_equal(x, ox)
    np.testing.assert_array_equal(z, oz)
    assert c.tobytes() == oc.tobytes()


def test_canonicalize_error_statuses() -> None:
    with pytest.raises(ValueError, match="invalid Pauli code 4 at index 1"):
        _native.canonicalize(2, np.asarray([[1, 4]], np.uint8), np.asarray([1.0 + 0j]))
    with pytest.raises(ValueError, match="coefficient at index 0 is not finite"):
        _native.canonicalize(1, np.asarray([[1]], np.uint8), np.asarray([np.inf + 0j]))


def test_last_error_is_thread_local_text() -> None:
    with pytest.raises(ValueError):
        _native.canonicalize(1, np.asarray([[9]], np.uint8), np.asarray([1.0 + 0j]))
    assert "invalid Pauli code 9" in _native.last_error()


def test_last_error_fields_rebuild_the_pauli_error_variant() -> None:
    """tcp_last_error_fields returns the numeric fields of the PauliError
    variant (crates/tencir-pauli-core/src/error.rs:5-74) beside the status."""
    with pytest.raises(ValueError):
        _native.canonicalize(2, np.asarray([[1, 4]], np.uint8), np.asarray([1.0 + 0j]))
    assert _native.last_error_fields() == (_native.TCP_ERR_INVALID_CODE, 4, 1)
    with pytest.raises(ValueError):
        _native.canonicalize(1, np.asarray([[1], [2]], np.uint8), np.asarray([1.0 + 0j, np.nan + 0j]))
    assert _native.last_error_fields() == (_native.TCP_ERR_NON_FINITE_COEFFICIENT, 1, 0)
    lib = _native.load_library()
    x = np.asarray([1], dtype=np.uint64)
    c = np.asarray([1.0, 0.0], dtype=np.float64)
    p64 = ctypes.POINTER(ctypes.c_uint64)
    pf = ctypes.POINTER(ctypes.c_double)
    handle = ctypes.c_void_p(None)
    assert lib.tcp_mvp_plan_create(2, 1, 3, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf), 0, 0,
                                   ctypes.byref(handle)) == _native.TCP_ERR_INVALID_WORD_LENGTH
    assert _native.last_error_fields() == (_native.TCP_ERR_INVALID_WORD_LENGTH, 1, 3)
    # eager budget: one group on 30 qubits needs 2^30 * 16 + 2 * 32 + 32 bytes
    assert lib.tcp_mvp_plan_create(30, 1, 1, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf),
                                   _native.TCP_STORAGE_EAGER, 1000, ctypes.byref(handle)) == _native.TCP_ERR_MEMORY_LIMIT
    assert _native.last_error_fields() == (_native.TCP_ERR_MEMORY_LIMIT, (1 << 30) * 16 + 96, 1000)
    assert lib.tcp_mvp_plan_create(64, 1, 1, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf), 0, 0,
                                   ctypes.byref(handle)) == _native.TCP_ERR_OVERFLOW
    assert _native.last_error_fields() == (_native.TCP_ERR_OVERFLOW, 0, 0)


def test_eager_budget_is_checked_before_any_device_use() -> None:
    # hamiltonian.rs:84-119: G * 2^n * 16 diagonal bytes against max_bytes
    lib = _native.load_library()
    x = np.asarray([1], dtype=np.uint64)
    z = np.asarray([0], dtype=np.uint64)
    c = np.asarray([1.0, 0.0], dtype=np.float64)
    handle = ctypes.c_void_p(None)
    status = lib.tcp_mvp_plan_create(
        30,
        1,
        1,
        x.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
        z.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
        c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        _native.TCP_STORAGE_EAGER,
        1 << 30,
        ctypes.byref(handle),
    )
    assert status == _native.TCP_ERR_MEMORY_LIMIT
    assert "exceeds memory limit 1073741824" in _native.last_error()
    assert handle.value is None


def test_plan_create_argument_errors() -> None:
    lib = _native.load_library()
    handle = ctypes.c_void_p(None)
    x = np.zeros(2, np.uint64)
    c = np.zeros(2, np.float64)
    p64 = ctypes.POINTER(ctypes.c_uint64)
    pf = ctypes.POINTER(ctypes.c_double)
    # bad storage label -> InvalidSector
    assert (
        lib.tcp_mvp_plan_create(2, 1, 1, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf), 7, 0, ctypes.byref(handle))
        == _native.TCP_ERR_INVALID_SECTOR
    )
    # wrong packed word count -> InvalidWordLength (pauli_action.rs:38-50)
    assert (
        lib.tcp_mvp_plan_create(2, 1, 2, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf), 0, 0, ctypes.byref(handle))
        == _native.TCP_ERR_INVALID_WORD_LENGTH
    )
    assert "expected 1 packed words, got 2" in _native.last_error()
    # n >= 64 -> Overflow
    assert (
        lib.tcp_mvp_plan_create(64, 1, 1, x.ctypes.data_as(p64), x.ctypes.data_as(p64), c.ctypes.data_as(pf), 0, 0, ctypes.byref(handle))
        == _native.TCP_ERR_OVERFLOW
    )
    # non-finite coefficient
    bad = np.asarray([np.nan, 0.0])
    assert (
        lib.tcp_mvp_plan_create(2, 1, 1, x.ctypes.data_as(p64), x.ctypes.data_as(p64), bad.ctypes.data_as(pf), 0, 0, ctypes.byref(handle))
        == _native.TCP_ERR_NON_FINITE_COEFFICIENT
    )
    assert lib.tcp_mvp_plan_create(2, 0, 1, None, None, None, 0, 0, None) == _native.TCP_ERR_INVALID_ARGUMENT


def test_solver_kernel_limits_are_checked_before_any_launch() -> None:
    """tcp_gram / tcp_block_combine reject shapes outside their launch limits
    with InvalidArgument, and empty problems return at once; none of these
    calls reaches the device."""
    lib = _native.load_library()
    dummy = ctypes.c_void_p(16)  # never dereferenced: every call below returns before a launch
    c128, c64 = _native.TCP_DTYPE_C128, _native.TCP_DTYPE_C64
    bad = _native.TCP_ERR_INVALID_ARGUMENT
    # Gram: p + q <= 96, p * q <= 512, known storage types
    assert lib.tcp_gram(dummy, c128, 90, dummy, c128, 7, 1024, dummy, dummy, None) == bad
    assert "p + q <= 96" in _native.last_error()
    assert lib.tcp_gram(dummy, c64, 40, dummy, c64, 13, 1024, dummy, dummy, None) == bad
    assert lib.tcp_gram(dummy, 5, 4, dummy, c128, 4, 1024, dummy, dummy, None) == bad
    assert lib.tcp_gram(dummy, c128, 0, dummy, c128, 4, 1024, dummy, dummy, None) == 0
    assert lib.tcp_gram(None, c128, 4, dummy, c128, 4, 1024, dummy, dummy, None) == bad
    # combine: up to 32 outputs, p x (outputs rounded up to 4, 8, 16 or 32) <= 6144
    assert lib.tcp_block_combine(dummy, c128, 8, dummy, 33, 1024, 1.0, 0.0, dummy, c128, None) == bad
    assert "k <= 32" in _native.last_error()
    assert lib.tcp_block_combine(dummy, c64, 400, dummy, 17, 1024, 1.0, 0.0, dummy, c64, None) == bad
    assert "coefficient block too large" in _native.last_error()
    assert lib.tcp_block_combine(dummy, c64, 192, dummy, 17, 0, 1.0, 0.0, dummy, c64, None) == 0
    assert lib.tcp_block_combine(dummy, c128, 8, dummy, 0, 1024, 1.0, 0.0, dummy, c128, None) == 0
    assert lib.tcp_block_combine(None, c128, 8, dummy, 4, 1024, 1.0, 0.0, dummy, c128, None) == bad


def test_noalloc_entry_point_names_no_allocating_routine() -> None:
    """The allocation-free host apply and its set-up name no allocating
    routine.  Its GPU test makes the library's own allocator fail; this source
    check also covers direct CUDA allocation calls added later."""
    path = os.path.join(ROOT, "tencirpauli_b200", "csrc", "tcp_mvp.cu")
    src = open(path).read()
    start = src.index("int noalloc_scratch(int device, unsigned char **out)")
    body = src[start:]
    forbidden = ("cudaMalloc", "cudaFree", "dev_malloc", "cudaHostAlloc", "cudaMallocHost", "malloc(", "new ")
    for name in forbidden:
        assert name not in body, f"{name} appears in the allocation-free path"


def test_debug_bounds_build_compiles() -> None:
    """The TCP_DEBUG_BOUNDS variant of the hot kernel's translation unit
    compiles for sm_100a (the full library is built on demand with
    ``python -m tencirpauli_b200.build --debug-bounds``)."""
    import subprocess
    import tempfile

    from tencirpauli_b200 import build

    src = os.path.join(ROOT, "tencirpauli_b200", "csrc", "tcp_mvp.cu")
    with tempfile.TemporaryDirectory() as tmp:
        proc = subprocess.run(
            [build.nvcc(), *build.ARCH, "-O1", "-std=c++17", "--expt-relaxed-constexpr", "-DTCP_DEBUG_BOUNDS", "-c", src,
             "-o", os.path.join(tmp, "tcp_mvp_debug.o")],
            capture_output=True, text=True,
        )
    assert proc.returncode == 0, proc.stderr[-2000:]
