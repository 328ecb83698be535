"""ctypes binding of ``libtcpmvp.so`` (the C ABI declared in ``include/tcp_mvp.h``).

This module is the process-internal boundary that replaces the reference's
PyO3 extension ``tencirpauli._native`` for the MVP path
(``crates/tencirpauli-native/src/hamiltonian.rs:31-194`` and
``crates/tencirpauli-native/src/operator.rs:164-267``).  It loads the in-tree
CUDA library and fails loudly when it is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
import sys
import threading
from typing import Any, Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TCP_LIBRARY=debug loads the TCP_DEBUG_BOUNDS build (python -m tencirpauli_b200.build --debug-bounds)
LIBRARY_PATH = os.path.join(_HERE, "_lib", "libtcpmvp_debug.so" if os.environ.get("TCP_LIBRARY") == "debug" else "libtcpmvp.so")

# Status codes of include/tcp_mvp.h
TCP_OK = 0
TCP_ERR_INVALID_CODE = 1
TCP_ERR_INVALID_WORD_LENGTH = 2
TCP_ERR_INCOMPATIBLE_QUBITS = 3
TCP_ERR_INVALID_STRUCTURE_LENGTH = 4
TCP_ERR_NON_FINITE_COEFFICIENT = 5
TCP_ERR_NON_CANONICAL_TERMS = 7
TCP_ERR_OVERFLOW = 8
TCP_ERR_MEMORY_LIMIT = 9
TCP_ERR_INVALID_SECTOR = 10
TCP_ERR_SECTOR_LEAKAGE = 11
TCP_ERR_INVALID_INDEX = 13
TCP_ERR_INVALID_ARGUMENT = 32
TCP_ERR_CUDA = 33
TCP_ERR_DEVICE_TIMEOUT = 34
TCP_ERR_ALLOCATION = 35
TCP_ERR_WRONG_DEVICE = 36

TCP_STORAGE_LAZY = 0
TCP_STORAGE_EAGER = 1
TCP_DTYPE_C128 = 0
TCP_DTYPE_C64 = 1

U64_MAX = (1 << 64) - 1

# Every symbol include/tcp_mvp.h declares.
EXPORTED_SYMBOLS = (
    "tcp_abi_version",
    "tcp_last_error",
    "tcp_last_error_fields",
    "tcp_pauli_canonicalize",
    "tcp_mvp_plan_create",
    "tcp_mvp_plan_destroy",
    "tcp_mvp_plan_info",
    "tcp_mvp_apply_into_host",
    "tcp_mvp_apply_into_host_c64",
    "tcp_mvp_apply_into_device",
    "tcp_mvp_apply_add_device",
    "tcp_mvp_apply_into_host_noalloc",
    "tcp_mvp_plan_device_status",
    "tcp_selftest_bounded_wait",
    "tcp_mvp_transition_count",
    "tcp_mvp_diagonal_device",
    "tcp_mvp_batch_create",
    "tcp_mvp_batch_destroy",
    "tcp_mvp_batch_configure",
    "tcp_mvp_batch_autotune",
    "tcp_mvp_batch_apply",
    "tcp_mvp_batch_info",
    "tcp_mvp_batch_device_status",
)

# Every symbol include/tcp_solver.h declares.
SOLVER_SYMBOLS = (
    "tcp_gram_work_bytes",
    "tcp_gram",
    "tcp_block_combine",
    "tcp_precond_jacobi",
    "tcp_state_features",
    "tcp_precond_mlp",
    "tcp_mlp_inputs",
    "tcp_mlp_train_work_bytes",
    "tcp_mlp_train_step",
    "tcp_mlp_forward",
    "tcp_mlp_backward_step",
    "tcp_mlp_alignment_work_bytes",
    "tcp_mlp_alignment_grad",
)


# Every symbol include/tcp_sector.h declares.
SECTOR_SYMBOLS = (
    "tcp_u1_dimension",
    "tcp_u1_rank_words",
    "tcp_u1_unrank_words",
    "tcp_u1_basis_words",
    "tcp_pauli_number_commutator",
    "tcp_u1_plan_create",
    "tcp_u1_plan_destroy",
    "tcp_u1_plan_info",
    "tcp_u1_apply_into_host",
    "tcp_u1_apply_into_device",
    "tcp_u1_diagonal_device",
    "tcp_u1_transition_count",
    "tcp_u1_csr",
    "tcp_u1_plan_device_status",
)


# Every symbol include/tcp_matrix.h declares.
MATRIX_SYMBOLS = ("tcp_mvp_dense", "tcp_mvp_sparse_count", "tcp_mvp_csr")
TCP_MATRIX_COO = 0
TCP_MATRIX_CSR = 1

# Every symbol include/tcp_probe.h declares.
PROBE_SYMBOLS = ("tcp_probe_fma_rate", "tcp_probe_smem_rate")


class TcpU1PlanInfo(ctypes.Structure):
    _fields_ = [
        ("nqubits", ctypes.c_uint32),
        ("particle_number", ctypes.c_uint32),
        ("dimension", ctypes.c_uint64),
        ("term_count", ctypes.c_uint64),
        ("group_count", ctypes.c_uint64),
        ("storage", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("transition_count", ctypes.c_int64),
        ("device_bytes", ctypes.c_uint64),
        ("estimated_bytes", ctypes.c_uint64),
        ("complement", ctypes.c_uint32),
        ("rank_chunks", ctypes.c_uint32),
        ("tables_in_shared", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class TcpPlanInfo(ctypes.Structure):
    _fields_ = [
        ("nqubits", ctypes.c_uint32),
        ("word_count", ctypes.c_uint32),
        ("dimension", ctypes.c_uint64),
        ("term_count", ctypes.c_uint64),
        ("group_count", ctypes.c_uint64),
        ("storage", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("transition_count", ctypes.c_int64),
        ("device_bytes", ctypes.c_uint64),
        ("tile_bits", ctypes.c_uint32),
        ("log_threads", ctypes.c_uint32),
        ("steps", ctypes.c_uint64),
        ("outer_patterns", ctypes.c_uint64),
        ("ring_steps", ctypes.c_uint64),
        ("cosets", ctypes.c_uint64),
    ]


_lib: Optional[ctypes.CDLL] = None
_lib_lock = threading.Lock()


def load_library() -> ctypes.CDLL:
    """Load the in-tree CUDA library; raise ImportError when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"libtcpmvp.so is not built ({LIBRARY_PATH}); run "
                "`python -m tencirpauli_b200.build` (the MVP has no CPU fallback)"
            )
        lib = ctypes.CDLL(LIBRARY_PATH)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        f64p = ctypes.POINTER(ctypes.c_double)
        f32p = ctypes.POINTER(ctypes.c_float)
        vp = ctypes.c_void_p
        u32, u64, i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
        lib.tcp_abi_version.restype = i32
        lib.tcp_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        lib.tcp_last_error_fields.argtypes = [u64p]
        lib.tcp_last_error_fields.restype = i32
        lib.tcp_last_error.restype = ctypes.c_size_t
        lib.tcp_pauli_canonicalize.argtypes = [u32, u64, u8p, f64p, u64p, u64p, f64p, u64p, u64p]
        lib.tcp_mvp_plan_create.argtypes = [u32, u64, u32, u64p, u64p, f64p, i32, u64, ctypes.POINTER(vp)]
        lib.tcp_mvp_plan_destroy.argtypes = [vp]
        lib.tcp_mvp_plan_info.argtypes = [vp, ctypes.POINTER(TcpPlanInfo)]
        lib.tcp_mvp_apply_into_host.argtypes = [vp, f64p, u64, f64p, u64, u64]
        lib.tcp_mvp_apply_into_host_c64.argtypes = [vp, f32p, u64, f32p, u64]
        lib.tcp_mvp_apply_into_device.argtypes = [vp, vp, vp, u64, u32, i32, vp]
        lib.tcp_mvp_apply_add_device.argtypes = [vp, vp, vp, u64, u32, i32, vp]
        lib.tcp_mvp_apply_into_host_noalloc.argtypes = [vp, f64p, u64, f64p, u64, vp]
        lib.tcp_mvp_plan_device_status.argtypes = [vp]
        lib.tcp_selftest_bounded_wait.argtypes = [vp, u64]
        lib.tcp_mvp_transition_count.argtypes = [vp, u64p]
        lib.tcp_mvp_diagonal_device.argtypes = [vp, vp, u64, vp]
        vpp = ctypes.POINTER(vp)
        lib.tcp_mvp_batch_create.argtypes = [u32, vpp, u32, i32, vpp]
        lib.tcp_mvp_batch_destroy.argtypes = [vp]
        lib.tcp_mvp_batch_configure.argtypes = [vp, u32, u32]
        lib.tcp_mvp_batch_autotune.argtypes = [vp, vpp, vpp, ctypes.c_char_p, u32, vp]
        lib.tcp_mvp_batch_apply.argtypes = [vp, vpp, vpp, vp]
        lib.tcp_mvp_batch_info.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(u32), ctypes.POINTER(u64), ctypes.POINTER(u32)]
        lib.tcp_mvp_batch_device_status.argtypes = [vp]
        dbl, flt = ctypes.c_double, ctypes.c_float
        lib.tcp_gram_work_bytes.argtypes = [u32, u32]
        lib.tcp_gram_work_bytes.restype = ctypes.c_size_t
        lib.tcp_gram.argtypes = [vp, i32, u32, vp, i32, u32, u64, vp, vp, vp]
        lib.tcp_block_combine.argtypes = [vp, i32, u32, vp, u32, u64, dbl, dbl, vp, i32, vp]
        lib.tcp_precond_jacobi.argtypes = [vp, i32, u64, u32, vp, vp, dbl, vp, i32, vp]
        lib.tcp_state_features.argtypes = [vp, vp, u64, vp]
        lib.tcp_precond_mlp.argtypes = [vp, i32, u64, u32, vp, vp, vp, dbl, dbl, flt, vp, vp, i32, vp]
        lib.tcp_mlp_inputs.argtypes = [vp, vp, vp, vp, u32, dbl, dbl, vp, vp, vp]
        lib.tcp_mlp_train_work_bytes.argtypes = []
        lib.tcp_mlp_train_work_bytes.restype = ctypes.c_size_t
        lib.tcp_mlp_train_step.argtypes = [vp, vp, vp, vp, vp, vp, u32, vp, vp, vp, vp, flt, u32, vp, vp, vp]
        lib.tcp_mlp_forward.argtypes = [vp, u32, vp, vp, vp]
        lib.tcp_mlp_backward_step.argtypes = [vp, vp, u32, vp, vp, vp, vp, flt, u32, vp, vp]
        lib.tcp_mlp_alignment_work_bytes.argtypes = [u32]
        lib.tcp_mlp_alignment_work_bytes.restype = ctypes.c_size_t
        lib.tcp_mlp_alignment_grad.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, u32, u64, flt, vp, vp, vp, vp]
        lib.tcp_u1_dimension.argtypes = [u32, u32, u64p]
        lib.tcp_u1_rank_words.argtypes = [u32, u32, u64p, u32, u64p]
        lib.tcp_u1_unrank_words.argtypes = [u32, u32, u64, u64p, u32]
        lib.tcp_u1_basis_words.argtypes = [u32, u32, u64p, u64, u64]
        lib.tcp_pauli_number_commutator.argtypes = [u32, u64, u32, u64p, u64p, f64p, u64p]
        lib.tcp_u1_plan_create.argtypes = [u32, u32, u64, u32, u64p, u64p, f64p, i32, u64, ctypes.POINTER(vp)]
        lib.tcp_u1_plan_destroy.argtypes = [vp]
        lib.tcp_u1_plan_info.argtypes = [vp, ctypes.POINTER(TcpU1PlanInfo)]
        lib.tcp_u1_apply_into_host.argtypes = [vp, f64p, u64, f64p, u64, u64]
        lib.tcp_u1_apply_into_device.argtypes = [vp, vp, vp, u64, u32, i32, vp]
        lib.tcp_u1_diagonal_device.argtypes = [vp, vp, u64, vp]
        lib.tcp_u1_transition_count.argtypes = [vp, u64p]
        lib.tcp_u1_csr.argtypes = [vp, u64p, u64p, f64p, u64, u64p]
        lib.tcp_u1_plan_device_status.argtypes = [vp]
        for name in SECTOR_SYMBOLS:
            getattr(lib, name).restype = i32
        lib.tcp_mvp_dense.argtypes = [vp, f64p, u64, u64]
        lib.tcp_mvp_sparse_count.argtypes = [vp, i32, u64, u64p]
        lib.tcp_mvp_csr.argtypes = [vp, i32, u64, u64p, u64p, f64p, u64, u64p]
        for name in MATRIX_SYMBOLS:
            getattr(lib, name).restype = i32
        lib.tcp_probe_fma_rate.argtypes = [i32, u32, f64p, f64p]
        lib.tcp_probe_fma_rate.restype = i32
        lib.tcp_probe_smem_rate.argtypes = [u32, f64p, f64p]
        lib.tcp_probe_smem_rate.restype = i32
        for name in SOLVER_SYMBOLS:
            if not name.endswith("_work_bytes"):
                getattr(lib, name).restype = i32
        for name in EXPORTED_SYMBOLS:
            if name not in ("tcp_last_error",):
                getattr(lib, name).restype = i32
        _lib = lib
    return _lib


def last_error() -> str:
    lib = load_library()
    buf = ctypes.create_string_buffer(1024)
    lib.tcp_last_error(buf, len(buf))
    return buf.value.decode("utf-8", "replace")


def last_error_fields() -> Tuple[int, int, int]:
    """(status, field 0, field 1) of this thread's last error: the numeric
    fields of the matching PauliError variant (see tcp_last_error_fields)."""
    lib = load_library()
    fields = (ctypes.c_uint64 * 2)()
    status = lib.tcp_last_error_fields(fields)
    return int(status), int(fields[0]), int(fields[1])


class NativeDeviceError(RuntimeError):
    """A CUDA runtime failure or an expired device-side wait."""

    def __init__(self, message: str, status: int) -> None:
        super().__init__(message)
        self.status = status


def raise_for_status(status: int) -> None:
    """Map a C-ABI status to the reference's Python exception classes.

    ``crates/tencirpauli-native/src/convert.rs:35-42``: MemoryLimit ->
    MemoryError, Overflow -> OverflowError, every other PauliError ->
    ValueError.  Device failures raise :class:`NativeDeviceError`; a failed
    device allocation raises MemoryError.
    """
    if status == TCP_OK:
        return
    message = last_error()
    if status == TCP_ERR_MEMORY_LIMIT or status == TCP_ERR_ALLOCATION:
        raise MemoryError(message)
    if status == TCP_ERR_OVERFLOW:
        raise OverflowError(message)
    if status in (TCP_ERR_CUDA, TCP_ERR_DEVICE_TIMEOUT, TCP_ERR_WRONG_DEVICE):
        raise NativeDeviceError(message, status)
    raise ValueError(message)


def _ptr(array: np.ndarray, ctype: Any) -> Any:
    return array.ctypes.data_as(ctypes.POINTER(ctype))


def canonicalize(
    nqubits: int, codes: np.ndarray, coefficients: np.ndarray
) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Canonicalize code rows through ``tcp_pauli_canonicalize`` (no device needed)."""
    lib = load_library()
    count = int(coefficients.shape[0])
    width = nqubits // 64 + (nqubits % 64 != 0)
    codes = np.ascontiguousarray(codes, dtype=np.uint8).reshape(count, nqubits)
    coeffs = np.ascontiguousarray(coefficients, dtype=np.complex128)
    out_x = np.zeros((max(count, 1), width), dtype=np.uint64)
    out_z = np.zeros((max(count, 1), width), dtype=np.uint64)
    out_c = np.zeros(max(count, 1), dtype=np.complex128)
    out_n = np.zeros(1, dtype=np.uint64)
    bad = np.zeros(1, dtype=np.uint64)
    status = lib.tcp_pauli_canonicalize(
        nqubits,
        count,
        _ptr(codes, ctypes.c_uint8),
        _ptr(coeffs.view(np.float64), ctypes.c_double),
        _ptr(out_x, ctypes.c_uint64),
        _ptr(out_z, ctypes.c_uint64),
        _ptr(out_c.view(np.float64), ctypes.c_double),
        _ptr(out_n, ctypes.c_uint64),
        _ptr(bad, ctypes.c_uint64),
    )
    raise_for_status(status)
    t = int(out_n[0])
    return out_x[:t].copy(), out_z[:t].copy(), out_c[:t].copy()


class NativeMvpPlan:
    """Execution handle of one device plan (mirror of the PyO3 ``NativeMvpPlan``,
    ``crates/tencirpauli-native/src/hamiltonian.rs:31-34,137-194``).

    Exposes ``nqubits``, ``term_count``, ``transition_count``,
    ``native_variant == "pauli"``, ``apply(state, max_bytes)`` and
    ``apply_into(state, output, max_bytes)`` on host complex128 arrays, plus
    device-resident entry points for torch CUDA tensors.
    """

    native_variant = "pauli"

    def __init__(
        self,
        nqubits: int,
        x_words: np.ndarray,
        z_words: np.ndarray,
        coefficients: np.ndarray,
        storage: str = "lazy",
        max_bytes: int = sys.maxsize,
    ) -> None:
        lib = load_library()
        self._lib = lib
        self._handle = ctypes.c_void_p(None)
        if storage not in ("lazy", "eager"):
            raise ValueError("invalid sector: storage must be either 'eager' or 'lazy'")
        count = int(coefficients.shape[0])
        width = nqubits // 64 + (nqubits % 64 != 0)
        xw = np.ascontiguousarray(x_words, dtype=np.uint64).reshape(count * width)
        zw = np.ascontiguousarray(z_words, dtype=np.uint64).reshape(count * width)
        coeffs = np.ascontiguousarray(coefficients, dtype=np.complex128)
        if count == 0:  # keep valid pointers for empty operators
            xw = np.zeros(1, np.uint64)
            zw = np.zeros(1, np.uint64)
            coeffs = np.zeros(1, np.complex128)
        handle = ctypes.c_void_p(None)
        status = lib.tcp_mvp_plan_create(
            nqubits,
            count,
            width,
            _ptr(xw, ctypes.c_uint64),
            _ptr(zw, ctypes.c_uint64),
            _ptr(coeffs.view(np.float64), ctypes.c_double),
            TCP_STORAGE_EAGER if storage == "eager" else TCP_STORAGE_LAZY,
            min(int(max_bytes), U64_MAX),
            ctypes.byref(handle),
        )
        raise_for_status(status)
        self._handle = handle
        info = TcpPlanInfo()
        raise_for_status(lib.tcp_mvp_plan_info(handle, ctypes.byref(info)))
        self._info = info
        self.storage = storage

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        try:
            if handle is not None and handle.value:
                self._lib.tcp_mvp_plan_destroy(handle)
                self._handle = None
        except Exception:  # interpreter shutdown: the library may be gone already
            pass

    # -- metadata ---------------------------------------------------------
    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    @property
    def nqubits(self) -> int:
        return int(self._info.nqubits)

    @property
    def dimension(self) -> int:
        return int(self._info.dimension)

    @property
    def term_count(self) -> int:
        return int(self._info.term_count)

    @property
    def group_count(self) -> int:
        return int(self._info.group_count)

    @property
    def transition_count(self) -> Optional[int]:
        value = int(self._info.transition_count)
        return None if value < 0 else value

    @property
    def device(self) -> int:
        return int(self._info.device)

    @property
    def info(self) -> TcpPlanInfo:
        return self._info

    # -- host apply (drop-in for MvpPlan::apply / apply_into) ---------------
    def apply_into(self, state: np.ndarray, output: np.ndarray, max_bytes: int) -> None:
        """``NativeMvpPlan.apply_into`` (hamiltonian.rs:176-193): strict buffers."""
        for name, value in (("input", state), ("output", output)):
            if not isinstance(value, np.ndarray):
                raise TypeError("apply_into input and output must be NumPy arrays")
            if value.dtype != np.complex128:
                raise TypeError("apply_into input and output must have dtype complex128")
            if value.ndim != 1:
                raise ValueError(f"apply_into {name} must be one-dimensional")
            if not value.flags.c_contiguous:
                raise ValueError(f"apply_into {name} must be C-contiguous")
        if not output.flags.writeable:
            raise ValueError("apply_into output must be writable")
        status = self._lib.tcp_mvp_apply_into_host(
            self._handle,
            _ptr(state.view(np.float64), ctypes.c_double),
            state.shape[0],
            _ptr(output.view(np.float64), ctypes.c_double),
            output.shape[0],
            min(int(max_bytes), U64_MAX),
        )
        raise_for_status(status)

    def apply(self, state: np.ndarray, max_bytes: int) -> np.ndarray:
        """``NativeMvpPlan.apply`` (hamiltonian.rs:160-174): owned complex128 output."""
        values = np.ascontiguousarray(state, dtype=np.complex128)
        if values.ndim != 1:
            raise ValueError(f"state must be one-dimensional, got shape {values.shape}")
        if values.shape[0] != self.dimension:
            raise ValueError(
                f"expected structure length {self.dimension}, got {values.shape[0]}"
            )
        out = np.empty(self.dimension, dtype=np.complex128)
        self.apply_into(values, out, max_bytes)
        return out

    def apply_c64(self, state: np.ndarray) -> np.ndarray:
        """Host complex64 apply (FP32 products, Kahan-compensated group sums)."""
        values = np.ascontiguousarray(state, dtype=np.complex64)
        out = np.empty(values.shape[0], dtype=np.complex64)
        self.apply_c64_into(values, out)
        return out

    def apply_c64_into(self, state: np.ndarray, output: np.ndarray) -> None:
        """complex64 host buffers, overwritten output (strict, like apply_into)."""
        for value in (state, output):
            if not isinstance(value, np.ndarray) or value.dtype != np.complex64:
                raise TypeError("apply_c64_into input and output must be complex64 NumPy arrays")
            if value.ndim != 1 or not value.flags.c_contiguous:
                raise ValueError("apply_c64_into buffers must be one-dimensional and C-contiguous")
        status = self._lib.tcp_mvp_apply_into_host_c64(
            self._handle,
            _ptr(state.view(np.float32), ctypes.c_float),
            state.shape[0],
            _ptr(output.view(np.float32), ctypes.c_float),
            output.shape[0],
        )
        raise_for_status(status)

    # -- device apply -----------------------------------------------------
    def apply_device(self, x: Any, y: Any, stream: Any = None, accumulate: bool = False) -> None:
        """Apply to torch CUDA tensors of shape (dim,) or (nrhs, dim).

        complex128 tensors run the FP64 kernel, complex64 tensors the FP32
        Kahan kernel.  Asynchronous on ``stream`` (default: torch's current
        stream on the plan's device).  ``accumulate`` adds H x to y
        (``tcp_mvp_apply_add_device``) instead of overwriting it.
        """
        import torch

        if not (isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor)):
            raise TypeError("apply_device needs torch tensors")
        if x.device.type != "cuda" or y.device.type != "cuda":
            raise ValueError("apply_device needs CUDA tensors")
        if x.dtype != y.dtype or x.dtype not in (torch.complex128, torch.complex64):
            raise TypeError("apply_device tensors must both be complex128 or complex64")
        if x.shape != y.shape or x.ndim not in (1, 2) or x.shape[-1] != self.dimension:
            raise ValueError(f"apply_device tensors must have shape ({self.dimension},) or (nrhs, {self.dimension})")
        if not (x.is_contiguous() and y.is_contiguous()):
            raise ValueError("apply_device tensors must be contiguous")
        nrhs = 1 if x.ndim == 1 else int(x.shape[0])
        if stream is None:
            stream = torch.cuda.current_stream(x.device)
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        dtype = TCP_DTYPE_C128 if x.dtype == torch.complex128 else TCP_DTYPE_C64
        entry = self._lib.tcp_mvp_apply_add_device if accumulate else self._lib.tcp_mvp_apply_into_device
        status = entry(
            self._handle,
            ctypes.c_void_p(x.data_ptr()),
            ctypes.c_void_p(y.data_ptr()),
            self.dimension,
            nrhs,
            dtype,
            ctypes.c_void_p(handle),
        )
        raise_for_status(status)

    def diagonal_device(self, out: Any, stream: Any = None) -> None:
        """Write H_ii (complex128, the x_mask == 0 group) into a CUDA tensor."""
        import torch

        if out.dtype != torch.complex128 or out.shape != (self.dimension,) or not out.is_contiguous():
            raise ValueError("diagonal_device needs a contiguous complex128 tensor of length dim")
        if stream is None:
            stream = torch.cuda.current_stream(out.device)
        handle = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        raise_for_status(
            self._lib.tcp_mvp_diagonal_device(
                self._handle, ctypes.c_void_p(out.data_ptr()), self.dimension, ctypes.c_void_p(handle)
            )
        )

    def device_status(self) -> None:
        """Synchronise and raise if a kernel of this plan reported a device error."""
        raise_for_status(self._lib.tcp_mvp_plan_device_status(self._handle))

    # -- materialisation (include/tcp_matrix.h) ------------------------------
    def dense(self, max_bytes: int) -> np.ndarray:
        """Row-major complex128 dense matrix (``pauli_dense_handle``)."""
        dim = self.dimension
        if dim * dim * 16 > min(int(max_bytes), U64_MAX):
            raise MemoryError(f"requested {dim * dim * 16} bytes exceeds memory limit {max_bytes}")
        out = np.zeros((dim, dim), np.complex128)
        raise_for_status(
            self._lib.tcp_mvp_dense(self._handle, _ptr(out.view(np.float64), ctypes.c_double), dim * dim,
                                    min(int(max_bytes), U64_MAX))
        )
        return out

    def sparse(self, target: str, max_bytes: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(indptr, columns, values) with the budget of ``target`` ("coo" or "csr")."""
        code = TCP_MATRIX_COO if target == "coo" else TCP_MATRIX_CSR
        limit = min(int(max_bytes), U64_MAX)
        nnz = np.zeros(1, np.uint64)
        raise_for_status(self._lib.tcp_mvp_sparse_count(self._handle, code, limit, _ptr(nnz, ctypes.c_uint64)))
        m = int(nnz[0])
        indptr = np.zeros(self.dimension + 1, np.uint64)
        cols = np.zeros(max(m, 1), np.uint64)
        vals = np.zeros(max(m, 1), np.complex128)
        raise_for_status(
            self._lib.tcp_mvp_csr(self._handle, code, limit, _ptr(indptr, ctypes.c_uint64), _ptr(cols, ctypes.c_uint64),
                                  _ptr(vals.view(np.float64), ctypes.c_double), cols.shape[0],
                                  _ptr(nnz, ctypes.c_uint64))
        )
        m = int(nnz[0])
        return indptr, cols[:m], vals[:m]


# ----------------------------------------------------------------------------
# U(1) sector plans (include/tcp_sector.h)
# ----------------------------------------------------------------------------
def _terms_arrays(nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray):
    count = int(coefficients.shape[0])
    width = nqubits // 64 + (nqubits % 64 != 0)
    xw = np.ascontiguousarray(x_words, dtype=np.uint64).reshape(count * width)
    zw = np.ascontiguousarray(z_words, dtype=np.uint64).reshape(count * width)
    coeffs = np.ascontiguousarray(coefficients, dtype=np.complex128)
    if count == 0 or width == 0:  # keep valid pointers
        xw = np.zeros(max(count * width, 1), np.uint64)
        zw = np.zeros(max(count * width, 1), np.uint64)
    if count == 0:
        coeffs = np.zeros(1, np.complex128)
    return count, width, xw, zw, coeffs


def u1_dimension(nqubits: int, particle_number: int) -> int:
    out = np.zeros(1, np.uint64)
    raise_for_status(load_library().tcp_u1_dimension(nqubits, particle_number, _ptr(out, ctypes.c_uint64)))
    return int(out[0])


def u1_rank_words(nqubits: int, particle_number: int, words: np.ndarray) -> int:
    w = np.ascontiguousarray(words, dtype=np.uint64).reshape(-1)
    count = int(w.shape[0])
    buf = w if count else np.zeros(1, np.uint64)
    out = np.zeros(1, np.uint64)
    raise_for_status(
        load_library().tcp_u1_rank_words(
            nqubits, particle_number, _ptr(buf, ctypes.c_uint64), count, _ptr(out, ctypes.c_uint64)
        )
    )
    return int(out[0])


def u1_unrank_words(nqubits: int, particle_number: int, index: int) -> np.ndarray:
    width = nqubits // 64 + (nqubits % 64 != 0)
    out = np.zeros(max(width, 1), np.uint64)
    if index < 0 or index > U64_MAX:
        raise IndexError("restricted basis index is out of range")
    raise_for_status(
        load_library().tcp_u1_unrank_words(nqubits, particle_number, index, _ptr(out, ctypes.c_uint64), width)
    )
    return out[:width]


def u1_basis_words(nqubits: int, particle_number: int, max_bytes: int) -> Tuple[int, int, np.ndarray]:
    """``u1_basis_words`` (symmetry.rs:395-436): (dimension, word_count, flat words)."""
    dim = u1_dimension(nqubits, particle_number)
    width = 1 if nqubits <= 64 else nqubits // 64 + (nqubits % 64 != 0)
    if dim * width * 8 > max_bytes:
        raise MemoryError(f"requested {dim * width * 8} bytes exceeds memory limit {max_bytes}")
    out = np.zeros(max(dim * width, 1), np.uint64)
    raise_for_status(
        load_library().tcp_u1_basis_words(
            nqubits, particle_number, _ptr(out, ctypes.c_uint64), out.shape[0], min(int(max_bytes), U64_MAX)
        )
    )
    return dim, width, out[: dim * width]


def number_commutator(nqubits: int, x_words: np.ndarray, z_words: np.ndarray, coefficients: np.ndarray) -> int:
    """Nonzero words of [H, N] by the reference's selection rule (0: conserved)."""
    count, width, xw, zw, coeffs = _terms_arrays(nqubits, x_words, z_words, coefficients)
    out = np.zeros(1, np.uint64)
    raise_for_status(
        load_library().tcp_pauli_number_commutator(
            nqubits,
            count,
            width,
            _ptr(xw, ctypes.c_uint64),
            _ptr(zw, ctypes.c_uint64),
            _ptr(coeffs.view(np.float64), ctypes.c_double),
            _ptr(out, ctypes.c_uint64),
        )
    )
    return int(out[0])


def _stream_handle(stream: Any, device: Any) -> int:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(device)
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class NativeU1Plan:
    """Execution handle of one device sector plan (mirror of the PyO3
    ``NativeU1LazyMvpPlan`` / ``NativeU1RestrictedOperator``,
    ``crates/tencirpauli-native/src/symmetry.rs:122-368``)."""

    native_variant = "qubit"

    def __init__(
        self,
        nqubits: int,
        particle_number: int,
        x_words: np.ndarray,
        z_words: np.ndarray,
        coefficients: np.ndarray,
        storage: str = "lazy",
        max_bytes: int = sys.maxsize,
    ) -> None:
        lib = load_library()
        self._lib = lib
        self._handle = ctypes.c_void_p(None)
        if storage not in ("lazy", "eager"):
            raise ValueError("invalid sector: storage must be either 'eager' or 'lazy'")
        count, width, xw, zw, coeffs = _terms_arrays(nqubits, x_words, z_words, coefficients)
        handle = ctypes.c_void_p(None)
        status = lib.tcp_u1_plan_create(
            nqubits,
            particle_number,
            count,
            width,
            _ptr(xw, ctypes.c_uint64),
            _ptr(zw, ctypes.c_uint64),
            _ptr(coeffs.view(np.float64), ctypes.c_double),
            TCP_STORAGE_EAGER if storage == "eager" else TCP_STORAGE_LAZY,
            min(int(max_bytes), U64_MAX),
            ctypes.byref(handle),
        )
        raise_for_status(status)
        self._handle = handle
        info = TcpU1PlanInfo()
        raise_for_status(lib.tcp_u1_plan_info(handle, ctypes.byref(info)))
        self._info = info
        self.storage = storage

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        try:
            if handle is not None and handle.value:
                self._lib.tcp_u1_plan_destroy(handle)
                self._handle = None
        except Exception:  # interpreter shutdown
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._handle

    @property
    def info(self) -> TcpU1PlanInfo:
        return self._info

    @property
    def nqubits(self) -> int:
        return int(self._info.nqubits)

    @property
    def particle_number(self) -> int:
        return int(self._info.particle_number)

    @property
    def dimension(self) -> int:
        return int(self._info.dimension)

    @property
    def term_count(self) -> int:
        return int(self._info.term_count)

    @property
    def group_count(self) -> int:
        return int(self._info.group_count)

    @property
    def estimated_bytes(self) -> int:
        return int(self._info.estimated_bytes)

    @property
    def transition_count(self) -> Optional[int]:
        value = int(self._info.transition_count)
        return None if value < 0 else value

    def count_transitions(self) -> int:
        out = np.zeros(1, np.uint64)
        raise_for_status(self._lib.tcp_u1_transition_count(self._handle, _ptr(out, ctypes.c_uint64)))
        return int(out[0])

    def apply_into(self, state: np.ndarray, output: np.ndarray, max_bytes: int) -> None:
        for name, value in (("input", state), ("output", output)):
            if not isinstance(value, np.ndarray):
                raise TypeError("apply_into input and output must be NumPy arrays")
            if value.dtype != np.complex128:
                raise TypeError("apply_into input and output must have dtype complex128")
            if value.ndim != 1:
                raise ValueError(f"apply_into {name} must be one-dimensional")
            if not value.flags.c_contiguous:
                raise ValueError(f"apply_into {name} must be C-contiguous")
        if not output.flags.writeable:
            raise ValueError("apply_into output must be writable")
        status = self._lib.tcp_u1_apply_into_host(
            self._handle,
            _ptr(state.view(np.float64), ctypes.c_double),
            state.shape[0],
            _ptr(output.view(np.float64), ctypes.c_double),
            output.shape[0],
            min(int(max_bytes), U64_MAX),
        )
        raise_for_status(status)

    def apply(self, state: np.ndarray, max_bytes: int) -> np.ndarray:
        values = np.ascontiguousarray(state, dtype=np.complex128)
        if values.ndim != 1 or values.shape[0] != self.dimension:
            raise ValueError(f"expected structure length {self.dimension}, got {values.shape[0] if values.ndim else 0}")
        if self.dimension * 16 > max_bytes:
            raise MemoryError(f"requested {self.dimension * 16} bytes exceeds memory limit {max_bytes}")
        out = np.empty(self.dimension, dtype=np.complex128)
        self.apply_into(values, out, max_bytes)
        return out

    def apply_device(self, x: Any, y: Any, stream: Any = None) -> None:
        """Apply to torch CUDA tensors of shape (dim,) or (nrhs, dim)."""
        import torch

        if not (isinstance(x, torch.Tensor) and isinstance(y, torch.Tensor)):
            raise TypeError("apply_device needs torch tensors")
        if x.device.type != "cuda" or y.device.type != "cuda":
            raise ValueError("apply_device needs CUDA tensors")
        if x.dtype != y.dtype or x.dtype not in (torch.complex128, torch.complex64):
            raise TypeError("apply_device tensors must both be complex128 or complex64")
        if x.shape != y.shape or x.ndim not in (1, 2) or x.shape[-1] != self.dimension:
            raise ValueError(f"apply_device tensors must have shape ({self.dimension},) or (nrhs, {self.dimension})")
        if not (x.is_contiguous() and y.is_contiguous()):
            raise ValueError("apply_device tensors must be contiguous")
        nrhs = 1 if x.ndim == 1 else int(x.shape[0])
        dtype = TCP_DTYPE_C128 if x.dtype == torch.complex128 else TCP_DTYPE_C64
        status = self._lib.tcp_u1_apply_into_device(
            self._handle,
            ctypes.c_void_p(x.data_ptr()),
            ctypes.c_void_p(y.data_ptr()),
            self.dimension,
            nrhs,
            dtype,
            ctypes.c_void_p(_stream_handle(stream, x.device)),
        )
        raise_for_status(status)

    def diagonal_device(self, out: Any, stream: Any = None) -> None:
        import torch

        if out.dtype != torch.complex128 or out.shape != (self.dimension,) or not out.is_contiguous():
            raise ValueError("diagonal_device needs a contiguous complex128 tensor of length dim")
        raise_for_status(
            self._lib.tcp_u1_diagonal_device(
                self._handle,
                ctypes.c_void_p(out.data_ptr()),
                self.dimension,
                ctypes.c_void_p(_stream_handle(stream, out.device)),
            )
        )

    def csr(self, max_bytes: int) -> Tuple[int, np.ndarray, np.ndarray, np.ndarray]:
        """(dimension, indptr, columns, values): destinations as rows, columns ascending."""
        nnz = self.count_transitions()
        dim = self.dimension
        need = (dim + 1) * 8 + nnz * 24
        if need > max_bytes:
            raise MemoryError(f"requested {need} bytes exceeds memory limit {max_bytes}")
        indptr = np.zeros(dim + 1, np.uint64)
        cols = np.zeros(max(nnz, 1), np.uint64)
        vals = np.zeros(max(nnz, 1), np.complex128)
        got = np.zeros(1, np.uint64)
        raise_for_status(
            self._lib.tcp_u1_csr(
                self._handle,
                _ptr(indptr, ctypes.c_uint64),
                _ptr(cols, ctypes.c_uint64),
                _ptr(vals.view(np.float64), ctypes.c_double),
                cols.shape[0],
                _ptr(got, ctypes.c_uint64),
            )
        )
        m = int(got[0])
        return dim, indptr, cols[:m], vals[:m]

    def device_status(self) -> None:
        raise_for_status(self._lib.tcp_u1_plan_device_status(self._handle))


def probe_fma_rate(dtype: str = "complex128", repeats: int = 5) -> Tuple[float, float]:
    """(flop/s, best launch ms) of the device's FP64 (complex128) or FP32
    (complex64) FMA pipe, measured by ``tcp_probe_fma_rate``."""
    rate = np.zeros(1, np.float64)
    ms = np.zeros(1, np.float64)
    code = TCP_DTYPE_C128 if dtype in ("complex128", "c128") else TCP_DTYPE_C64
    raise_for_status(
        load_library().tcp_probe_fma_rate(code, repeats, _ptr(rate, ctypes.c_double), _ptr(ms, ctypes.c_double))
    )
    return float(rate[0]), float(ms[0])


def probe_smem_rate(repeats: int = 5) -> Tuple[float, float]:
    """(bytes/s, best launch ms) that the device's shared memory delivers to
    registers in the tiled kernels' access pattern (``tcp_probe_smem_rate``)."""
    rate = np.zeros(1, np.float64)
    ms = np.zeros(1, np.float64)
    raise_for_status(load_library().tcp_probe_smem_rate(repeats, _ptr(rate, ctypes.c_double), _ptr(ms, ctypes.c_double)))
    return float(rate[0]), float(ms[0])
