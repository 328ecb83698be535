"""Batched MVP over many Hamiltonians and right-hand-side blocks.

``BatchedMVP(plans, nrhs, dtype)`` applies every plan to its own block of
``nrhs`` state vectors, replayed from one CUDA graph (``tcp_mvp_batch_*`` in
``include/tcp_mvp.h``): either one persistent kernel launch over (member,
tile, RHS block) work items, or -- the ring configuration (12, 1), the
default when every member has at least 12 qubits -- one ring-kernel launch
per member over all its tiles and right-hand sides.  ``autotune`` times the
configurations (tile rows x RHS block, and the ring one) on the caller's
buffers and keeps the fastest, caching the choice on disk.
"""

from __future__ import annotations

import ctypes
import os
from typing import Any, Dict, List, Optional, Sequence

from . import _native

DEFAULT_CACHE = os.path.join(os.path.expanduser("~"), ".cache", "tencirpauli_b200", "batch_autotune.txt")


class BatchedMVP:
    def __init__(self, plans: Sequence[Any], nrhs: int, dtype: str = "complex64") -> None:
        if dtype not in ("complex64", "complex128"):
            raise ValueError("dtype must be 'complex64' or 'complex128'")
        self._lib = _native.load_library()
        self._plans = [getattr(p, "_native_plan", p) for p in plans]  # keep the plans alive
        self.nrhs = int(nrhs)
        self.dtype = dtype
        handles = (ctypes.c_void_p * len(self._plans))(*[p.handle.value for p in self._plans])
        out = ctypes.c_void_p(None)
        code = _native.TCP_DTYPE_C64 if dtype == "complex64" else _native.TCP_DTYPE_C128
        _native.raise_for_status(self._lib.tcp_mvp_batch_create(len(self._plans), handles, self.nrhs, code, ctypes.byref(out)))
        self._handle = out

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        try:
            if handle is not None and handle.value:
                self._lib.tcp_mvp_batch_destroy(handle)
                self._handle = None
        except Exception:  # interpreter shutdown
            pass

    @staticmethod
    def _tables(xs: Sequence[Any], ys: Sequence[Any]):
        n = len(xs)
        if len(ys) != n:
            raise ValueError("xs and ys must have one entry per plan")
        xt = (ctypes.c_void_p * n)(*[int(x.data_ptr()) for x in xs])
        yt = (ctypes.c_void_p * n)(*[int(y.data_ptr()) for y in ys])
        return xt, yt

    def _check(self, xs: Sequence[Any], ys: Sequence[Any]) -> None:
        import torch

        want = torch.complex64 if self.dtype == "complex64" else torch.complex128
        if len(xs) != len(self._plans) or len(ys) != len(self._plans):
            raise ValueError("one input and one output block per plan")
        for plan, x, y in zip(self._plans, xs, ys):
            shape = (self.nrhs, plan.dimension)
            for t in (x, y):
                if t.dtype != want or tuple(t.shape) != shape or not t.is_contiguous() or t.device.type != "cuda":
                    raise ValueError(f"batch buffers must be contiguous CUDA {want} tensors of shape {shape}")

    @staticmethod
    def _stream(stream: Any) -> int:
        import torch

        if stream is None:
            stream = torch.cuda.current_stream()
        return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)

    def apply(self, xs: Sequence[Any], ys: Sequence[Any], stream: Any = None) -> None:
        self._check(xs, ys)
        xt, yt = self._tables(xs, ys)
        _native.raise_for_status(self._lib.tcp_mvp_batch_apply(self._handle, xt, yt, ctypes.c_void_p(self._stream(stream))))

    def configure(self, tile_rows_log2: int, rhs_block: int) -> None:
        _native.raise_for_status(self._lib.tcp_mvp_batch_configure(self._handle, tile_rows_log2, rhs_block))

    def autotune(
        self, xs: Sequence[Any], ys: Sequence[Any], cache_path: Optional[str] = DEFAULT_CACHE, repeats: int = 3, stream: Any = None
    ) -> Dict[str, int]:
        self._check(xs, ys)
        if cache_path:
            os.makedirs(os.path.dirname(cache_path), exist_ok=True)
        xt, yt = self._tables(xs, ys)
        path = cache_path.encode() if cache_path else None
        _native.raise_for_status(
            self._lib.tcp_mvp_batch_autotune(self._handle, xt, yt, path, repeats, ctypes.c_void_p(self._stream(stream)))
        )
        return self.info()

    def info(self) -> Dict[str, int]:
        logt, rb, grid = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        items = ctypes.c_uint64()
        _native.raise_for_status(
            self._lib.tcp_mvp_batch_info(self._handle, ctypes.byref(logt), ctypes.byref(rb), ctypes.byref(items), ctypes.byref(grid))
        )
        return {"tile_rows_log2": logt.value, "rhs_block": rb.value, "items": items.value, "grid": grid.value}

    def device_status(self) -> None:
        _native.raise_for_status(self._lib.tcp_mvp_batch_device_status(self._handle))

    @property
    def plans(self) -> List[Any]:
        return list(self._plans)
