"""torch-facing wrappers of the eigensolver kernels (``include/tcp_solver.h``).

Vectors are RHS-major torch CUDA tensors of shape (k, n), complex64 or
complex128; small coefficient matrices are complex128 CUDA tensors.  Every
reduction and combination runs in FP64 on the device.
"""

from __future__ import annotations

import ctypes
from typing import Any, Tuple

from . import _native

TCP_FEATURES = 8
TCP_MLP_IN = 8
TCP_MLP_HIDDEN = 16
TCP_MLP_PARAMS = 433


def _lib():
    return _native.load_library()


def _dtype_code(t: Any) -> int:
    import torch

    if t.dtype == torch.complex128:
        return _native.TCP_DTYPE_C128
    if t.dtype == torch.complex64:
        return _native.TCP_DTYPE_C64
    raise TypeError("vectors must be complex64 or complex128")


def _stream(stream: Any = None) -> ctypes.c_void_p:
    import torch

    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _ptr(t: Any) -> ctypes.c_void_p:
    return ctypes.c_void_p(int(t.data_ptr()))


def _vectors(t: Any):
    if t.ndim != 2 or not t.is_contiguous() or t.device.type != "cuda":
        raise ValueError("vector blocks must be contiguous CUDA tensors of shape (k, n)")
    return t.shape[0], t.shape[1]


class Workspace:
    """Reusable device scratch for the Gram kernel."""

    def __init__(self) -> None:
        self._buf = None

    def get(self, nbytes: int):
        import torch

        if self._buf is None or self._buf.numel() < nbytes:
            self._buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device="cuda")
        return self._buf


_WS = Workspace()


def _gram_once(A: Any, B: Any, stream: Any) -> Any:
    import torch

    p, n = _vectors(A)
    q, _ = _vectors(B)
    out = torch.empty((q, p), dtype=torch.complex128, device=A.device)  # column-major p x q
    work = _WS.get(int(_lib().tcp_gram_work_bytes(p, q)))
    _native.raise_for_status(
        _lib().tcp_gram(_ptr(A), _dtype_code(A), p, _ptr(B), _dtype_code(B), q, n, _ptr(out), _ptr(work), _stream(stream))
    )
    return out.transpose(0, 1)


def gram(A: Any, B: Any, stream: Any = None) -> Any:
    """G = A^H B (p x q, complex128) accumulated in FP64.  Blocks larger than
    one kernel launch takes (p + q <= 96, p * q <= 512) are split."""
    import torch

    p, n = _vectors(A)
    q, n2 = _vectors(B)
    if n != n2:
        raise ValueError("vector lengths differ")
    if p + q <= 96 and p * q <= 512:
        return _gram_once(A, B, stream)
    G = torch.empty((p, q), dtype=torch.complex128, device=A.device)
    pa = min(p, 64)
    qb = max(1, min(q, 512 // pa, 96 - pa))
    for i in range(0, p, pa):
        for j in range(0, q, qb):
            G[i : i + pa, j : j + qb] = _gram_once(A[i : i + pa], B[j : j + qb], stream)
    return G


def combine(A: Any, S: Any, out: Any, alpha: float = 1.0, beta: float = 0.0, stream: Any = None) -> Any:
    """out[j] = alpha * sum_i A[i] S[i, j] + beta * out[j] (FP64 arithmetic);
    the outputs go 32 at a time (fewer when p is so large that p x 32
    coefficients do not fit one launch's shared-memory block)."""
    import torch

    p, n = _vectors(A)
    k, n2 = _vectors(out)
    if n != n2 or tuple(S.shape) != (p, k):
        raise ValueError("shape mismatch in combine")
    step = 32
    while step > 4 and p * step > 6144:
        step //= 2
    for j0 in range(0, k, step):
        j1 = min(k, j0 + step)
        Sc = S[:, j0:j1].to(device=A.device, dtype=torch.complex128).transpose(0, 1).contiguous()  # column-major
        o = out[j0:j1]
        _native.raise_for_status(
            _lib().tcp_block_combine(
                _ptr(A), _dtype_code(A), p, _ptr(Sc), j1 - j0, n, alpha, beta, _ptr(o), _dtype_code(o), _stream(stream)
            )
        )
    return out


def jacobi(R: Any, diag: Any, theta: Any, out: Any, eps: float = 1e-8, stream: Any = None) -> Any:
    k, n = _vectors(R)
    th = theta.to(device=R.device, dtype=__import__("torch").float64).contiguous()
    _native.raise_for_status(
        _lib().tcp_precond_jacobi(_ptr(R), _dtype_code(R), n, k, _ptr(diag), _ptr(th), eps, _ptr(out), _dtype_code(out), _stream(stream))
    )
    return out


def state_features(plan: Any, out: Any = None, stream: Any = None) -> Any:
    import torch

    execution = getattr(plan, "_native_plan", plan)
    n = execution.dimension
    if out is None:
        out = torch.empty((n, TCP_FEATURES), dtype=torch.float32, device="cuda")
    _native.raise_for_status(_lib().tcp_state_features(execution.handle, _ptr(out), n, _stream(stream)))
    return out


def mlp_precondition(
    R: Any, features: Any, diag: Any, theta: Any, params: Any, scale: float, out: Any, eps: float = 1e-8, clamp: float = 4.0,
    stream: Any = None,
) -> Any:
    import torch

    k, n = _vectors(R)
    th = theta.to(device=R.device, dtype=torch.float64).contiguous()
    _native.raise_for_status(
        _lib().tcp_precond_mlp(
            _ptr(R), _dtype_code(R), n, k, _ptr(features), _ptr(diag), _ptr(th), scale, eps, clamp, _ptr(params), _ptr(out),
            _dtype_code(out), _stream(stream),
        )
    )
    return out


def mlp_inputs(features: Any, rows: Any, theta: Any, which: Any, scale: float, eps: float = 1e-8, stream: Any = None):
    import torch

    count = int(rows.numel())
    X = torch.empty((count, TCP_MLP_IN), dtype=torch.float32, device="cuda")
    den = torch.empty(count, dtype=torch.float32, device="cuda")
    th = theta.to(device="cuda", dtype=torch.float64).contiguous()
    _native.raise_for_status(
        _lib().tcp_mlp_inputs(_ptr(features), _ptr(rows), _ptr(th), _ptr(which), count, scale, eps, _ptr(X), _ptr(den), _stream(stream))
    )
    return X, den


def mlp_forward(X: Any, params: Any, out: Any = None, stream: Any = None) -> Any:
    import torch

    count = int(X.shape[0])
    if out is None:
        out = torch.empty(count, dtype=torch.float32, device="cuda")
    _native.raise_for_status(_lib().tcp_mlp_forward(_ptr(X), count, _ptr(params), _ptr(out), _stream(stream)))
    return out


def alignment_grad(c: Any, den: Any, alpha: Any, a: Any, gamma: Any, E: Any, seg: Any, seg_begin: Any, clamp: float,
                   work: Any = None, dc: Any = None, stream: Any = None) -> Tuple[float, Any]:
    """(objective, dL/dc) of the alignment objective (tcp_mlp_alignment_grad):
    float32 c and den, complex128 alpha and gamma, float64 a per state; float64
    E per set; int64 set index per state and int64 set offsets (nsets + 1)."""
    import torch

    nsets = int(E.shape[0])
    count = int(c.shape[0])
    for t, dt in ((c, torch.float32), (den, torch.float32), (alpha, torch.complex128), (a, torch.float64),
                  (gamma, torch.complex128), (E, torch.float64), (seg, torch.int64), (seg_begin, torch.int64)):
        if t.dtype != dt or not t.is_contiguous() or t.device.type != "cuda":
            raise ValueError("alignment inputs must be contiguous CUDA tensors of the documented dtypes")
    if seg_begin.shape[0] != nsets + 1 or any(int(t.shape[0]) != count for t in (den, alpha, a, gamma, seg)):
        raise ValueError("alignment inputs have inconsistent lengths")
    if work is None or work.numel() * 8 < int(_lib().tcp_mlp_alignment_work_bytes(nsets)):
        work = torch.empty(int(_lib().tcp_mlp_alignment_work_bytes(nsets)) // 8, dtype=torch.float64, device="cuda")
    if dc is None:
        dc = torch.empty(count, dtype=torch.float32, device="cuda")
    loss = torch.empty(1, dtype=torch.float64, device="cuda")
    _native.raise_for_status(
        _lib().tcp_mlp_alignment_grad(
            _ptr(c), _ptr(den), _ptr(alpha), _ptr(a), _ptr(gamma), _ptr(E), _ptr(seg), _ptr(seg_begin), nsets, count,
            float(clamp), _ptr(work), _ptr(dc), _ptr(loss), _stream(stream),
        )
    )
    return float(loss.item()), dc


class MLPTrainer:
    """Device training state (parameters, Adam moments, scratch)."""

    def __init__(self, params: Any) -> None:
        import torch

        self.params = params
        self.m = torch.zeros_like(params)
        self.v = torch.zeros_like(params)
        self.work = torch.empty(int(_lib().tcp_mlp_train_work_bytes()) // 4, dtype=torch.float32, device="cuda")
        self.grad = torch.empty_like(params)
        self.loss = torch.empty(1, dtype=torch.float32, device="cuda")
        self.step_count = 0

    def backward_step(self, X, dc, lr: float, stream: Any = None) -> None:
        """Weight gradient from given dL/dc per sample; Adam step when lr > 0."""
        if lr > 0:
            self.step_count += 1
        _native.raise_for_status(
            _lib().tcp_mlp_backward_step(
                _ptr(X), _ptr(dc), int(X.shape[0]), _ptr(self.params), _ptr(self.m), _ptr(self.v), _ptr(self.work), lr,
                max(self.step_count, 1), _ptr(self.grad), _stream(stream),
            )
        )

    def step(self, X, den, a, b, e2, wt, lr: float, stream: Any = None) -> None:
        if lr > 0:
            self.step_count += 1
        _native.raise_for_status(
            _lib().tcp_mlp_train_step(
                _ptr(X), _ptr(den), _ptr(a), _ptr(b), _ptr(e2), _ptr(wt), int(X.shape[0]), _ptr(self.params), _ptr(self.m),
                _ptr(self.v), _ptr(self.work), lr, max(self.step_count, 1), _ptr(self.grad), _ptr(self.loss), _stream(stream),
            )
        )
