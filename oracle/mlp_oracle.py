"""NumPy restatement of the learned-preconditioner math -- TEST INFRASTRUCTURE ONLY.

Checks the device kernels of ``include/tcp_solver.h``: the per-basis-state
features (``tcp_state_features``), the network inputs (``tcp_mlp_inputs``),
the MLP forward pass and correction (``tcp_precond_mlp``), the training loss
and its gradient (``tcp_mlp_train_step``), and the Jacobi correction.  The
reference project has no eigensolver or preconditioner (it hands its MVP
plan to SciPy's ``eigsh``), so these restate the build's own definitions.
Only the test-suite imports this module.
"""

from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

IN = 8
HID = 16
FEATURES = 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID
NPARAM = OFF_B3 + 1


def unpack(p: np.ndarray) -> Dict[str, np.ndarray]:
    p = np.asarray(p, dtype=np.float64)
    return {
        "W1": p[OFF_W1:OFF_B1].reshape(HID, IN),
        "b1": p[OFF_B1:OFF_W2],
        "W2": p[OFF_W2:OFF_B2].reshape(HID, HID),
        "b2": p[OFF_B2:OFF_W3],
        "w3": p[OFF_W3:OFF_B3],
        "b3": p[OFF_B3],
    }


def pack(d: Dict[str, np.ndarray]) -> np.ndarray:
    return np.concatenate([d["W1"].ravel(), d["b1"], d["W2"].ravel(), d["b2"], d["w3"], np.atleast_1d(d["b3"])])


def forward(p: np.ndarray, X: np.ndarray) -> Tuple[np.ndarray, Dict[str, np.ndarray]]:
    """c = w3 . tanh(W2 tanh(W1 x + b1) + b2) + b3 for every row of X."""
    w = unpack(p)
    h1 = np.tanh(X @ w["W1"].T + w["b1"])
    h2 = np.tanh(h1 @ w["W2"].T + w["b2"])
    c = h2 @ w["w3"] + w["b3"]
    return c, {"h1": h1, "h2": h2}


def loss_and_grad(p, X, den, a, b, e2, wt) -> Tuple[float, np.ndarray]:
    """Loss sum wt (g^2 a - 2 g b + e2) with g = -exp(c)/den, and its gradient."""
    w = unpack(p)
    c, act = forward(p, X)
    h1, h2 = act["h1"], act["h2"]
    g = -np.exp(c) / den
    loss = float(np.sum(wt * (g * g * a - 2 * g * b + e2)))
    dc = wt * (2 * g * a - 2 * b) * g
    grads = {}
    grads["w3"] = h2.T @ dc
    grads["b3"] = np.array([dc.sum()])
    dh2 = dc[:, None] * w["w3"][None, :] * (1 - h2 * h2)
    grads["W2"] = dh2.T @ h1
    grads["b2"] = dh2.sum(0)
    dh1 = (dh2 @ w["W2"]) * (1 - h1 * h1)
    grads["W1"] = dh1.T @ X
    grads["b1"] = dh1.sum(0)
    return loss, pack(grads)


def finite_difference_grad(p, X, den, a, b, e2, wt, h: float = 1e-6) -> np.ndarray:
    p = np.asarray(p, dtype=np.float64)
    out = np.zeros_like(p)
    for i in range(p.size):
        q = p.copy()
        q[i] += h
        lp, _ = loss_and_grad(q, X, den, a, b, e2, wt)
        q[i] -= 2 * h
        lm, _ = loss_and_grad(q, X, den, a, b, e2, wt)
        out[i] = (lp - lm) / (2 * h)
    return out


def state_features(nqubits: int, x_mask, z_mask, weighted) -> np.ndarray:
    """Per-basis-state features (TCP_FEATURES floats) from compiled terms."""
    dim = 1 << nqubits
    rows = np.arange(dim, dtype=np.uint64)
    masks = np.unique(x_mask)

    def group_diag(mask, cols):
        sel = x_mask == mask
        total = np.zeros(cols.shape, dtype=np.complex128)
        for z, wgt in zip(z_mask[sel], weighted[sel]):
            par = np.bitwise_count(np.bitwise_and(cols, np.uint64(z))) & 1
            total += np.where(par == 1, -wgt, wgt)
        return total

    hii = group_diag(0, rows).real if 0 in masks else np.zeros(dim)
    sum_abs = np.zeros(dim)
    sum_sq = np.zeros(dim)
    sum_nd = np.zeros(dim)
    min_nd = np.full(dim, np.inf)
    count = np.zeros(dim)
    for mask in masks:
        if mask == 0:
            continue
        cols = rows ^ np.uint64(mask)
        d = group_diag(mask, cols)
        a2 = np.abs(d) ** 2
        nz = a2 != 0
        dj = hii[cols.astype(np.int64)]
        sum_abs += np.where(nz, np.sqrt(a2), 0)
        sum_sq += np.where(nz, a2, 0)
        sum_nd += np.where(nz, dj, 0)
        min_nd = np.where(nz, np.minimum(min_nd, dj), min_nd)
        count += nz
    f = np.zeros((dim, FEATURES))
    f[:, 0] = hii
    f[:, 1] = np.where(count > 0, sum_nd / np.maximum(count, 1), hii)
    f[:, 2] = np.where(count > 0, min_nd, hii)
    f[:, 3] = sum_abs
    f[:, 4] = sum_sq
    f[:, 5] = count
    f[:, 6] = np.bitwise_count(rows) / max(1, nqubits) - 0.5
    return f


def inputs(features: np.ndarray, theta: float, scale: float, eps: float = 1e-8) -> Tuple[np.ndarray, np.ndarray]:
    f = np.asarray(features, dtype=np.float64)
    d = f[:, 0] - theta
    den = np.where(np.abs(d) < eps, np.where(d < 0, -eps, eps), d)
    x = np.zeros((f.shape[0], IN))
    x[:, 0] = d / scale
    x[:, 1] = (f[:, 1] - theta) / scale
    x[:, 2] = (f[:, 2] - theta) / scale
    x[:, 3] = f[:, 3] / scale
    x[:, 4] = f[:, 4] / scale / scale
    x[:, 5] = f[:, 5] * 0.05
    x[:, 6] = f[:, 6]
    ratio = f[:, 4] / (np.abs(den) * np.maximum(np.abs(f[:, 1] - theta), eps))
    x[:, 7] = ratio / (1 + ratio)
    return x, den


def mlp_correction(p, features, r: np.ndarray, theta: float, scale: float, clamp: float = 4.0) -> np.ndarray:
    x, den = inputs(features, theta, scale)
    c, _ = forward(p, x)
    c = np.clip(c, -clamp, clamp)
    return -np.exp(c) * r / den


def jacobi(diag: np.ndarray, r: np.ndarray, theta: float, eps: float = 1e-8) -> np.ndarray:
    d = diag.real - theta
    den = np.where(np.abs(d) < eps, np.where(d < 0, -eps, eps), d)
    return -r / den


def alignment_loss(c, den, alpha, a, gamma, E, seg, nsets: int, clamp: float = 4.0) -> float:
    """Alignment objective of the preconditioner's training: the mean over
    training sets of 1 - |A|^2 / (E (B - |C|^2)) with g = -exp(clip(c)) / den,
    A = sum g alpha, B = sum g^2 a, C = sum g gamma over the set's states."""
    g = -np.exp(np.clip(np.asarray(c, np.float64), -clamp, clamp)) / np.asarray(den, np.float64)
    A = np.zeros(nsets, np.complex128)
    B = np.zeros(nsets)
    C = np.zeros(nsets, np.complex128)
    np.add.at(A, seg, g * alpha)
    np.add.at(B, seg, g * g * a)
    np.add.at(C, seg, g * gamma)
    D = np.maximum(B - np.abs(C) ** 2, 1e-300)
    return float(np.mean(1.0 - np.abs(A) ** 2 / (E * D)))


def alignment_loss_and_dc(c, den, alpha, a, gamma, E, seg, nsets: int, clamp: float = 4.0) -> Tuple[float, np.ndarray]:
    """The objective and its derivative with respect to each network output
    (zero where the clip is active), by the chain rule through g."""
    c = np.asarray(c, np.float64)
    g = -np.exp(np.clip(c, -clamp, clamp)) / np.asarray(den, np.float64)
    A = np.zeros(nsets, np.complex128)
    B = np.zeros(nsets)
    C = np.zeros(nsets, np.complex128)
    np.add.at(A, seg, g * alpha)
    np.add.at(B, seg, g * g * a)
    np.add.at(C, seg, g * gamma)
    D = np.maximum(B - np.abs(C) ** 2, 1e-300)
    A2 = np.abs(A) ** 2
    loss = float(np.mean(1.0 - A2 / (E * D)))
    dA2 = 2.0 * np.real(np.conj(A[seg]) * alpha)
    dD = 2.0 * g * a - 2.0 * np.real(np.conj(C[seg]) * gamma)
    dLdg = -(dA2 * D[seg] - A2[seg] * dD) / (E[seg] * D[seg] ** 2) / nsets
    inside = (c > -clamp) & (c < clamp)
    return loss, np.where(inside, dLdg * g, 0.0)
