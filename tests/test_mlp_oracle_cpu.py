"""CPU checks of the learned-preconditioner oracle (test infrastructure):
its analytic gradient against central finite differences, and the
zero-output network reducing to the Jacobi correction."""

from __future__ import annotations

import numpy as np

from oracle import mlp_oracle as mo
from tencirpauli_b200 import precond


def _data(seed: int = 0, count: int = 64):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(count, mo.IN))
    den = rng.uniform(0.5, 3.0, size=count) * rng.choice([-1, 1], size=count)
    r = rng.normal(size=count) + 1j * rng.normal(size=count)
    e = rng.normal(size=count) + 1j * rng.normal(size=count)
    a = np.abs(r) ** 2
    b = (np.conj(e) * r).real
    e2 = np.abs(e) ** 2
    wt = np.full(count, 1.0 / e2.sum())
    return X, den, a, b, e2, wt


def test_analytic_gradient_matches_finite_differences() -> None:
    X, den, a, b, e2, wt = _data()
    p = np.random.default_rng(3).normal(scale=0.3, size=mo.NPARAM)
    loss, grad = mo.loss_and_grad(p, X, den, a, b, e2, wt)
    fd = mo.finite_difference_grad(p, X, den, a, b, e2, wt)
    np.testing.assert_allclose(grad, fd, rtol=1e-5, atol=1e-7)
    assert loss > 0


def test_initial_network_is_jacobi() -> None:
    p = precond.init_params(0)
    assert p.size == mo.NPARAM
    rng = np.random.default_rng(1)
    feats = rng.normal(size=(32, mo.FEATURES))
    feats[:, 0] = rng.uniform(2, 5, size=32)
    r = rng.normal(size=32) + 1j * rng.normal(size=32)
    t = mo.mlp_correction(p, feats, r, theta=-1.0, scale=1.0)
    diag = feats[:, 0].astype(np.complex128)
    np.testing.assert_allclose(t, mo.jacobi(diag, r, -1.0), rtol=1e-12)


def test_pack_roundtrip_and_sizes() -> None:
    p = np.arange(mo.NPARAM, dtype=np.float64)
    np.testing.assert_array_equal(mo.pack(mo.unpack(p)), p)
    assert mo.NPARAM == 433


def alignment_data(seed: int = 0, sizes=(40, 25, 57)):
    """Random alignment-objective sets: contiguous states per set."""
    rng = np.random.default_rng(seed)
    count = sum(sizes)
    seg = np.repeat(np.arange(len(sizes)), sizes)
    c = rng.normal(scale=0.8, size=count)
    c[::17] = 5.0  # some outputs beyond the clamp
    den = rng.uniform(0.5, 3.0, size=count) * rng.choice([-1, 1], size=count)
    r = rng.normal(size=count) + 1j * rng.normal(size=count)
    u = rng.normal(size=count) + 1j * rng.normal(size=count)
    e = rng.normal(size=count) + 1j * rng.normal(size=count)
    for s in range(len(sizes)):  # per set: u a unit vector, e orthogonal to it
        m = seg == s
        u[m] /= np.linalg.norm(u[m])
        e[m] -= u[m] * np.vdot(u[m], e[m])
    E = np.zeros(len(sizes))
    np.add.at(E, seg, np.abs(e) ** 2)
    return c, den, np.conj(e) * r, np.abs(r) ** 2, np.conj(u) * r, E, seg, len(sizes)


def test_alignment_derivative_matches_finite_differences() -> None:
    c, den, alpha, a, gamma, E, seg, S = alignment_data()
    loss, dc = mo.alignment_loss_and_dc(c, den, alpha, a, gamma, E, seg, S)
    assert 0.0 < loss < 1.0
    h = 1e-6
    for i in range(0, c.size, 7):
        cp, cm = c.copy(), c.copy()
        cp[i] += h
        cm[i] -= h
        fd = (mo.alignment_loss(cp, den, alpha, a, gamma, E, seg, S) - mo.alignment_loss(cm, den, alpha, a, gamma, E, seg, S)) / (2 * h)
        assert abs(dc[i] - fd) <= 1e-6 * max(1.0, abs(fd)), (i, dc[i], fd)
    # outputs beyond the clamp get no gradient
    assert np.all(dc[c >= 4.0] == 0.0)
