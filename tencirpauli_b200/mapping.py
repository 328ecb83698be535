"""Jordan-Wigner mapping of fermionic integrals to Pauli terms (host side).

Restates the reference's Jordan-Wigner convention
(``crates/tencir-pauli-core/src/structured/fermion.rs:245-283``): mode p is
qubit p, ``a_p = (X_p + i Y_p)/2`` and ``a†_p = (X_p - i Y_p)/2`` with Z on
every mode below p; and the integral convention of
``python/tencirpauli/_structured/fermion.py:154-156``:
``H = sum_pq h_pq a†_p a_q + 1/2 sum_pqrs g_pqrs a†_p a†_q a_s a_r``.

The products are vectorised over all integral entries in the symplectic
form X^x Z^z (per qubit X first, then Z): (X^a Z^b)(X^c Z^d) =
(-1)^{popcount(b & c)} X^{a^c} Z^{b^d}, and X^x Z^z = (-i)^{popcount(x & z)}
P(x, z) with P the Hermitian word (Y = i X Z).  Duplicate words are merged
and exact zeros dropped by the library's canonicalization
(``tcp_pauli_canonicalize``).  Supports up to 64 modes.
"""

from __future__ import annotations

from typing import Tuple

import numpy as np

_PHASE = np.array([1.0, -1.0j, -1.0, 1.0j], dtype=np.complex128)  # (-i)^k


def _ladder(n: int, mode: np.ndarray, creation: bool):
    """The two symplectic terms of a†_p (creation) or a_p for an array of modes."""
    mode = mode.astype(np.uint64)
    below = (np.uint64(1) << mode) - np.uint64(1)  # Z on modes < p
    bit = np.uint64(1) << mode
    x = np.stack([bit, bit])
    z = np.stack([below, below | bit])
    # a† = X/2 + (X Z)/2 ;  a = X/2 - (X Z)/2   (since -iY = XZ and iY = -XZ)
    c = np.array([0.5, 0.5 if creation else -0.5], dtype=np.complex128)
    return x, z, c


def _multiply(xa, za, ca, xb, zb, cb):
    """All pairwise products (outer over the term axis 0) of two symplectic
    term sets, vectorised over the trailing entry axis."""
    x = (xa[:, None] ^ xb[None, :]).reshape(-1, xa.shape[-1])
    z = (za[:, None] ^ zb[None, :]).reshape(-1, xa.shape[-1])
    anti = np.bitwise_count(za[:, None] & xb[None, :]) & 1
    sign = np.where(anti == 1, -1.0, 1.0)
    c = (ca[:, None, :] * cb[None, :, :] * sign).reshape(-1, xa.shape[-1])
    return x, z, c


def _to_codes(n: int, x: np.ndarray, z: np.ndarray) -> np.ndarray:
    codes = np.zeros((x.shape[0], n), dtype=np.uint8)
    for q in range(n):
        xb = (x >> np.uint64(q)) & np.uint64(1)
        zb = (z >> np.uint64(q)) & np.uint64(1)
        codes[:, q] = np.where(xb == 1, np.where(zb == 1, 2, 1), np.where(zb == 1, 3, 0))
    return codes


def jordan_wigner_integrals(
    h: np.ndarray, g: np.ndarray, tol: float = 0.0, constant: complex = 0.0
) -> Tuple[np.ndarray, np.ndarray]:
    """Pauli code rows and coefficients (not yet canonical) of
    constant + sum h_pq a†_p a_q + 1/2 sum g_pqrs a†_p a†_q a_s a_r (the
    constant is the identity word, as the reference keeps the nuclear
    constant of ``FermionOperator.from_integrals``)."""
    n = h.shape[0]
    if n > 64:
        raise ValueError("at most 64 modes")
    words_x, words_z, coeffs = [], [], []
    if constant != 0:
        words_x.append(np.zeros(1, dtype=np.uint64))
        words_z.append(np.zeros(1, dtype=np.uint64))
        coeffs.append(np.asarray([constant], dtype=np.complex128))
    # one-body
    p, q = np.nonzero(np.abs(h) > tol)
    if p.size:
        xa, za, ca = _ladder(n, p, True)
        xb, zb, cb = _ladder(n, q, False)
        x, z, c = _multiply(xa, za, ca[:, None] * np.ones(p.size), xb, zb, cb[:, None] * np.ones(q.size))
        c = c * h[p, q][None, :]
        words_x.append(x.ravel())
        words_z.append(z.ravel())
        coeffs.append(c.ravel())
    # two-body: a†_p a†_q a_s a_r, skipping p == q or r == s (zero operators)
    idx = np.argwhere(np.abs(g) > tol)
    idx = idx[(idx[:, 0] != idx[:, 1]) & (idx[:, 2] != idx[:, 3])]
    for chunk in np.array_split(idx, max(1, idx.shape[0] // 200000 + 1)):
        if chunk.size == 0:
            continue
        P, Q, R, S = chunk.T
        x, z, c = _ladder(n, P, True)
        c = c[:, None] * np.ones(P.size)
        for mode, creation in ((Q, True), (S, False), (R, False)):
            xb, zb, cb = _ladder(n, mode, creation)
            x, z, c = _multiply(x, z, c, xb, zb, cb[:, None] * np.ones(mode.size))
        c = c * (0.5 * g[P, Q, R, S])[None, :]
        words_x.append(x.ravel())
        words_z.append(z.ravel())
        coeffs.append(c.ravel())
    if not coeffs:
        return np.zeros((0, n), dtype=np.uint8), np.zeros(0, dtype=np.complex128)
    X = np.concatenate(words_x)
    Z = np.concatenate(words_z)
    C = np.concatenate(coeffs)
    keep = C != 0
    X, Z, C = X[keep], Z[keep], C[keep]
    C = C * _PHASE[np.bitwise_count(X & Z) % 4]  # X^x Z^z -> Hermitian word
    return _to_codes(n, X, Z), C


def chemistry_integrals(n: int = 28, seed: int = 20261203) -> Tuple[np.ndarray, np.ndarray]:
    """Random real integrals: symmetric h ~ N(0, 1/n); two-body values with the
    8-fold symmetry of real orbitals drawn N(0, 0.1/n^2), then their
    magnitudes multiplied by a log-uniform factor in [1e-6, 1] (sign kept).
    Returned in the a†_p a†_q a_s a_r convention g_pqrs = (pr|qs)."""
    rng = np.random.default_rng(seed)
    h = rng.normal(scale=np.sqrt(1.0 / n), size=(n, n))
    h = (h + h.T) / np.sqrt(2.0)
    c = np.zeros((n, n, n, n))
    for i in range(n):
        for j in range(i + 1):
            for k in range(n):
                for l in range(k + 1):
                    if i * (i + 1) // 2 + j < k * (k + 1) // 2 + l:
                        continue
                    v = rng.normal(scale=np.sqrt(0.1) / n) * 10.0 ** rng.uniform(-6.0, 0.0)
                    for a, b, cc, d in ((i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k)):
                        c[a, b, cc, d] = v
                        c[cc, d, a, b] = v
    g = np.transpose(c, (0, 2, 1, 3))  # g_pqrs = (pr|qs): g[p,q,r,s] = c[p,r,q,s]
    return h, np.ascontiguousarray(g)
