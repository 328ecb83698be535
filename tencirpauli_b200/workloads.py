"""Deterministic synthetic workloads for the MVP path (seeds recorded here).

Each generator returns raw ``(codes uint8[T, n], coefficients complex128[T])``
term rows; :class:`~tencirpauli_b200.pauli.PauliOperator` canonicalizes them
(duplicate words merge, so the canonical term count can be below the raw one).

* :func:`heisenberg_chain`     periodic XX+YY+ZZ chain plus a uniform Z field
* :func:`random_k_local`       random 2..4-local words, real N(0,1) coefficients
* :func:`heisenberg_2d_open`   open L_x x L_y lattice, one J ~ U[0.5, 1.5] per bond
* :func:`j1j2_periodic`        periodic J1-J2 square lattice
* :func:`random_state`         i.i.d. normal re/im, L2-normalised
"""

from __future__ import annotations

from typing import Optional, List, Tuple

import numpy as np

SEED = 20261203

X, Y, Z = 1, 2, 3


def _two_site(n: int, a: int, b: int, letter: int) -> np.ndarray:
    row = np.zeros(n, dtype=np.uint8)
    row[a] = letter
    row[b] = letter
    return row


def heisenberg_chain(n: int = 20, field: float = 0.5) -> Tuple[np.ndarray, np.ndarray]:
    """sum_i (X_i X_{i+1} + Y_i Y_{i+1} + Z_i Z_{i+1}) + field * sum_i Z_i, periodic."""
    rows: List[np.ndarray] = []
    coeffs: List[complex] = []
    for i in range(n):
        j = (i + 1) % n
        if i == j:
            continue
        for letter in (X, Y, Z):
            rows.append(_two_site(n, i, j, letter))
            coeffs.append(1.0)
    for i in range(n):
        row = np.zeros(n, dtype=np.uint8)
        row[i] = Z
        rows.append(row)
        coeffs.append(field)
    return np.asarray(rows, dtype=np.uint8).reshape(-1, n), np.asarray(coeffs, dtype=np.complex128)


def random_k_local(
    n: int = 28, words: int = 2000, seed: int = SEED, weights: Tuple[int, ...] = (2, 3, 4)
) -> Tuple[np.ndarray, np.ndarray]:
    """``words`` Pauli words: weight uniform in ``weights`` on distinct uniformly
    random qubits, each letter uniform over X/Y/Z, coefficient real N(0,1)."""
    rng = np.random.default_rng(seed)
    codes = np.zeros((words, n), dtype=np.uint8)
    for t in range(words):
        w = int(rng.choice(weights))
        qubits = rng.choice(n, size=w, replace=False)
        codes[t, qubits] = rng.integers(1, 4, size=w)
    coeffs = rng.normal(size=words).astype(np.complex128)
    return codes, coeffs


def lattice_shape(n: int) -> Tuple[int, int]:
    """Most-square factorisation L_x * L_y == n with L_x <= L_y (prime n: 1 x n)."""
    best = (1, n)
    for lx in range(1, int(np.sqrt(n)) + 1):
        if n % lx == 0:
            best = (lx, n // lx)
    return best


def heisenberg_2d_open(n: int, seed: int) -> Tuple[np.ndarray, np.ndarray]:
    """Open L_x x L_y nearest-neighbour XX+YY+ZZ with one J ~ U[0.5, 1.5] per bond."""
    rng = np.random.default_rng(seed)
    lx, ly = lattice_shape(n)
    rows: List[np.ndarray] = []
    coeffs: List[float] = []
    for yy in range(ly):
        for xx in range(lx):
            site = yy * lx + xx
            for nb in ((site + 1) if xx + 1 < lx else None, (site + lx) if yy + 1 < ly else None):
                if nb is None:
                    continue
                j = float(rng.uniform(0.5, 1.5))
                for letter in (X, Y, Z):
                    rows.append(_two_site(n, site, nb, letter))
                    coeffs.append(j)
    return np.asarray(rows, dtype=np.uint8).reshape(-1, n), np.asarray(coeffs, dtype=np.complex128)


def batched_heisenberg_set(count: int = 64, seed: int = SEED, nmin: int = 16, nmax: int = 26):
    """``count`` open 2D Heisenberg lattices with n ~ U{nmin..nmax}; yields (n, codes, coeffs)."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nmin, nmax + 1, size=count)
    return [(int(n), *heisenberg_2d_open(int(n), seed + 1 + i)) for i, n in enumerate(sizes)]


def j1j2_periodic(lx: int = 4, ly: int = 6, j1: float = 1.0, j2: float = 0.5) -> Tuple[np.ndarray, np.ndarray]:
    """Periodic J1-J2 Heisenberg on an lx x ly square lattice (sites y*lx + x).

    J1 bonds: right and up neighbours; J2 bonds: both diagonals.  Each bond
    contributes J (X X + Y Y + Z Z)."""
    n = lx * ly
    rows: List[np.ndarray] = []
    coeffs: List[float] = []

    def site(xx: int, yy: int) -> int:
        return (yy % ly) * lx + (xx % lx)

    bonds = []
    for yy in range(ly):
        for xx in range(lx):
            s = site(xx, yy)
            bonds.append((s, site(xx + 1, yy), j1))
            bonds.append((s, site(xx, yy + 1), j1))
            if j2 != 0.0:
                bonds.append((s, site(xx + 1, yy + 1), j2))
                bonds.append((s, site(xx - 1, yy + 1), j2))
    for a, b, j in bonds:
        if a == b:
            continue
        for letter in (X, Y, Z):
            rows.append(_two_site(n, a, b, letter))
            coeffs.append(j)
    return np.asarray(rows, dtype=np.uint8).reshape(-1, n), np.asarray(coeffs, dtype=np.complex128)


def random_state(n: int, seed: int = SEED, dtype: type = np.complex128) -> np.ndarray:
    """re, im i.i.d. N(0,1) from ``seed``, then L2-normalised (host numpy)."""
    rng = np.random.default_rng(seed)
    dim = 1 << n
    state = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
    state /= np.linalg.norm(state)
    return state.astype(dtype)


def random_state_device(n: int, seed: int = SEED, dtype=None, device: str = "cuda", nrhs: int = 0,
                        length: Optional[int] = None):
    """The same distribution generated on the device with torch (large n).
    ``length`` overrides the 2^n entries (restricted sector states)."""
    import torch

    dtype = dtype or torch.complex128
    real = torch.float64 if dtype == torch.complex128 else torch.float32
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    size = (1 << n) if length is None else int(length)
    shape = (nrhs, size) if nrhs else (size,)
    re = torch.randn(shape, generator=gen, device=device, dtype=real)
    im = torch.randn(shape, generator=gen, device=device, dtype=real)
    state = torch.complex(re, im)
    del re, im
    norm = torch.linalg.vector_norm(state, dim=-1, keepdim=True)
    state /= norm
    return state
