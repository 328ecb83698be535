"""Learned Davidson preconditioner: a small MLP over per-basis-state features.

The Jacobi correction is ``t_i = -r_i / (H_ii - theta)``.  The learned one is
``t_i = -exp(c_i) r_i / (H_ii - theta)`` where ``c_i`` is the output of a
two-hidden-layer tanh MLP (``TCP_MLP_IN`` -> 16 -> 16 -> 1) evaluated on the
basis state's features (``tcp_state_features``: ``H_ii - theta``, the
diagonals of the states it couples to, its coupling strengths and count, its
Hamming weight; energies divided by a size-intensive scale).  ``c = 0`` is
exactly Jacobi, so an untrained network reproduces the plain method.

Training data come from the method's own solves on smaller lattices: for each
(lattice, J2) the lowest eigenpairs are first converged to 1e-10 with the
plain method; then a Jacobi-preconditioned Davidson run is replayed and, at
every iteration, each Ritz vector ``u`` with residual ``r`` yields the exact
correction ``e = P u - u`` (``P``: projector onto the exact eigenspace of the
matching eigenvalue), made orthogonal to ``u`` and scaled to the Jacobi
correction's norm.  Per sampled basis state the loss is
``|g r_i - e_i|^2`` with ``g = -exp(c) / den``; it is minimised with Adam by
the device kernels ``tcp_mlp_train_step`` (forward, backward, Adam) -- the
gradient is checked against a NumPy restatement in the test-suite.

Weights are saved as versioned ``.npz`` files (``format_version``, the layer
shape, the training configuration).
"""

from __future__ import annotations

import os
from dataclasses import dataclass
from typing import Any, Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import solver_ops

FORMAT_VERSION = 1
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "mlp_precond_j1j2.npz")


def energy_scale(op: Any) -> float:
    """Size-intensive energy unit: sum of |coefficients| per qubit."""
    return float(np.abs(op.coefficients).sum()) / max(1, op.nqubits)


def init_params(seed: int = 0) -> np.ndarray:
    """Small random hidden layers and a zero output layer (= Jacobi)."""
    rng = np.random.default_rng(seed)
    IN, H = solver_ops.TCP_MLP_IN, solver_ops.TCP_MLP_HIDDEN
    w1 = rng.normal(scale=1.0 / np.sqrt(IN), size=(H, IN))
    b1 = np.zeros(H)
    w2 = rng.normal(scale=1.0 / np.sqrt(H), size=(H, H))
    b2 = np.zeros(H)
    w3 = np.zeros(H)
    b3 = np.zeros(1)
    return np.concatenate([w1.ravel(), b1, w2.ravel(), b2, w3, b3]).astype(np.float32)


class MLPPreconditioner:
    """Davidson correction from the trained network (Jacobi when c = 0)."""

    name = "mlp"

    def __init__(self, params: np.ndarray, scale: Optional[float] = None, clamp: float = 4.0) -> None:
        import torch

        params = np.asarray(params, dtype=np.float32).ravel()
        if params.size != solver_ops.TCP_MLP_PARAMS:
            raise ValueError(f"expected {solver_ops.TCP_MLP_PARAMS} parameters, got {params.size}")
        self.params = torch.from_numpy(params.copy()).cuda()
        self.scale = scale
        self.clamp = clamp
        self.features = None

    def prepare(self, plan: Any, diag: Any) -> None:
        self.features = solver_ops.state_features(plan)
        self.diag = diag
        if self.scale is None:
            raise ValueError("MLPPreconditioner needs the operator's energy scale")

    def __call__(self, R: Any, theta: Any, out: Any) -> bool:
        solver_ops.mlp_precondition(R, self.features, self.diag, theta, self.params, self.scale, out, clamp=self.clamp)
        return True

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, scale: Optional[float] = None) -> "MLPPreconditioner":
        with np.load(path) as data:
            if int(data["format_version"]) != FORMAT_VERSION:
                raise ValueError(f"unsupported weight format {int(data['format_version'])}")
            if tuple(int(v) for v in data["layers"]) != (solver_ops.TCP_MLP_IN, solver_ops.TCP_MLP_HIDDEN, solver_ops.TCP_MLP_HIDDEN, 1):
                raise ValueError("weight file layer shape does not match this build")
            params = data["params"]
        return cls(params, scale=scale)


def save_params(path: str, params: np.ndarray, config: Dict[str, Any]) -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez(
        path,
        format_version=np.int64(FORMAT_VERSION),
        layers=np.asarray([solver_ops.TCP_MLP_IN, solver_ops.TCP_MLP_HIDDEN, solver_ops.TCP_MLP_HIDDEN, 1], dtype=np.int64),
        params=np.asarray(params, dtype=np.float32),
        config=np.asarray(repr(config)),
    )


@dataclass
class TrainingSet:
    X: Any  # (S, TCP_MLP_IN) float32 CUDA
    den: Any
    a: Any
    b: Any
    e2: Any
    wt: Any

    @property
    def size(self) -> int:
        return int(self.X.shape[0])


def _cat(sets: Sequence[TrainingSet]) -> TrainingSet:
    import torch

    return TrainingSet(*[torch.cat([getattr(s, f) for s in sets]) for f in ("X", "den", "a", "b", "e2", "wt")])


def collect_samples(
    op: Any,
    nev: int = 4,
    rows_per_vector: int = 8192,
    max_iterations: int = 60,
    seed: int = 0,
    tol_exact: float = 1e-10,
) -> TrainingSet:
    """Samples (inputs, denominators, |r|^2, Re(conj(e) r), |e|^2, weights)
    from a Jacobi Davidson trajectory on `op`, against its exact eigenpairs."""
    import torch

    from .davidson import davidson

    plan = op.native_mvp_plan()
    exact = davidson(plan, nev=nev + 2, tol=tol_exact, seed=seed + 1000, max_subspace=48)
    lam = torch.from_numpy(exact.eigenvalues)
    Uex = exact.vectors  # (nev+2, n) complex128
    scale = energy_scale(op)
    features = solver_ops.state_features(plan)
    diag = torch.empty(plan.dimension, dtype=torch.complex128, device="cuda")
    plan._native_plan.diagonal_device(diag)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    out: List[TrainingSet] = []

    def record(dtype, iteration, theta, U, R, V, norms):
        if iteration > max_iterations:
            return
        U64 = U.to(torch.complex128)
        R64 = R.to(torch.complex128)
        for j in range(U64.shape[0]):
            if not (1e-9 < norms[j] < 1e-1):
                continue
            # exact eigenspace of the eigenvalue nearest theta_j
            near = torch.abs(lam - float(theta[j])) < 1e-6 + 1e-3 * float(norms[j])
            if not bool(near.any()):
                near = torch.abs(lam - float(theta[j])) == torch.abs(lam - float(theta[j])).min()
            Q = Uex[near.nonzero().flatten().cuda()]
            c = solver_ops.gram(Q, U64[j : j + 1]).reshape(-1)  # Q^H u
            Pu = (c[:, None] * Q).sum(0)
            e = Pu - U64[j]
            e = e - torch.vdot(U64[j], e) * U64[j]
            t_j = -R64[j] / torch.clamp(torch.abs(diag.real - float(theta[j])), min=1e-8) * torch.sign(diag.real - float(theta[j]))
            en = torch.linalg.vector_norm(e)
            if float(en) == 0.0:
                continue
            e = e * (torch.linalg.vector_norm(t_j) / en)
            rows = torch.randint(0, plan.dimension, (rows_per_vector,), generator=gen, device="cuda")
            rows_u = rows.to(torch.int64).contiguous()
            which = torch.zeros(rows_per_vector, dtype=torch.int32, device="cuda")
            X, den = solver_ops.mlp_inputs(features, rows_u, theta[j : j + 1], which, scale)
            rr = R64[j][rows]
            ee = e[rows]
            a = (rr.real**2 + rr.imag**2).float()
            b = (ee.real * rr.real + ee.imag * rr.imag).float()
            e2 = (ee.real**2 + ee.imag**2).float()
            wsum = float(e2.sum()) + 1e-300
            wt = torch.full_like(a, 1.0 / wsum)
            out.append(TrainingSet(X, den, a, b, e2, wt))

    davidson(plan, nev=nev, tol=1e-9, seed=seed, callback=record, max_iter=max_iterations + 5, switch_tol=1e-6)
    return _cat(out) if out else None


def train(
    data: TrainingSet,
    params: Optional[np.ndarray] = None,
    steps: int = 600,
    lr: float = 3e-3,
    seed: int = 0,
    log_every: int = 100,
) -> Tuple[np.ndarray, List[float]]:
    """Full-batch Adam on the device kernels; returns (params, loss history)."""
    import torch

    p = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).cuda()
    trainer = solver_ops.MLPTrainer(p)
    losses: List[float] = []
    for s in range(steps):
        trainer.step(data.X, data.den, data.a, data.b, data.e2, data.wt, lr)
        if s % log_every == 0 or s == steps - 1:
            losses.append(float(trainer.loss.item()))
    return p.cpu().numpy(), losses


def training_lattices(count: int = 6, seed: int = 0) -> List[Tuple[int, int, float]]:
    """(lx, ly, J2) for the training solves: 4x4 and 4x5 with J2 ~ U[0, 0.6]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        lx, ly = (4, 4) if i % 2 == 0 else (4, 5)
        out.append((lx, ly, float(rng.uniform(0.0, 0.6))))
    return out


def train_from_lattices(
    lattices: Iterable[Tuple[int, int, float]], steps: int = 600, seed: int = 0, rows_per_vector: int = 8192
) -> Tuple[np.ndarray, Dict[str, Any]]:
    from .pauli import PauliOperator
    from .workloads import j1j2_periodic

    sets = []
    for i, (lx, ly, j2) in enumerate(lattices):
        op = PauliOperator.from_code_arrays(*j1j2_periodic(lx, ly, 1.0, j2))
        s = collect_samples(op, seed=seed + i, rows_per_vector=rows_per_vector)
        if s is not None:
            sets.append(s)
    data = _cat(sets)
    params, losses = train(data, steps=steps, seed=seed)
    return params, {"samples": data.size, "losses": losses, "lattices": list(lattices), "steps": steps}


# ---------------------------------------------------------------------------
# Alignment objective: train the network so that its correction points along
# the direction Davidson is missing.  For a Ritz vector u of a trajectory with
# basis V and residual r, the ideal new direction is e = (I - V V^H) v, with v
# the projection of u onto the exact eigenspace.  The correction t = g o r
# (g = -exp(c) / den per basis state) is scored by the squared cosine between
# t, made orthogonal to u, and e:
#     L = 1 - |<e, t>|^2 / (||e||^2 (||t||^2 - |<u, t>|^2))
# (<e, t> needs no projection since e is orthogonal to V).  The loss is
# invariant to the scale of t, as the Davidson expansion is.
# ---------------------------------------------------------------------------
@dataclass
class AlignmentSets:
    X: Any  # (N, TCP_MLP_IN) float32 network inputs, all basis states of every set
    den: Any  # (N,) float32
    alpha: Any  # (N,) complex128: conj(e_i) r_i
    a: Any  # (N,) float64: |r_i|^2
    gamma: Any  # (N,) complex128: conj(u_i) r_i
    E: Any  # (S,) float64: ||e||^2 per set
    seg: Any  # (N,) int64 set index
    nsets: int
    seg_begin: Any = None  # (S + 1,) int64 offsets of the sets (contiguous)


def _cat_alignment(parts: Sequence[AlignmentSets]) -> AlignmentSets:
    import torch

    offset = 0
    segs = []
    for p in parts:
        segs.append(p.seg + offset)
        offset += p.nsets
    return AlignmentSets(
        X=torch.cat([p.X for p in parts]),
        den=torch.cat([p.den for p in parts]),
        alpha=torch.cat([p.alpha for p in parts]),
        a=torch.cat([p.a for p in parts]),
        gamma=torch.cat([p.gamma for p in parts]),
        E=torch.cat([p.E for p in parts]),
        seg=torch.cat(segs),
        nsets=offset,
        seg_begin=_offsets(torch.cat(segs), offset),
    )


def _offsets(seg: Any, nsets: int) -> Any:
    """Offsets of the sets; the states of a set must be contiguous."""
    import torch

    if seg.numel() > 1 and not bool(torch.all(seg[1:] >= seg[:-1])):
        raise ValueError("alignment training sets must be contiguous (set index non-decreasing)")
    begin = torch.zeros(nsets + 1, dtype=torch.int64, device=seg.device)
    begin[1:] = torch.cumsum(torch.bincount(seg, minlength=nsets), 0)
    return begin


def collect_alignment_sets(
    op: Any, nev: int = 4, every: int = 3, max_iterations: int = 45, seed: int = 0, tol_exact: float = 1e-10
) -> Optional[AlignmentSets]:
    """Full-vector training sets from a Jacobi Davidson trajectory on `op`."""
    import torch

    from .davidson import davidson

    plan = op.native_mvp_plan()
    exact = davidson(plan, nev=nev + 2, tol=tol_exact, seed=seed + 1000)
    lam = torch.from_numpy(exact.eigenvalues)
    Uex = exact.vectors
    scale = energy_scale(op)
    features = solver_ops.state_features(plan)
    n = plan.dimension
    all_rows = torch.arange(n, dtype=torch.int64, device="cuda")
    zeros = torch.zeros(n, dtype=torch.int32, device="cuda")
    parts: List[AlignmentSets] = []

    def record(dtype, iteration, theta, U, R, V, norms):
        if iteration > max_iterations or iteration % every:
            return
        for j in range(U.shape[0]):
            if not (1e-9 < norms[j] < 1e-1):
                continue
            dist = torch.abs(lam - float(theta[j]))
            near = dist < 1e-6 + 1e-3 * float(norms[j])
            if not bool(near.any()):
                near = dist == dist.min()
            Q = Uex[near.nonzero().flatten().cuda()]
            uj = U[j : j + 1].to(torch.complex128).contiguous()
            c = solver_ops.gram(Q, uj)  # Q^H u
            v = torch.empty_like(uj)
            solver_ops.combine(Q, c, v)
            e = v.clone()
            for _ in range(2):  # e = (I - V V^H) v
                C = solver_ops.gram(V, e)
                solver_ops.combine(V, C, e, alpha=-1.0, beta=1.0)
            E = float(torch.linalg.vector_norm(e) ** 2)
            if E <= 1e-30:
                continue
            X, den = solver_ops.mlp_inputs(features, all_rows, theta[j : j + 1], zeros, scale)
            r = R[j].to(torch.complex128)
            u = uj[0]
            parts.append(
                AlignmentSets(
                    X=X,
                    den=den,
                    alpha=torch.conj(e[0]) * r,
                    a=(r.real**2 + r.imag**2),
                    gamma=torch.conj(u) * r,
                    E=torch.tensor([E], dtype=torch.float64, device="cuda"),
                    seg=torch.zeros(n, dtype=torch.int64, device="cuda"),
                    nsets=1,
                )
            )

    davidson(plan, nev=nev, tol=1e-9, seed=seed, callback=record, max_iter=max_iterations + 1)
    return _cat_alignment(parts) if parts else None


def alignment_loss_and_dc(c: Any, data: AlignmentSets, clamp: float = 4.0, work: Any = None):
    """Mean alignment loss over the sets and dL/dc per basis state, from the
    device kernels of tcp_mlp_alignment_grad (per-set sums in a fixed order,
    then the elementwise derivative)."""
    seg_begin = data.seg_begin if data.seg_begin is not None else _offsets(data.seg, data.nsets)
    return solver_ops.alignment_grad(c, data.den, data.alpha, data.a, data.gamma, data.E, data.seg, seg_begin, clamp,
                                     work=work)


def train_alignment(
    data: AlignmentSets, params: Optional[np.ndarray] = None, steps: int = 300, lr: float = 3e-3, seed: int = 0, log_every: int = 50
) -> Tuple[np.ndarray, List[float]]:
    """Adam on the alignment loss, every step on the device kernels:
    tcp_mlp_forward, tcp_mlp_alignment_grad (the loss and dL/dc) and
    tcp_mlp_backward_step (back-propagation and the Adam update)."""
    import torch

    p = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).cuda()
    trainer = solver_ops.MLPTrainer(p)
    work = torch.empty(int(solver_ops._lib().tcp_mlp_alignment_work_bytes(data.nsets)) // 8, dtype=torch.float64,
                       device="cuda")
    losses: List[float] = []
    for s in range(steps):
        c = solver_ops.mlp_forward(data.X, p)
        loss, dc = alignment_loss_and_dc(c, data, work=work)
        trainer.backward_step(data.X, dc, lr)
        if s % log_every == 0 or s == steps - 1:
            losses.append(loss)
    return p.cpu().numpy(), losses


def train_alignment_from_lattices(
    lattices: Iterable[Tuple[int, int, float]], steps: int = 300, seed: int = 0, every: int = 3
) -> Tuple[np.ndarray, Dict[str, Any]]:
    from .pauli import PauliOperator
    from .workloads import j1j2_periodic

    parts = []
    for i, (lx, ly, j2) in enumerate(lattices):
        op = PauliOperator.from_code_arrays(*j1j2_periodic(lx, ly, 1.0, j2))
        s = collect_alignment_sets(op, seed=seed + i, every=every)
        if s is not None:
            parts.append(s)
    data = _cat_alignment(parts)
    params, losses = train_alignment(data, steps=steps, seed=seed)
    return params, {"objective": "alignment", "sets": data.nsets, "states": int(data.X.shape[0]), "losses": losses,
                    "lattices": list(lattices), "steps": steps}
