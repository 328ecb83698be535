"""State-sharded MVP over several ranks (one process per GPU).

The 2^n state is split over P = 2^p ranks by its top p index bits (qubits
0 .. p-1, the most significant ones): rank r holds rows
[r * 2^(n-p), (r + 1) * 2^(n-p)).  A term with x mask m and z mask z maps the
partner shard r ^ (m >> (n-p)) onto rank r's rows, so

    y_r = sum over distinct top patterns d of  H_d(r) x_{r ^ d}

where H_d(r) is a Pauli operator on the n-p low qubits: the terms whose top
x bits equal d, with their low masks and their coefficients multiplied by the
top-bit sign (-1)^{popcount(z_top & (r ^ d))} (the column's top bits are
those of the partner shard) -- the sign rule of
``crates/tencir-pauli-core/src/hamiltonian.rs:238-243`` split across shards.

Every rank takes the same exchange steps in the same order: for each nonzero
pattern d (ascending), one pairwise send/receive with rank r ^ d through
``torch.distributed`` (NCCL on GPUs, gloo on CPU), then one local apply of
H_d(r) to the received shard, added into y by the kernel itself
(``tcp_mvp_apply_add_device``).  Two receive buffers alternate, and the
exchange of pattern d+1 is posted before the apply of pattern d, so the
transfer overlaps the compute.  The pattern d = 0 is applied to the local
shard without communication.  Transfers go into receive buffers in the
rank's own memory and the local kernels read only local memory.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable, Dict, List, Optional, Tuple

import numpy as np

from .pauli import PauliOperator


@dataclass
class ShardTerms:
    """Low-qubit term list of H_d(r) for one top pattern d on one rank."""

    pattern: int
    partner: int
    codes: np.ndarray  # (T_d, n - p) uint8
    coefficients: np.ndarray  # (T_d,) complex128, top-bit sign folded in


def split_operator(op: PauliOperator, world: int, rank: int) -> List[ShardTerms]:
    """Per-pattern low-qubit operators of rank `rank` out of `world` ranks."""
    if world < 1 or world & (world - 1):
        raise ValueError("the number of ranks must be a power of two")
    p = world.bit_length() - 1
    n = op.nqubits
    if p > n:
        raise ValueError("more ranks than basis-state blocks")
    codes = op.codes
    coeffs = op.coefficients
    # Top index bits are qubits 0..p-1 (qubit 0 is the most significant bit):
    # pattern bit (p-1-q) <- qubit q.
    x_top = np.zeros(len(coeffs), dtype=np.int64)
    z_top = np.zeros(len(coeffs), dtype=np.int64)
    for q in range(p):
        bit = 1 << (p - 1 - q)
        x_top |= np.where((codes[:, q] == 1) | (codes[:, q] == 2), bit, 0)
        z_top |= np.where((codes[:, q] == 2) | (codes[:, q] == 3), bit, 0)
    # Y letters on the top qubits keep their i factor: the phase i^{#Y} of the
    # whole word equals i^{#Y_top} * i^{#Y_low}; carry i^{#Y_top} explicitly.
    y_top = np.zeros(len(coeffs), dtype=np.int64)
    for q in range(p):
        y_top += codes[:, q] == 2
    phase = np.array([1, 1j, -1, -1j], dtype=np.complex128)[y_top % 4]
    out: List[ShardTerms] = []
    for d in sorted(set(int(v) for v in x_top)):
        sel = x_top == d
        partner = rank ^ d
        sign = np.array([-1.0 if bin(int(z) & partner).count("1") & 1 else 1.0 for z in z_top[sel]])
        out.append(
            ShardTerms(
                pattern=d,
                partner=partner,
                codes=np.ascontiguousarray(codes[sel, p:]),
                coefficients=coeffs[sel] * phase[sel] * sign,
            )
        )
    return out


class ShardedMVP:
    """y = H x with x, y split by the top bits over the ranks of a process group.

    Each shard exchange waits at most `timeout_s` seconds; a partner that left
    the group surfaces as an exception on the remaining ranks.

    ``apply_fn(shard_terms, x_shard, y_shard, accumulate)`` applies the low-qubit
    operator of one pattern to a shard; by default it builds device plans
    (``PauliOperator.native_mvp_plan``) and runs them on torch CUDA tensors.
    """

    def __init__(
        self, op: PauliOperator, group: Any = None, apply_fn: Optional[Callable] = None, timeout_s: float = 60.0
    ) -> None:
        import datetime

        import torch.distributed as dist

        self.timeout = datetime.timedelta(seconds=timeout_s)
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.nqubits = op.nqubits
        self.local_qubits = op.nqubits - (self.world.bit_length() - 1)
        self.shard_len = 1 << self.local_qubits
        self.parts = split_operator(op, self.world, self.rank)
        self.apply_fn = apply_fn or self._device_apply
        self._plans: Dict[int, Any] = {}
        # every rank must take the same exchange steps: the union of patterns
        self.patterns = sorted(set(d for d in range(1, self.world) if any(pt.pattern == d for pt in self.parts)))

    def _device_apply(self, part: ShardTerms, x: Any, y: Any, accumulate: bool) -> None:
        plan = self._plans.get(part.pattern)
        if plan is None:
            low = PauliOperator.from_code_arrays(part.codes, part.coefficients) if len(part.coefficients) else PauliOperator.empty(self.local_qubits)
            plan = low.native_mvp_plan()
            self._plans[part.pattern] = plan
        plan.apply_device(x, y, accumulate=accumulate)

    def receive_buffers(self, like: Any) -> List[Any]:
        """The receive buffers that ``apply`` alternates between (two when
        there are at least two exchange steps)."""
        import torch

        return [torch.empty_like(like) for _ in range(min(2, len(self.patterns)))]

    def _post(self, d: int, x: Any, buf: Any) -> List[Any]:
        partner = self.rank ^ d
        ops = [
            self.dist.P2POp(self.dist.isend, x, partner, group=self.group),
            self.dist.P2POp(self.dist.irecv, buf, partner, group=self.group),
        ]
        return self.dist.batch_isend_irecv(ops)

    def apply(self, x: Any, y: Any, recv: Optional[Any] = None) -> None:
        """y_r = sum_d H_d(r) x_{r ^ d}; x, y are this rank's shards.  ``recv``
        is one buffer or a list of buffers shaped like x (default: fresh ones)."""
        if x.shape[-1] != self.shard_len or y.shape != x.shape:
            raise ValueError(f"shards must have length {self.shard_len}")
        by_pattern = {pt.pattern: pt for pt in self.parts}
        local = by_pattern.get(0)
        if local is not None:
            self.apply_fn(local, x, y, False)
        else:
            y.zero_()
        if not self.patterns:
            return
        if recv is None:
            bufs = self.receive_buffers(x)
        else:
            bufs = list(recv) if isinstance(recv, (list, tuple)) else [recv]
        pending = self._post(self.patterns[0], x, bufs[0])
        for i, d in enumerate(self.patterns):
            reqs, buf = pending, bufs[i % len(bufs)]
            following = None
            if i + 1 < len(self.patterns) and len(bufs) > 1:
                # the next exchange runs while this pattern is applied; its
                # buffer was read by the apply before the previous one, which
                # is ordered before it on the device
                following = self._post(self.patterns[i + 1], x, bufs[(i + 1) % len(bufs)])
            # A partner that left makes this wait end with an error after the
            # timeout instead of blocking the rank for good.
            for req in reqs:
                req.wait(self.timeout)
            part = by_pattern.get(d)
            if part is not None:
                self.apply_fn(part, buf, y, True)
            if i + 1 < len(self.patterns):
                pending = following if following is not None else self._post(self.patterns[i + 1], x, bufs[0])
