"""Multi-rank sharded MVP on CPU: world sizes 2 and 4 as gloo process groups.

Each rank holds the shard of the state selected by the top index bits and
exchanges shards pairwise (``tencirpauli_b200/sharded.py``); the local applies
run through the oracle here (the CPU checker), on the GPU they run the device
plans.  The gathered result must equal the oracle's full MVP.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from oracle import oracle


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle_apply(part, x, y, accumulate):
    import torch

    n_local = part.codes.shape[1]
    if len(part.coefficients):
        xw, zw, c = oracle.canonicalize(n_local, part.codes, part.coefficients)
        xm, zm, wp = oracle.matrix_terms(n_local, xw, zw, c)
        out = oracle.apply_term_direct(n_local, xm, zm, wp, x.numpy())
    else:
        out = np.zeros(x.shape[0], dtype=np.complex128)
    if accumulate:
        y += torch.from_numpy(out)
    else:
        y.copy_(torch.from_numpy(out))


def _worker(rank: int, world: int, port: int, n: int, seed: int, result_path: str) -> None:
    import torch
    import torch.distributed as dist

    from tencirpauli_b200 import PauliOperator, workloads
    from tencirpauli_b200.sharded import ShardedMVP

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    codes, coeffs = workloads.random_k_local(n=n, words=60, seed=seed)
    coeffs = coeffs * (1.0 + 0.25j)
    op = PauliOperator.from_code_arrays(codes, coeffs)
    state = workloads.random_state(n, seed=seed + 1)
    mvp = ShardedMVP(op, apply_fn=_oracle_apply)
    shard = mvp.shard_len
    x = torch.from_numpy(state[rank * shard : (rank + 1) * shard].copy())
    y = torch.empty_like(x)
    mvp.apply(x, y)
    gathered = [torch.empty_like(y) for _ in range(world)]
    dist.all_gather(gathered, y)
    if rank == 0:
        np.save(result_path, torch.cat(gathered).numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_sharded_mvp_matches_full_oracle(world: int, tmp_path) -> None:
    import torch.multiprocessing as mp

    from tencirpauli_b200 import PauliOperator, workloads

    n, seed = 10, 11
    result = str(tmp_path / "y.npy")
    mp.start_processes(_worker, args=(world, _free_port(), n, seed, result), nprocs=world, join=True, start_method="spawn")
    y = np.load(result)
    codes, coeffs = workloads.random_k_local(n=n, words=60, seed=seed)
    op = PauliOperator.from_code_arrays(codes, coeffs * (1.0 + 0.25j))
    xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
    ref = oracle.apply_term_direct(n, xm, zm, wp, workloads.random_state(n, seed=seed + 1))
    np.testing.assert_allclose(y, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_split_operator_patterns_and_signs() -> None:
    from tencirpauli_b200 import PauliOperator
    from tencirpauli_b200.sharded import split_operator

    # X on qubit 0 (top bit) and Z on qubit 0: patterns 1 and 0 for 2 ranks
    op = PauliOperator.from_terms(3, [("XII", 1.0), ("ZIZ", 0.5), ("YZI", 2.0)])
    for rank in (0, 1):
        parts = {p.pattern: p for p in split_operator(op, 2, rank)}
        assert set(parts) == {0, 1}
        assert parts[1].partner == rank ^ 1
        # ZIZ: column top bit = rank (pattern 0) -> sign (-1)^rank
        z_coeff = parts[0].coefficients[0]
        assert z_coeff == (0.5 if rank == 0 else -0.5)
    with pytest.raises(ValueError, match="power of two"):
        split_operator(op, 3, 0)


def _leaving_worker(rank: int, world: int, port: int, result_path: str) -> None:
    import datetime

    import torch
    import torch.distributed as dist

    from tencirpauli_b200 import PauliOperator
    from tencirpauli_b200.sharded import ShardedMVP

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=3))
    op = PauliOperator.from_terms(4, [("XIII", 1.0), ("ZZII", 0.5)])
    mvp = ShardedMVP(op, apply_fn=_oracle_apply, timeout_s=3.0)
    x = torch.ones(mvp.shard_len, dtype=torch.complex128)
    y = torch.empty_like(x)
    mvp.apply(x, y)  # one healthy step on both ranks
    if rank == 1:
        os._exit(0)  # leaves between steps, with nothing in flight
    try:
        mvp.apply(x, y)  # the partner is gone: the exchange must end in an error
        outcome = "no error"
    except Exception as exc:  # gloo raises on the closed connection or the timeout
        outcome = "error: " + type(exc).__name__
    with open(result_path, "w") as fh:
        fh.write(outcome)
    os._exit(0)


def test_rank_leaving_ends_the_partners_exchange_with_an_error(tmp_path) -> None:
    import torch.multiprocessing as mp

    result = str(tmp_path / "outcome.txt")
    import time

    ctx = mp.start_processes(_leaving_worker, args=(2, _free_port(), result), nprocs=2, join=False, start_method="spawn")
    deadline = time.time() + 90
    while time.time() < deadline and not os.path.exists(result):
        time.sleep(0.2)
    time.sleep(0.5)
    for proc in ctx.processes:
        if proc.is_alive():
            proc.kill()
        proc.join(5)
    assert open(result).read().startswith("error")
