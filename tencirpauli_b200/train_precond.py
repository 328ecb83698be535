"""Train the learned Davidson preconditioner on the GPU and save its weights.

    python -m tencirpauli_b200.train_precond --objective alignment --out tencirpauli_b200/data/mlp_precond_j1j2.npz

Training solves: periodic J1-J2 lattices 4x4 and 4x5 with J2 ~ U[0, 0.6]
(``precond.training_lattices``); see ``tencirpauli_b200/precond.py``.
Objectives: ``l2`` (distance of the correction to the exact one on sampled
rows) and ``alignment`` (squared cosine between the correction, made
orthogonal to the Ritz vector, and the direction Davidson is missing).
"""

from __future__ import annotations

import argparse
import json
import time

from . import precond


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=precond.DEFAULT_WEIGHTS)
    ap.add_argument("--lattices", type=int, default=6)
    ap.add_argument("--steps", type=int, default=800)
    ap.add_argument("--rows", type=int, default=8192)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--objective", choices=["l2", "alignment"], default="alignment")
    args = ap.parse_args()
    t0 = time.perf_counter()
    lattices = precond.training_lattices(args.lattices, seed=args.seed)
    if args.objective == "alignment":
        params, info = precond.train_alignment_from_lattices(lattices, steps=args.steps, seed=args.seed)
    else:
        params, info = precond.train_from_lattices(lattices, steps=args.steps, seed=args.seed, rows_per_vector=args.rows)
    info["seconds"] = time.perf_counter() - t0
    precond.save_params(args.out, params, info)
    print(json.dumps({"out": args.out, **{k: v for k, v in info.items() if k != "lattices"}, "lattices": lattices}))


if __name__ == "__main__":
    main()
