"""Benchmark of the B200 matrix-free Pauli MVP (one JSON line on rank 0).

Workload (default): the random 2..4-local Hamiltonian on n = 28 qubits --
2,000 raw words (weight uniform in {2,3,4} on distinct uniformly random
qubits, letters uniform over X/Y/Z, real N(0,1) coefficients, seed 20261203),
canonicalized -- applied to a complex128 statevector (re/im i.i.d. N(0,1),
L2-normalised).  A step is one y = H x over the whole 2^28 state.

Metric: amplitude-terms/s = T_canonical * 2^n * (vectors per step) / step time.
``value`` is device time (CUDA events on the launching stream, inputs resident
in HBM, 4 GiB vectors > L2 so no flush is needed); ``e2e`` is the same metric
through the public host ``apply_into`` path (H2D + kernel + D2H in every
step).  ``--impl reference`` times the reference's CPU algorithm (the C
restatement of the Rust TermDirect loop, all host cores) in fixed blocks of
rows of the same workload.

Multi-GPU (``torchrun --nproc-per-node N``): the one n = 28 state is sharded
over the ranks by its top index bits (strong scaling; pairwise shard
exchanges over NCCL, double-buffered against the applies); ``--replicas``
instead runs one independent state per rank (weak scaling, no collective on
the data path).  The step time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from typing import Any, Dict, List, Optional

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MVP amplitude-terms/s"
UNIT = "amp-terms/s"
FALLBACK_HBM_GBS = 6650.0


def _measured_peaks() -> Dict[str, Any]:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
        return {"hbm_gbs": float(data["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


def _profile_traffic(kernel: str) -> Optional[float]:
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            try:
                return float(parts[1])
            except ValueError:
                return None
    return None


def _profile_instructions(kernel: str, workload: str) -> Optional[float]:
    """Warp instructions per launch (smsp__inst_executed.sum) from the
    committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "instructions.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        parts = line.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


def _issue_roofline(kernel: str, workload: str, kernel_ms: float, clocks: Dict[str, Any]) -> Optional[Dict[str, Any]]:
    """Instruction-issue ceiling: an SM issues at most one warp instruction
    per clock on each of its 4 schedulers.  Achieved = the kernel's warp
    instructions per launch (ncu, committed) over the CUDA-event launch time;
    peak = 4 x SMs x the median SM clock sampled during the timed region."""
    import torch

    inst = _profile_instructions(kernel, workload)
    mhz = clocks.get("sm_mhz") if isinstance(clocks, dict) else None
    if inst is None or not mhz:
        return None
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    peak = 4.0 * sms * float(mhz) * 1e6
    achieved = inst / (kernel_ms / 1000.0)
    return {"achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "T warp-instructions/s", "frac": achieved / peak,
            "instructions_per_launch": inst, "source": "profiles/instructions.txt (ncu smsp__inst_executed.sum)"}


def manifest(with_gpu: bool = True) -> Dict[str, Any]:
    """What produced a bench line: the library's build record (source commit,
    nvcc release), a digest of the sources as they ran, host core count,
    driver, toolkit and framework versions."""
    import hashlib
    import platform

    info: Dict[str, Any] = {"nproc": os.cpu_count(), "python": platform.python_version(), "numpy": np.__version__}
    build_info = os.path.join(ROOT, "tencirpauli_b200", "_lib", "build_info.json")
    if os.path.exists(build_info):
        with open(build_info) as fh:
            info["build"] = json.load(fh)
    digest = hashlib.sha256()
    csrc = os.path.join(ROOT, "tencirpauli_b200", "csrc")
    for name in sorted(os.listdir(csrc)) + ["../../bench.py"]:
        with open(os.path.join(csrc, name), "rb") as fh:
            digest.update(fh.read())
    info["sources_sha16"] = digest.hexdigest()[:16]
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=driver_version,name", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout.strip().splitlines()
        if out:
            driver, name = (p.strip() for p in out[0].split(",", 1))
            info["driver"] = driver
            info["gpu"] = name
    except (OSError, subprocess.SubprocessError, ValueError):
        pass
    if with_gpu:
        import torch

        info["torch"] = torch.__version__
        info["torch_cuda"] = torch.version.cuda
    return info


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device_index: int) -> None:
        self.device_index = device_index
        self.proc: Optional[subprocess.Popen] = None
        self.path = tempfile.mktemp(prefix="tcp_clocks_", suffix=".csv")

    def start(self) -> None:
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                [
                    "nvidia-smi",
                    f"--id={self.device_index}",
                    f"--query-gpu={self.FIELDS}",
                    "--format=csv,noheader,nounits",
                    "-lms",
                    "200",
                ],
                stdout=self.fh,
                stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> Dict[str, Any]:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm: List[float] = []
        smax: List[float] = []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def _smi_id(device: int) -> str:
    """nvidia-smi --id for a torch ordinal (PCI bus id: robust to CUDA_VISIBLE_DEVICES)."""
    import torch

    props = torch.cuda.get_device_properties(device)
    try:
        return f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    except AttributeError:
        return str(device)


def build_operator(args: argparse.Namespace):
    from tencirpauli_b200 import PauliOperator, workloads

    codes, coeffs = workloads.random_k_local(n=args.nqubits, words=args.words, seed=args.seed)
    return PauliOperator.from_code_arrays(codes, coeffs)


def cpu_reference_rate(op, state_host: np.ndarray, seconds: float, threads: int = 0) -> Dict[str, Any]:
    """The C restatement of the reference's Rust/rayon TermDirect row loop
    (crates/tencir-pauli-core/src/hamiltonian.rs:204-270) on a random row
    sample sized to about ``seconds`` of CPU work."""
    from oracle import oracle

    n = op.nqubits
    xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
    rng = np.random.default_rng(1)
    cores = threads or oracle.max_threads()
    dim = 1 << n

    # Contiguous row blocks, as rayon's par_iter_mut walks rows in order.
    def block(count: int) -> np.ndarray:
        start = int(rng.integers(0, max(1, dim - count + 1)))
        return np.arange(start, start + count, dtype=np.uint64)

    probe = block(min(dim, 1 << 14))
    t0 = time.perf_counter()
    oracle.apply_rows(n, xm, zm, wp, state_host, probe, cores)
    dt = max(time.perf_counter() - t0, 1e-6)
    per_row = dt / probe.size
    rows = int(min(dim, max(probe.size, seconds / per_row)))
    sample = block(rows)
    t0 = time.perf_counter()
    oracle.apply_rows(n, xm, zm, wp, state_host, sample, cores)
    dt = time.perf_counter() - t0
    rate = op.term_count * rows / dt
    return {
        "value": rate,
        "unit": UNIT,
        "cores": cores,
        "kind": "port",
        "sample": f"{rows} consecutive rows of the 2^{n} state x {op.term_count} terms "
        f"(TermDirect row loop, {dt:.1f} s)",
        "seconds": dt,
    }


def _standalone_workloads():
    """``tencirpauli_b200/workloads.py`` loaded on its own (pure NumPy), so that
    the reference arm never imports the product package or maps its library."""
    import importlib.util

    path = os.path.join(ROOT, "tencirpauli_b200", "workloads.py")
    spec = importlib.util.spec_from_file_location("_tcp_bench_workloads", path)
    module = importlib.util.module_from_spec(spec)
    assert spec.loader is not None
    spec.loader.exec_module(module)
    return module


def run_reference(args: argparse.Namespace) -> None:
    """The reference's CPU algorithm on this host's cores: the C restatement
    of the Rust/rayon TermDirect row loop (crates/tencir-pauli-core/src/
    hamiltonian.rs:204-270; the Rust build is unavailable), on the same
    canonical operator and state as the GPU arm.  A step is the row loop over
    one block of ``2^reference_rows_log2`` consecutive rows (blocks walk the
    state in order), so ``ms_per_step`` x ``steps`` is the time this arm ran.
    The canonical term list comes from the oracle's restatement of
    PauliOperator::from_terms (operator.rs:117-155): nothing of the product
    is imported.  After the timed steps, one full TermDirect pass over the
    whole state is timed once and reported as ``full_pass_s``."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle

    wl = _standalone_workloads()
    n = args.nqubits
    codes, coeffs = wl.random_k_local(n=n, words=args.words, seed=args.seed)
    xw, zw, cf = oracle.canonicalize(n, codes, coeffs)
    xm, zm, wp = oracle.matrix_terms(n, xw, zw, cf)
    T = len(cf)
    dim = 1 << n
    rng = np.random.default_rng(args.seed)
    state = rng.standard_normal(dim) + 1j * rng.standard_normal(dim)
    state /= np.linalg.norm(state)
    cores = oracle.max_threads()
    rows_per_step = min(dim, 1 << args.reference_rows_log2)
    blocks = dim // rows_per_step
    block_rows = np.arange(rows_per_step, dtype=np.uint64)

    def step(i: int) -> float:
        rows = block_rows + np.uint64((i % blocks) * rows_per_step)
        t0 = time.perf_counter()
        oracle.apply_rows(n, xm, zm, wp, state, rows, cores)
        return time.perf_counter() - t0

    for i in range(args.warmup):
        step(i)
    times = [step(args.warmup + i) for i in range(args.steps)]
    seconds = float(sum(times))
    value = T * rows_per_step * args.steps / seconds
    full_pass_s = None
    if args.reference_full_pass:
        t0 = time.perf_counter()
        oracle.apply_term_direct(n, xm, zm, wp, state, cores)
        full_pass_s = time.perf_counter() - t0
    config = workload_config(args, None, terms=T)
    config["rows_per_step"] = rows_per_step
    sample = (f"{args.steps} blocks of {rows_per_step} consecutive rows of the 2^{n} state x {T} terms "
              f"(TermDirect row loop, {seconds:.1f} s); C restatement of the reference Rust MVP "
              "(Rust build unavailable)")
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 * seconds / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": config,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_pass_s": full_pass_s,
        "full_pass_amp_terms_per_s": (T * dim / full_pass_s) if full_pass_s else None,
        "manifest": manifest(with_gpu=False),
    }
    print(json.dumps(line), flush=True)


def workload_config(args: argparse.Namespace, op, terms: Optional[int] = None) -> Dict[str, Any]:
    return {
        "workload": f"random {args.words}-word 2..4-local Hamiltonian, n={args.nqubits}",
        "nqubits": args.nqubits,
        "raw_words": args.words,
        "terms": op.term_count if op is not None else terms,
        "seed": args.seed,
        "state": "complex128" if args.dtype == "c128" else "complex64",
        "vectors_per_step_per_gpu": 1,
        "l2": _l2_note(args.nqubits, 16 if args.dtype == "c128" else 8),
    }


def _l2_note(n: int, elem: int) -> str:
    vec = (1 << n) * elem
    if vec > 126 * 2**20:
        return f"inputs larger than L2 ({vec / 2**30:.2f} GiB per vector), no flush"
    return f"vector of {vec / 2**20:.1f} MiB fits in L2 (not flushed between steps)"


def run_batched(args: argparse.Namespace) -> None:
    """64 open 2D Heisenberg lattices (n uniform in 16..26, one J per bond),
    8 complex64 right-hand sides each, one persistent graph-launched kernel
    per step, tile shape and RHS block chosen by the autotuner."""
    import torch

    from tencirpauli_b200 import PauliOperator, workloads
    from tencirpauli_b200.batch import BatchedMVP

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    members = workloads.batched_heisenberg_set(args.batch_count, seed=args.seed, nmax=args.batch_nmax)
    ops = [PauliOperator.from_code_arrays(c, w) for _, c, w in members]
    plans = [op.native_mvp_plan() for op in ops]
    nrhs = args.batch_rhs
    dtype = torch.complex64
    xs = [workloads.random_state_device(op.nqubits, seed=args.seed + i, dtype=dtype, nrhs=nrhs) for i, op in enumerate(ops)]
    ys = [torch.empty_like(x) for x in xs]
    batch = BatchedMVP(plans, nrhs=nrhs, dtype="complex64")
    if args.batch_config:
        logt, rb = (int(v) for v in args.batch_config.split(","))
        batch.configure(logt, rb)
        tune = dict(batch.info(), fixed=True)
    else:
        cache = os.path.join(tempfile.gettempdir(), "tcp_batch_autotune.txt")
        tune = batch.autotune(xs, ys, cache_path=cache, repeats=2)
    ring = tune["tile_rows_log2"] == 12
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        batch.apply(xs, ys, stream)
    torch.cuda.synchronize()
    batch.device_status()
    sampler = ClockSampler(_smi_id(torch.cuda.current_device()))
    sampler.start()
    time.sleep(0.3)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        batch.apply(xs, ys, stream)
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    batch.device_status()
    ms = t0.elapsed_time(t1) / args.steps
    amp_terms = sum(op.term_count * (1 << op.nqubits) * nrhs for op in ops)
    state_bytes = sum((1 << op.nqubits) * nrhs * 8 for op in ops)
    peaks = _measured_peaks()
    achieved = 2 * state_bytes / (ms / 1000.0) / 1e9
    # Both batched kernels read one 8-byte complex64 operand per (row, x-mask
    # group, right-hand side) from shared memory (the ring kernel once per
    # coset of groups, so slightly less): the binding ceiling is the
    # shared-memory rate, probed on this GPU.
    from tencirpauli_b200 import _native as native_mod

    smem_rate, _ = native_mod.probe_smem_rate()
    fma_rate, _ = native_mod.probe_fma_rate("complex64")
    smem_bytes = sum((1 << op.nqubits) * nrhs * plan.group_count * 8 for op, plan in zip(ops, plans))
    flops = sum((1 << op.nqubits) * nrhs * (2 * op.term_count + 8 * plan.group_count) for op, plan in zip(ops, plans))
    smem_ach = smem_bytes / (ms / 1000.0)
    # accuracy: one RHS of the largest and the smallest member against the oracle rows
    from oracle import oracle

    errs = []
    for idx in (max(range(len(ops)), key=lambda i: ops[i].nqubits), min(range(len(ops)), key=lambda i: ops[i].nqubits)):
        op = ops[idx]
        rows = np.sort(np.random.default_rng(5).choice(1 << op.nqubits, size=1024, replace=False)).astype(np.uint64)
        xm, zm, wp = oracle.matrix_terms(op.nqubits, op.x_words, op.z_words, op.coefficients)
        ref = oracle.apply_rows(op.nqubits, xm, zm, wp, xs[idx][nrhs - 1].cpu().numpy().astype(np.complex128), rows)
        got = ys[idx][nrhs - 1][torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
        errs.append(float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
    smem_roofline = {
        "bound": "smem",
        "achieved": smem_ach / 1e12,
        "peak": smem_rate / 1e12,
        "unit": "TB/s",
        "frac": smem_ach / smem_rate,
        "traffic": None,
        "peak_source": "tcp_probe_smem_rate on this GPU, best of 5",
        "kernel": "k_ring (one launch per member, blockIdx.y = RHS)" if ring else "k_batched",
        "smem_bytes_per_launch": smem_bytes,
        "fp": {"achieved": flops / (ms / 1000.0) / 1e12, "peak": fma_rate / 1e12, "unit": "TFLOP/s",
               "frac": flops / (ms / 1000.0) / fma_rate},
        "hbm": {"achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                "peak_source": peaks["source"]},
    }
    # The ring configuration is bound by instruction issue, as the
    # single-vector kernel: its committed instruction count per apply (the
    # 64 member launches) leads, shared memory, the FMA pipe and HBM beside it.
    issue = (_issue_roofline("k_ring<float,rhs_block>", f"heisenberg{args.batch_count}_nmax{args.batch_nmax}_rhs{nrhs}_seed{args.seed}", ms,
                             clocks) if ring else None)
    if issue is not None:
        batch_roofline = {"bound": "issue", **{k: issue[k] for k in ("achieved", "peak", "unit", "frac")}, "traffic": None,
                          "kernel": smem_roofline["kernel"], "instructions_per_apply": issue["instructions_per_launch"],
                          "peak_source": "4 warp instructions per SM clock x SMs x sampled SM clock; " + issue["source"],
                          "smem": {k: v for k, v in smem_roofline.items() if k not in ("bound", "fp", "hbm", "kernel")},
                          "fp": smem_roofline["fp"], "hbm": smem_roofline["hbm"]}
    else:
        batch_roofline = smem_roofline
    line = {
        "metric": METRIC,
        "value": amp_terms / (ms / 1000.0),
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {
            "workload": f"batched: {len(ops)} open 2D Heisenberg lattices, n in 16..26, {nrhs} complex64 RHS each",
            "qubits": sorted(op.nqubits for op in ops),
            "terms_total": sum(op.term_count for op in ops),
            "state_bytes": state_bytes,
            "autotuned": tune,
            "l2": "inputs larger than L2, no flush",
        },
        "roofline": batch_roofline,
        "e2e": None,
        "gpu_launches": args.steps * (tune["grid"] if ring else 1),
        "clocks": clocks,
        "accuracy": {"rel_err_vs_oracle_rows": errs},
    }
    print(json.dumps(line), flush=True)


def run_davidson(args: argparse.Namespace) -> None:
    """Lowest 4 eigenpairs of the periodic 4x6 J1-J2 model (J1 = 1, J2 = 0.5)
    to an exact FP64-MVP residual of 1e-8: plain (Jacobi) Davidson against
    the learned-preconditioned one, same GPU, same start, same precision
    schedule (complex64 MVP, then FP64)."""
    import torch

    from tencirpauli_b200 import PauliOperator, precond, workloads
    from tencirpauli_b200.davidson import JacobiPreconditioner, davidson

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    op = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(4, 6, 1.0, 0.5))
    plan = op.native_mvp_plan()
    weights = args.weights or precond.DEFAULT_WEIGHTS
    trained_info = None
    if args.train or not os.path.exists(weights):
        t0 = time.perf_counter()
        params, info = precond.train_from_lattices(precond.training_lattices(6, seed=0), steps=800)
        trained_info = {"seconds": time.perf_counter() - t0, "samples": info["samples"], "final_loss": info["losses"][-1]}
    else:
        params = precond.MLPPreconditioner.load(weights, scale=1.0).params.cpu().numpy()
    scale = precond.energy_scale(op)
    small = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(4, 4, 1.0, 0.5)).native_mvp_plan()
    davidson(small, nev=4, tol=1e-8, seed=0)  # warm-up: kernel loading, allocator
    davidson(small, nev=4, tol=1e-8, seed=0, preconditioner=precond.MLPPreconditioner(params, scale=scale))
    runs = {}
    for name in ("jacobi", "learned"):
        pc = JacobiPreconditioner() if name == "jacobi" else precond.MLPPreconditioner(params, scale=scale)
        torch.cuda.synchronize()
        res = davidson(plan, nev=4, tol=1e-8, seed=args.seed % 1000, preconditioner=pc, max_iter=args.davidson_max_iter)
        runs[name] = {
            "seconds": res.seconds,
            "iterations": res.iterations,
            "phase_iterations": res.phase_iterations,
            "mvps": res.mvps,
            "converged": res.converged,
            "eigenvalues": [float(v) for v in res.eigenvalues],
            "residuals": [float(v) for v in res.residuals],
            "fallbacks": res.fallbacks,
        }
    # the same solve inside the half-filling U(1) sector (the ground state and
    # the low singlets of the even lattice live there): 6x fewer amplitudes
    from tencirpauli_b200 import U1Sector

    sector_plan = op.restrict_charge(U1Sector(op.nqubits, op.nqubits // 2)).mvp_plan()
    torch.cuda.synchronize()
    sres = davidson(sector_plan, nev=4, tol=1e-8, seed=args.seed % 1000, max_iter=args.davidson_max_iter)
    runs["jacobi_half_filling_sector"] = {
        "seconds": sres.seconds,
        "iterations": sres.iterations,
        "mvps": sres.mvps,
        "converged": sres.converged,
        "dimension": sector_plan.dimension,
        "eigenvalues": [float(v) for v in sres.eigenvalues],
        "max_abs_diff_vs_full_space": float(max(abs(a - b) for a, b in zip(sres.eigenvalues, runs["jacobi"]["eigenvalues"]))),
    }
    line = {
        "metric": "Davidson wall time to residual 1e-8 (lowest 4 eigenpairs)",
        "value": runs["learned"]["seconds"],
        "unit": "s",
        "higher_is_better": False,
        "n_gpus": 1,
        "dtype": "c64 MVP + f64 polish",
        "data": "synthetic",
        "config": {"workload": "4x6 periodic J1-J2 Heisenberg, J1=1, J2=0.5, 24 qubits", "terms": op.term_count},
        "learned_over_plain_time": runs["learned"]["seconds"] / runs["jacobi"]["seconds"],
        "runs": runs,
        "training": trained_info,
    }
    print(json.dumps(line), flush=True)


def run_chemistry(args: argparse.Namespace) -> None:
    """Jordan-Wigner chemistry-like Hamiltonian on n spin-orbitals (random
    integrals, see tencirpauli_b200.mapping.chemistry_integrals): one FP64
    complex128 MVP, one complex64 MVP and one 16-RHS complex64 block through
    the batched kernel; exact rows against the oracle."""
    import torch

    from tencirpauli_b200 import PauliOperator, workloads
    from tencirpauli_b200.batch import BatchedMVP
    from tencirpauli_b200.mapping import chemistry_integrals, jordan_wigner_integrals

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.nqubits
    t0 = time.perf_counter()
    h, g = chemistry_integrals(n, seed=args.seed)
    op = PauliOperator.from_code_arrays(*jordan_wigner_integrals(h, g))
    build_s = time.perf_counter() - t0
    plan = op.native_mvp_plan()
    res = {}
    from oracle import oracle

    rows = np.sort(np.random.default_rng(7).choice(1 << n, size=512, replace=False)).astype(np.uint64)
    xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
    for dt, name in ((torch.complex128, "c128"), (torch.complex64, "c64")):
        x = workloads.random_state_device(n, seed=args.seed, dtype=dt)
        y = torch.empty_like(x)
        plan.apply_device(x, y)  # warm-up
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps):
            plan.apply_device(x, y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        ref = oracle.apply_rows(n, xm, zm, wp, x.cpu().numpy().astype(np.complex128), rows)
        got = y[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
        res[name] = {"ms": ms, "amp_terms_per_s": op.term_count * (1 << n) / (ms / 1e3),
                     "rel_err_rows": float(np.linalg.norm(got - ref) / np.linalg.norm(ref))}
        del x, y
    nrhs = args.chem_block_rhs
    if nrhs <= 0:
        print(json.dumps({"workload": f"Jordan-Wigner chemistry-like Hamiltonian, n={n}", "terms": op.term_count,
                          "groups": plan.group_count, "host_build_s": build_s, "results": res}), flush=True)
        return
    xs = [workloads.random_state_device(n, seed=args.seed + 1, dtype=torch.complex64, nrhs=nrhs)]
    ys = [torch.empty_like(xs[0])]
    batch = BatchedMVP([plan], nrhs=nrhs, dtype="complex64")
    batch.configure(9, 8)
    batch.apply(xs, ys)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    batch.apply(xs, ys)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ref = oracle.apply_rows(n, xm, zm, wp, xs[0][5].cpu().numpy().astype(np.complex128), rows)
    got = ys[0][5][torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
    res["c64_16rhs"] = {"ms": ms, "amp_terms_per_s": op.term_count * (1 << n) * nrhs / (ms / 1e3),
                        "rel_err_rows": float(np.linalg.norm(got - ref) / np.linalg.norm(ref))}
    print(json.dumps({"workload": f"Jordan-Wigner chemistry-like Hamiltonian, n={n}", "terms": op.term_count,
                      "groups": plan.group_count, "host_build_s": build_s, "results": res}), flush=True)


def run_sector(args: argparse.Namespace) -> None:
    """Restricted MVP in the half-filling U(1) sector of the periodic J1-J2
    model (J1 = 1, J2 = 0.5) on ``--lattice`` (default 4x7: n = 28, k = 14,
    dimension C(28, 14) = 40,116,600).  A step is one y = H x over the whole restricted state.
    Metric: restricted amplitude-terms/s = T_canonical * dimension / step
    time.  ``e2e`` runs the host C-ABI apply (pinned buffers, H2D + kernel +
    D2H); ``cpu_baseline`` pulls a bounded sample of rows with the oracle."""
    import torch

    from tencirpauli_b200 import PauliOperator, U1Sector, workloads

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    lx, ly = (int(v) for v in args.lattice.lower().split("x"))
    n, k = lx * ly, (lx * ly) // 2
    op = PauliOperator.from_code_arrays(*workloads.j1j2_periodic(lx, ly, 1.0, 0.5))
    t0 = time.perf_counter()
    plan = op.restrict_charge(U1Sector(n, k)).mvp_plan()
    build_s = time.perf_counter() - t0
    native = plan._native_plan
    dim, T = plan.dimension, op.term_count
    cdtype = torch.complex128 if args.dtype == "c128" else torch.complex64
    elem = 16 if args.dtype == "c128" else 8
    x = workloads.random_state_device(n, seed=args.seed, dtype=cdtype, length=dim)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        plan.apply_device(x, y, stream)
    torch.cuda.synchronize()
    sampler = ClockSampler(_smi_id(torch.cuda.current_device()))
    sampler.start()
    time.sleep(0.3)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for i in range(args.steps):
        starts[i].record(stream)
        plan.apply_device(x, y, stream)
        ends[i].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    native.device_status()
    times = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    ms = statistics.mean(times)
    value = T * dim / (ms / 1e3)
    # end to end through the host C ABI (pinned host buffers)
    x_host = torch.empty(dim, dtype=torch.complex128, pin_memory=True)
    y_host = torch.empty(dim, dtype=torch.complex128, pin_memory=True)
    x_host.copy_(x.to(torch.complex128))
    xh, yh = x_host.numpy(), y_host.numpy()
    native.apply_into(xh, yh, 2**63 - 1)
    e2e = []
    for _ in range(args.e2e_steps):
        t1 = time.perf_counter()
        native.apply_into(xh, yh, 2**63 - 1)
        e2e.append(time.perf_counter() - t1)
    e2e_s = statistics.median(e2e)
    # accuracy on a row sample and the CPU baseline (oracle, all host cores)
    from oracle import oracle

    rng = np.random.default_rng(3)
    rows = np.sort(rng.choice(dim, size=4096, replace=False)).astype(np.uint64)
    ref = oracle.u1_apply_rows(n, k, op.x_words, op.z_words, op.coefficients, xh, rows)
    if args.dtype == "c128":
        got = yh[rows.astype(np.int64)]
    else:
        got = y[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
    cpu = None
    if not args.no_cpu_baseline:
        probe = np.arange(0, 20000, dtype=np.uint64)
        t1 = time.perf_counter()
        oracle.u1_apply_rows(n, k, op.x_words, op.z_words, op.coefficients, xh, probe)
        per_row = (time.perf_counter() - t1) / probe.size
        count = int(min(dim, max(probe.size, args.cpu_seconds / per_row)))
        sample = np.arange(0, count, dtype=np.uint64)
        t1 = time.perf_counter()
        oracle.u1_apply_rows(n, k, op.x_words, op.z_words, op.coefficients, xh, sample)
        dt = time.perf_counter() - t1
        cpu = {"value": T * count / dt, "unit": UNIT, "cores": oracle.max_threads(), "kind": "port",
               "sample": f"{count} consecutive sector rows x {T} terms pulled by the oracle ({dt:.1f} s)"}
    peaks = _measured_peaks()
    b_alg = dim * (4 + 16 + 2 * elem)  # basis word, diagonal, x, y
    achieved = b_alg / (ms / 1e3) / 1e9
    # k_u1_apply is bound by instruction issue (gathers and table lookups
    # in flight, not bytes): its roofline is the issue rate, with the
    # compulsory HBM bytes beside it
    hbm = {"achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
           "bytes_per_launch": b_alg, "peak_source": peaks["source"]}
    issue = _issue_roofline("k_u1_apply", f"j1j2_{lx}x{ly}_half_{args.dtype}", ms, clocks)
    if issue is not None:
        sector_roofline = dict(bound="issue", **{k: issue[k] for k in ("achieved", "peak", "unit", "frac")},
                               kernel="k_u1_apply", kernel_ms=ms, instructions_per_launch=issue["instructions_per_launch"],
                               peak_source="4 warp instructions per SM clock x SMs x sampled SM clock; "
                               + issue["source"], hbm=hbm)
    else:
        sector_roofline = dict(bound="issue (instruction count not profiled for this lattice; HBM shown)",
                               **{k: hbm[k] for k in ("achieved", "peak", "unit", "frac")}, kernel="k_u1_apply",
                               kernel_ms=ms, bytes_per_launch=b_alg, peak_source=peaks["source"])
    line = {
        "metric": "Sector MVP amplitude-terms/s",
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.dtype == "c128" else "f32",
        "data": "synthetic",
        "config": {"workload": f"periodic {lx}x{ly} J1-J2 (J1=1, J2=0.5), half-filling U(1) sector", "nqubits": n,
                   "particle_number": k, "dimension": dim, "terms": T, "groups": native.group_count,
                   "l2": f"restricted state {dim * 16 / 1e6:.0f} MB" + ("; > L2, no flush needed" if dim * 16 > 126e6 else "; fits in L2")},
        "roofline": sector_roofline,
        "e2e": {"value": T * dim / e2e_s, "unit": UNIT, "h2d_bytes_per_step": dim * 16, "d2h_bytes_per_step": dim * 16,
                "ms_per_step": 1e3 * e2e_s},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "accuracy": {"rows_checked": int(rows.size),
                     "rel_err_vs_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref))},
        "plan_build_s": build_s,
    }
    print(json.dumps(line), flush=True)


def run_solver(args: argparse.Namespace) -> None:
    """The two vector kernels of the Davidson solver at its sizes: the FP64
    Gram C = V^H T and the update T -= V C of block Gram-Schmidt, for a
    64-vector basis V and a 4-vector block T of length n (2^24 for the 4x6
    lattice), in complex128 and complex64 storage.  Bandwidth counts the
    algorithmic bytes of one launch: Gram reads V and T; the update reads V
    and T and writes T.  V alone (64 vectors) exceeds L2, so no flush is
    needed between launches."""
    import torch

    from tencirpauli_b200 import solver_ops

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, p, q = args.solver_n, 64, 4
    peaks = _measured_peaks()
    results = {}
    for name in (["c128", "c64"] if args.solver_dtype == "both" else [args.solver_dtype]):
        dtype = torch.complex128 if name == "c128" else torch.complex64
        es = 16 if name == "c128" else 8
        g = torch.Generator(device="cuda")
        g.manual_seed(args.seed % 1000)
        V = torch.randn((p, n), dtype=dtype, device="cuda", generator=g)
        T = torch.randn((q, n), dtype=dtype, device="cuda", generator=g)
        C = solver_ops.gram(V, T)
        for _ in range(args.warmup):
            solver_ops.gram(V, T)
            solver_ops.combine(V, C, T, alpha=-1.0, beta=1.0)
        torch.cuda.synchronize()
        times = {}
        for op in ("gram", "combine"):
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
            for _ in range(args.steps):
                if op == "gram":
                    solver_ops.gram(V, T)
                else:
                    solver_ops.combine(V, C, T, alpha=-1.0, beta=1.0)
            end.record()
            torch.cuda.synchronize()
            times[op] = start.elapsed_time(end) / args.steps
        gram_bytes = (p + q) * n * es
        comb_bytes = (p + 2 * q) * n * es
        results[name] = {
            "gram_ms": times["gram"], "gram_gbs": gram_bytes / times["gram"] / 1e6,
            "combine_ms": times["combine"], "combine_gbs": comb_bytes / times["combine"] / 1e6,
            "gram_bytes": gram_bytes, "combine_bytes": comb_bytes,
        }
        del V, T
        torch.cuda.empty_cache()
    first = next(iter(results.values()))
    print(json.dumps({
        "metric": "Davidson Gram / block-combine bandwidth", "value": first["gram_gbs"], "unit": "GB/s",
        "higher_is_better": True, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "data": "synthetic",
        "config": {"workload": f"basis of {p} vectors x block of {q}, length {n}", "l2": "inputs larger than L2"},
        "peak_hbm_gbs": peaks["hbm_gbs"], "peak_source": peaks["source"], "results": results,
    }), flush=True)


def run_sharded(args: argparse.Namespace, world: int, rank: int) -> None:
    """The state-sharded MVP (tencirpauli_b200/sharded.py) on ``world`` GPUs
    over NCCL: the same n = ``--nqubits`` workload split by its top log2(world)
    index bits, one shard per rank (strong scaling: total work fixed).  A step
    is one y = H x over the whole state: the local apply plus one pairwise
    shard exchange per top-bit pattern, each partner's contribution added into
    y by the kernel; exchanges are double-buffered so they overlap the applies.
    The step time is the max over ranks of the CUDA-event time."""
    import datetime

    import torch
    import torch.distributed as dist

    from tencirpauli_b200 import workloads
    from tencirpauli_b200.sharded import ShardedMVP

    if world & (world - 1):
        raise SystemExit("the sharded MVP needs a power-of-two number of GPUs")
    op = build_operator(args)
    n, T, dim = op.nqubits, op.term_count, 1 << op.nqubits
    mvp = ShardedMVP(op, timeout_s=120.0)
    cdtype = torch.complex128 if args.dtype == "c128" else torch.complex64
    elem = 16 if args.dtype == "c128" else 8
    x = workloads.random_state_device(mvp.local_qubits, seed=args.seed + rank, dtype=cdtype)
    y = torch.empty_like(x)
    bufs = mvp.receive_buffers(x)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        mvp.apply(x, y, bufs)
    torch.cuda.synchronize()
    dist.barrier()
    sampler = ClockSampler(_smi_id(torch.cuda.current_device()))
    sampler.start()
    time.sleep(0.3)
    t_begin, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize()
    t_begin.record(stream)
    for _ in range(args.steps):
        mvp.apply(x, y, bufs)
    t_end.record(stream)
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    for plan in mvp._plans.values():
        plan._native_plan.device_status()
    ms = torch.tensor([t_begin.elapsed_time(t_end) / args.steps], device="cuda", dtype=torch.float64)
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_per_step = float(ms.item())
    value = T * dim / (ms_per_step / 1e3)
    # end to end: each rank's shard from page-locked host memory, the sharded
    # apply, the shard of y back to the host; max over ranks
    xh = torch.empty(mvp.shard_len, dtype=cdtype, pin_memory=True)
    yh = torch.empty(mvp.shard_len, dtype=cdtype, pin_memory=True)
    xh.copy_(x)
    xd = torch.empty_like(x)
    e2e = []
    for _ in range(max(1, args.e2e_steps)):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xd.copy_(xh, non_blocking=True)
        mvp.apply(xd, y, bufs)
        yh.copy_(y, non_blocking=True)
        torch.cuda.synchronize()
        e2e.append(time.perf_counter() - t0)
    e2e_t = torch.tensor([statistics.median(e2e)], device="cuda", dtype=torch.float64)
    dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    # size-independent check: <a, H b> == <H a, b> across all shards
    a = workloads.random_state_device(mvp.local_qubits, seed=args.seed + 1000 + rank, dtype=cdtype)
    ha = torch.empty_like(a)
    mvp.apply(a, ha, bufs)
    mvp.apply(x, y, bufs)
    dots = torch.stack([torch.vdot(a, y), torch.vdot(ha, x)]).to(torch.complex128)
    dist.all_reduce(dots)
    herm = abs(complex(dots[0]) - complex(dots[1])) / max(abs(complex(dots[0])), 1e-300)
    # Ceilings of one step per rank: instruction issue for the applies (the
    # single-GPU launch's committed instruction count split evenly over the
    # ranks, an estimate: the per-pattern plans are not the full plan) and
    # NVLink for the exchanges (one shard per nonzero top pattern received,
    # against the 770 GB/s per direction measured for a peer copy on this
    # pool).  The step time covers both, so both achieved rates are lower
    # bounds.
    step_s = ms_per_step / 1000.0
    recv_bytes = len(mvp.patterns) * mvp.shard_len * elem
    nvlink = {"achieved": recv_bytes / step_s / 1e9, "peak": 770.0, "unit": "GB/s",
              "frac": recv_bytes / step_s / 770e9, "bytes_per_rank_per_step": recv_bytes,
              "peak_source": "peer copy measured on this pool, per direction"}
    kernel_name = "k_ring<double>" if args.dtype == "c128" else "k_ring<float>"
    issue = _issue_roofline(kernel_name, f"random{args.words}_n{n}", ms_per_step * world, clocks)
    if issue is not None:
        roofline = {"bound": "issue (estimated per rank)", **{k: issue[k] for k in ("achieved", "peak", "unit", "frac")},
                    "traffic": None, "kernel": kernel_name,
                    "note": "instructions of the single-GPU launch / ranks over the step time", "nvlink": nvlink}
    else:
        roofline = {"bound": "nvlink", **{k: nvlink[k] for k in ("achieved", "peak", "unit", "frac")}, "traffic": None,
                    "kernel": kernel_name}
    line = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64" if args.dtype == "c128" else "f32",
        "data": "synthetic",
        "config": dict(workload_config(args, op), parallelism=f"state sharded over {world} GPUs by the top "
                       f"{world.bit_length() - 1} index bits", shard_amplitudes=mvp.shard_len,
                       exchange_patterns=len(mvp.patterns)),
        "e2e": {"value": T * dim / float(e2e_t.item()), "unit": UNIT, "h2d_bytes_per_step": dim * elem,
                "d2h_bytes_per_step": dim * elem, "ms_per_step": 1e3 * float(e2e_t.item()),
                "note": "bytes summed over ranks; each rank copies its own shard"},
        "gpu_launches": args.steps * (len(mvp.patterns) + 1),
        "roofline": roofline,
        "clocks": clocks,
        "accuracy": {"hermiticity_rel": herm},
        "manifest": manifest(),
    }
    for b in bufs:
        del b
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--weights", default=None)
    parser.add_argument("--train", action="store_true")
    parser.add_argument("--davidson-max-iter", type=int, default=600)
    parser.add_argument("--workload", choices=["random28", "batched", "davidson", "chemistry", "sector", "solver"],
                        default="random28")
    parser.add_argument("--solver-n", type=int, default=1 << 24, help="solver workload: vector length")
    parser.add_argument("--solver-dtype", choices=["both", "c128", "c64"], default="both")
    parser.add_argument("--batch-count", type=int, default=64)
    parser.add_argument("--lattice", default="4x7", help="sector workload: periodic J1-J2 lattice LXxLY")
    parser.add_argument("--batch-rhs", type=int, default=8)
    parser.add_argument("--chem-block-rhs", type=int, default=16,
                        help="chemistry workload: right-hand sides of the batched complex64 block (0: skip it)")
    parser.add_argument("--batch-nmax", type=int, default=26, help="batched workload: largest member size")
    parser.add_argument("--batch-config", default=None,
                        help="batched workload: fixed 'tile_rows_log2,rhs_block' instead of the autotuner "
                             "(12,1 = one ring-kernel launch per member)")
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=10)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--nqubits", type=int, default=28)
    parser.add_argument("--words", type=int, default=2000)
    parser.add_argument("--seed", type=int, default=20261203)
    parser.add_argument("--dtype", choices=["c128", "c64"], default="c128")
    parser.add_argument("--e2e-steps", type=int, default=3)
    parser.add_argument("--cpu-seconds", type=float, default=15.0)
    parser.add_argument("--reference-rows-log2", type=int, default=22,
                        help="reference arm: rows per step (log2) of the TermDirect row loop")
    parser.add_argument("--reference-full-pass", type=int, default=1,
                        help="reference arm: also time one full pass over the state (1) or not (0)")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--replicas", action="store_true",
                        help="with several GPUs: one independent state per GPU instead of one sharded state")
    args = parser.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "davidson":
        run_davidson(args)
        return
    if args.workload == "chemistry":
        run_chemistry(args)
        return
    if args.workload == "sector":
        run_sector(args)
        return
    if args.workload == "solver":
        run_solver(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        if not args.replicas:
            run_sharded(args, world, rank)
            return

    from tencirpauli_b200 import workloads

    op = build_operator(args)
    plan = op.native_mvp_plan()
    n = op.nqubits
    T = op.term_count
    dim = 1 << n
    cdtype = torch.complex128 if args.dtype == "c128" else torch.complex64
    elem = 16 if args.dtype == "c128" else 8
    x = workloads.random_state_device(n, seed=args.seed + rank, dtype=cdtype)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        plan.apply_device(x, y, stream)
    torch.cuda.synchronize()
    plan._native_plan.device_status()

    sampler = ClockSampler(_smi_id(torch.cuda.current_device()))
    sampler.start()
    time.sleep(0.3)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_begin = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_begin.record(stream)
    for k in range(args.steps):
        starts[k].record(stream)
        plan.apply_device(x, y, stream)
        ends[k].record(stream)
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    plan._native_plan.device_status()
    total_ms = t_begin.elapsed_time(t_end)
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms_local = total_ms / args.steps
    ms_tensor = torch.tensor([ms_local], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_tensor, op=dist.ReduceOp.MAX)
    ms_per_step = float(ms_tensor.item())
    amp_terms = T * dim
    value = amp_terms * world / (ms_per_step / 1000.0)

    # end to end through the public host apply_into: ordinary NumPy buffers
    # (what the reference's facade passes) for the headline, page-locked
    # buffers beside it
    x_host = torch.empty(dim, dtype=cdtype, pin_memory=True)
    y_host = torch.empty(dim, dtype=cdtype, pin_memory=True)
    x_host.copy_(x)
    native = plan._native_plan

    def host_apply(xh: np.ndarray, yh: np.ndarray) -> None:
        if args.dtype == "c128":
            native.apply_into(xh, yh, 2**63 - 1)
        else:
            native.apply_c64_into(xh, yh)

    def e2e_time(xh: np.ndarray, yh: np.ndarray) -> float:
        host_apply(xh, yh)
        times = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            host_apply(xh, yh)
            times.append(time.perf_counter() - t0)
        t = torch.tensor([statistics.median(times)], device="cuda", dtype=torch.float64)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    x_page = np.array(x_host.numpy(), copy=True)
    y_page = np.empty_like(x_page)
    e2e_pageable_s = e2e_time(x_page, y_page)
    e2e_pinned_s = e2e_time(x_host.numpy(), y_host.numpy())
    del x_page, y_page
    e2e_value = amp_terms * world / e2e_pageable_s

    # accuracy of this run's result on a row sample (rank 0), vs the oracle
    line: Dict[str, Any] = {}
    if rank == 0:
        peaks = _measured_peaks()
        kern_ms = statistics.mean(kernel_ms)
        b_alg = dim * 2 * elem
        achieved = b_alg / (kern_ms / 1000.0) / 1e9
        kernel_name = "k_ring<double>" if args.dtype == "c128" else "k_ring<float>"
        traffic = _profile_traffic(kernel_name)
        # Ceilings of k_ring.  Binding: shared-memory operand delivery -- per
        # output row one operand per coset (groups whose inner masks agree on
        # the thread bits share it) read by the consumer warps, plus one value
        # per ring step written by the TMA engine -- against the device's own
        # shared-memory rate.  Beside it: the FMA pipe, F_alg = 2^n (2T + 8G)
        # real flops (the +-w_k sums into D_m once per amplitude, one complex
        # multiply-add per group), and HBM (read x once, write y once).
        from tencirpauli_b200 import _native as native_mod

        fma_rate, _ = native_mod.probe_fma_rate("complex128" if args.dtype == "c128" else "complex64")
        smem_rate, _ = native_mod.probe_smem_rate()
        G = plan.group_count
        info = native.info
        f_alg = dim * (2 * T + 8 * G)
        f_ach = f_alg / (kern_ms / 1000.0)
        smem_bytes = dim * (int(info.cosets) + int(info.ring_steps)) * elem
        smem_ach = smem_bytes / (kern_ms / 1000.0)
        # The binding resource is instruction issue (the per-record integer
        # chain ahead of the multiply-adds; ncu: issue active about half the
        # cycles, neither the shared-memory nor the FMA pipe saturated), so
        # the main roofline is the issue rate; shared memory, the FMA pipe
        # and HBM are reported beside it.
        smem_obj = {
            "achieved": smem_ach / 1e12,
            "peak": smem_rate / 1e12,
            "unit": "TB/s",
            "frac": smem_ach / smem_rate,
            "peak_source": "tcp_probe_smem_rate: 16-byte shared-memory reads in the kernel's pattern on every SM "
            "of this GPU, best of 5",
            "bytes_per_launch": smem_bytes,
            "units": f"2^{n} rows x ({int(info.cosets)} coset operands + {int(info.ring_steps)} tile fills) x {elem} B",
        }
        fp_obj = {
            "achieved": f_ach / 1e12,
            "peak": fma_rate / 1e12,
            "unit": "TFLOP/s",
            "frac": f_ach / fma_rate,
            "flops_per_launch": f_alg,
            "peak_source": "tcp_probe_fma_rate: FMA chains on every SM of this GPU, best of 5",
        }
        hbm_obj = {
            "achieved": achieved,
            "peak": peaks["hbm_gbs"],
            "unit": "GB/s",
            "frac": achieved / peaks["hbm_gbs"],
            "bytes_per_launch": b_alg,
            "peak_source": peaks["source"],
            "traffic_gbs": (traffic / (kern_ms / 1000.0) / 1e9) if traffic else None,
        }
        issue_obj = _issue_roofline(kernel_name, f"random{args.words}_n{n}", kern_ms, clocks)
        if issue_obj is not None:
            ring_roofline = {"bound": "issue", **{k: issue_obj[k] for k in ("achieved", "peak", "unit", "frac")},
                             "traffic": traffic, "kernel": kernel_name, "kernel_ms": kern_ms,
                             "instructions_per_launch": issue_obj["instructions_per_launch"],
                             "peak_source": "4 warp instructions per SM clock x SMs x sampled SM clock; " + issue_obj["source"],
                             "smem": smem_obj, "fp": fp_obj, "hbm": hbm_obj}
        else:  # no committed instruction count for this workload: shared memory leads
            ring_roofline = {"bound": "smem", **{k: smem_obj[k] for k in ("achieved", "peak", "unit", "frac")},
                             "traffic": traffic, "kernel": kernel_name, "kernel_ms": kern_ms,
                             "peak_source": smem_obj["peak_source"], "smem_bytes_per_launch": smem_bytes,
                             "fp": fp_obj, "hbm": hbm_obj}
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_per_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.dtype == "c128" else "f32",
            "data": "synthetic",
            "config": workload_config(args, op),
            "roofline": ring_roofline,
            "e2e": {
                "value": e2e_value,
                "unit": UNIT,
                "h2d_bytes_per_step": dim * elem,
                "d2h_bytes_per_step": dim * elem,
                "ms_per_step": 1000.0 * e2e_pageable_s,
                "host_buffers": "ordinary (pageable) NumPy arrays",
                "pinned": {"value": amp_terms * world / e2e_pinned_s, "ms_per_step": 1000.0 * e2e_pinned_s,
                           "host_buffers": "page-locked"},
            },
            "gpu_launches": args.steps,
            "clocks": clocks,
            "manifest": manifest(),
            "plan": {
                "groups": plan.group_count,
                "tile_bits": int(native.info.tile_bits),
                "ring_steps": int(native.info.ring_steps),
                "cosets": int(native.info.cosets),
                "outer_patterns": int(native.info.outer_patterns),
            },
        }
        if world == 1 and not args.no_cpu_baseline:
            state_host = x_host.numpy() if args.dtype == "c128" else x_host.numpy().astype(np.complex128)
            cb = cpu_reference_rate(op, state_host, seconds=args.cpu_seconds)
            cb.pop("seconds", None)
            line["cpu_baseline"] = cb
        # row-sample accuracy against the oracle (the checker)
        from oracle import oracle

        rows = np.sort(np.random.default_rng(3).choice(dim, size=2048, replace=False)).astype(np.uint64)
        xm, zm, wp = oracle.matrix_terms(n, op.x_words, op.z_words, op.coefficients)
        state_host = x_host.numpy().astype(np.complex128)
        ref = oracle.apply_rows(n, xm, zm, wp, state_host, rows)
        got = y[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy().astype(np.complex128)
        line["accuracy"] = {
            "rows_checked": int(rows.size),
            "rel_err_vs_oracle": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
        }
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
