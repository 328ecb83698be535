"""Compile ``libtcpmvp.so`` in-tree for sm_100a with nvcc.

The library is a plain C-ABI shared object (no torch or Python inside); it is
written to ``tencirpauli_b200/_lib/libtcpmvp.so`` so that it travels with the
source tree.  Run ``python -m tencirpauli_b200.build`` or call :func:`build`.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBPATH = os.path.join(LIBDIR, "libtcpmvp.so")
SOURCES = ["tcp_plan.cpp", "tcp_mvp.cu", "tcp_batched.cu", "tcp_solver.cu", "tcp_sector.cu", "tcp_probe.cu", "tcp_matrix.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if candidate and os.path.exists(candidate):
            return candidate
    raise RuntimeError("nvcc not found")


def _host_compiler() -> List[str]:
    # nvcc needs a host g++ whose OpenMP/libstdc++ runtime exists on this image.
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if os.path.exists(gxx) else []


DEBUG_LIBPATH = os.path.join(LIBDIR, "libtcpmvp_debug.so")


def build(verbose: bool = False, ptxas_verbose: bool = False, debug_bounds: bool = False) -> str:
    """Compile the library.  ``debug_bounds`` builds ``libtcpmvp_debug.so``
    with TCP_DEBUG_BOUNDS: the hot kernel checks every plan block against its
    shared-memory stage before walking it and reports a failed check as
    TCP_ERR_INVALID_ARGUMENT instead of reading outside the stage.  Select it
    at run time with TCP_LIBRARY=debug."""
    os.makedirs(LIBDIR, exist_ok=True)
    target = DEBUG_LIBPATH if debug_bounds else LIBPATH
    cmd = [
        nvcc(),
        *ARCH,
        *_host_compiler(),
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-shared",
        "-Xcompiler",
        "-fPIC,-O3",
        "--expt-relaxed-constexpr",
        "-o",
        target + ".tmp",
    ]
    if debug_bounds:
        cmd += ["-DTCP_DEBUG_BOUNDS"]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{proc.stdout}\n{proc.stderr}")
    if ptxas_verbose or verbose:
        sys.stdout.write(proc.stdout + proc.stderr)
    os.replace(target + ".tmp", target)
    if not debug_bounds:
        _write_build_info()
    return target


def _git(*args: str) -> str:
    try:
        proc = subprocess.run(["git", *args], cwd=os.path.dirname(HERE), capture_output=True, text=True, timeout=30)
        return proc.stdout.strip() if proc.returncode == 0 else ""
    except (OSError, subprocess.SubprocessError):
        return ""


def _write_build_info() -> None:
    """Record what the library was built from (``_lib/build_info.json``): the
    source commit (and whether the tree had local changes), the nvcc release
    and the target architecture.  Benchmark lines carry it as their manifest."""
    import json

    try:
        release = subprocess.run([nvcc(), "--version"], capture_output=True, text=True).stdout.strip().splitlines()[-1]
    except (OSError, IndexError):
        release = ""
    info = {
        "commit": _git("rev-parse", "HEAD"),
        "dirty": bool(_git("status", "--porcelain", "--", "tencirpauli_b200", "include")),
        "nvcc": release,
        "arch": "sm_100a",
    }
    with open(os.path.join(LIBDIR, "build_info.json"), "w") as fh:
        json.dump(info, fh)


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv, debug_bounds="--debug-bounds" in sys.argv)
