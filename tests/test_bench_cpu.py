"""CPU checks of bench.py's committed profile inputs: the per-launch DRAM
traffic and warp-instruction counts that its roofline reads must be present
for the default workloads and parse as positive numbers."""

from __future__ import annotations

import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def test_profile_counts_for_the_default_workloads() -> None:
    bench = _bench()
    for kernel in ("k_ring<double>", "k_ring<float>"):
        count = bench._profile_instructions(kernel, "random2000_n28")
        assert count is not None and count > 1e10, kernel
    for lattice in ("4x6", "4x7"):
        count = bench._profile_instructions("k_u1_apply", f"j1j2_{lattice}_half_c128")
        assert count is not None and count > 1e8, lattice
    count = bench._profile_instructions("k_ring<float,rhs_block>", "heisenberg64_nmax26_rhs8_seed20261203")
    assert count is not None and count > 1e10
    assert bench._profile_instructions("k_ring<double>", "random2000_n99") is None
    traffic = bench._profile_traffic("k_ring<double>")
    # at least the compulsory bytes of one n = 28 launch (x read, y written)
    assert traffic is not None and traffic >= 2 * 16 * (1 << 28)
