"""GPU: bench.py end to end on the tiny workload: one JSON line with the contract's keys, and
the next-rows section (range, paged, inmem, construction) filled in."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_tiny_workload(tmp_path):
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--workload", "tiny",
                        "--steps", "3", "--warmup", "3", "--serve-seconds", "0.1",
                        "--cache", str(tmp_path)],
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    line = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "dtype", "config", "e2e", "gpu_launches",
                "roofline", "cpu_baseline", "clocks"):
        assert key in line, key
    assert line["value"] > 0 and line["e2e"]["value"] > 0 and line["gpu_launches"] > 0
    nr = line["next_rows"]
    assert nr["range"]["qps"] > 0 and nr["paged"]["pages_per_s"] > 0
    assert nr["inmem_u8"]["qps"] > 0 and nr["inmem_f16"]["qps"] > 0
    assert nr["build_100k"]["identical_graph"]
    # The CPU-baseline leg checks the GPU against the oracle on a sample of the same queries.
    for name, row in line["parity"].items():
        assert row["of"] > 0
        for key in ("ids_equal", "dist_bits_equal", "cmps_equal", "hops_equal",
                    "result_count_equal"):
            assert row[key] == row["of"], (name, key, row)
    assert set(line["precision_vs_fp32"]) == {"bf16", "fp8"}


def test_bench_reference_arm_maps_only_the_oracle(tmp_path):
    """The timed CPU reference arm builds its graph with the oracle's restatement and never
    loads this library."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--workload', "
            "'tiny', '--steps', '3', '--warmup', '3', '--cache', %r]\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
            "except SystemExit:\n    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('MAPPED', 'libdiskann_b200' in maps, 'liboracle' in maps)\n") % str(tmp_path)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=900,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-3000:]
    line = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert "MAPPED False True" in p.stdout
