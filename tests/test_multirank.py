"""CPU, world_size 2 over gloo: the replica path of bench.py (one process per GPU on a B200
node).  Rank 0 prepares the workload while rank 1 waits for it; timings are combined as the
maximum over ranks; the reference arm runs on rank 0 only and the other rank exits at once.
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, cache, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        data = bench.prepare("tiny", rank, cache)
        bench.barrier(world)
        slowest = bench.max_over_ranks(1.5 + rank, world)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"slowest": slowest, "n": int(data["n"]),
                       "gt0": data["gt"][0].tolist(), "deg_sum": int(data["deg"].sum())}, f)
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_ranks_share_the_workload_and_the_max_time(tmp_path):
    cache = str(tmp_path / "cache")
    mp.start_processes(_rank_main, args=(2, _free_port(), cache, str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert r0["slowest"] == r1["slowest"] == 2.5
    assert r0["n"] == r1["n"] == 3000
    assert r0["gt0"] == r1["gt0"] and r0["deg_sum"] == r1["deg_sum"]


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    env = dict(os.environ, WORLD_SIZE="2", DK_BENCH_CACHE=str(tmp_path / "cache"))
    outs = []
    for rank in (0, 1):
        e = dict(env, RANK=str(rank), LOCAL_RANK=str(rank))
        p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                            "--workload", "tiny", "--gpus", "2", "--steps", "1", "--warmup", "3"],
                           env=e, capture_output=True, text=True, timeout=300)
        assert p.returncode == 0, p.stderr[-2000:]
        outs.append(p.stdout.strip())
    line = json.loads(outs[0])
    assert line["impl"] == "reference" and line["value"] > 0 and line["n_gpus"] == 2
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
    assert outs[1] == ""
