"""Benchmark: QPS at recall@10 >= 0.95 of batched greedy beam search on one B200.

Default workload (``pq1m``): 1M x 128 float32 seeded Gaussian mixture (256 components,
sigma 8, means U[0,100], clipped to [0,255]); PQ 32 x 256 trained on a 100k sample; Vamana
R=64, L_build=100, alpha=1.2 (slot width 83); 10,000 queries from the same mixture; k=10;
Hybrid strategy (ADC traversal, exact FP32 L2 rerank of the top L); L is the smallest of
50/75/100/150/200 whose recall@10 against float64 ground truth is >= 0.95.

A step = one batched search of all queries.  ``value`` times the search with queries and
outputs resident in HBM (CUDA events on the launching stream, L2 flushed before every step);
``e2e`` times the same search through the C ABI with host buffers (``dk_search``: host->device
copy of the queries, search, device->host copy of ids, distances and stats).

``--impl reference`` times the CPU restatement of the reference search (the oracle, all host
threads) on the same workload, metric and L.

Multi-GPU (``torchrun --nproc-per-node N``): replicas — each rank holds the whole index and
searches its own copy of the query batch; ``value`` = all ranks' queries / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "pq1m": dict(n=1_000_000, dim=128, comps=256, sigma=8.0, nq=10_000, R=64, l_build=100,
                 alpha=1.2, pq_chunks=32, pq_train=100_000, k=10,
                 l_sweep=[50, 75, 100, 150, 200, 250, 300, 400], strategy="hybrid",
                 seed=0xD15CA77 + 1),
    "fp100k": dict(n=100_000, dim=128, comps=64, sigma=10.0, nq=1000, R=32, l_build=50,
                   alpha=1.2, pq_chunks=0, pq_train=0, k=10, l_sweep=[100], strategy="full",
                   seed=0xD15CA77),
    "pq100k": dict(n=100_000, dim=128, comps=256, sigma=8.0, nq=10_000, R=64, l_build=100,
                   alpha=1.2, pq_chunks=32, pq_train=100_000, k=10,
                   l_sweep=[50, 75, 100, 150, 200, 250, 300, 400], strategy="hybrid",
                   seed=0xD15CA77 + 11),
}
TARGET_RECALL = 0.95
METRIC_NAME = "QPS at recall@10>=0.95"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_key(w: dict) -> str:
    return hashlib.sha1(json.dumps(w, sort_keys=True).encode()).hexdigest()[:12]


def prepare(name: str, rank: int, cache_root: str):
    """Generate (or load from the per-box cache) data, graph, PQ and ground truth."""
    from diskann_b200 import datasets, graph
    from diskann_b200.groundtruth import knn_f64

    w = WORKLOADS[name]
    cdir = os.path.join(cache_root, f"{name}-{workload_key(w)}")
    ready = os.path.join(cdir, "READY")
    if rank != 0:
        t0 = time.time()
        while not os.path.exists(ready):
            if time.time() - t0 > 1800:
                raise TimeoutError("rank 0 did not finish preparing the workload")
            time.sleep(1.0)
    elif not os.path.exists(ready):
        os.makedirs(cdir, exist_ok=True)
        t0 = time.time()
        base, queries = datasets.gaussian_mixture(w["n"], w["dim"], w["comps"], w["sigma"],
                                                  seed=w["seed"], n_queries=w["nq"])
        log(f"[prepare] data {time.time() - t0:.1f}s")
        t0 = time.time()
        vectors, adj, deg, n = graph.build_vamana(base, pruned_degree=w["R"], l_build=w["l_build"],
                                                  alpha=w["alpha"])
        log(f"[prepare] vamana build {time.time() - t0:.1f}s, mean degree {deg[:n].mean():.1f}")
        np.save(os.path.join(cdir, "vectors.npy"), vectors)
        np.save(os.path.join(cdir, "queries.npy"), queries)
        np.save(os.path.join(cdir, "adj.npy"), adj)
        np.save(os.path.join(cdir, "deg.npy"), deg)
        if w["pq_chunks"]:
            t0 = time.time()
            pq = graph.build_pq(vectors, w["pq_chunks"], w["pq_train"], seed=w["seed"])
            log(f"[prepare] pq {time.time() - t0:.1f}s")
            np.save(os.path.join(cdir, "pq_offsets.npy"), pq.offsets)
            np.save(os.path.join(cdir, "pq_pivots.npy"), pq.pivots)
            np.save(os.path.join(cdir, "pq_codes.npy"), pq.codes)
        t0 = time.time()
        gt, _ = knn_f64(base, queries, w["k"], 2)
        log(f"[prepare] float64 ground truth {time.time() - t0:.1f}s")
        np.save(os.path.join(cdir, "gt.npy"), gt)
        with open(ready, "w") as f:
            f.write("ok\n")
    out = dict(w=w, n=w["n"])
    for key in ("vectors", "queries", "adj", "deg", "gt"):
        out[key] = np.load(os.path.join(cdir, f"{key}.npy"))
    if w["pq_chunks"]:
        from diskann_b200 import PQData

        out["pq"] = PQData(np.load(os.path.join(cdir, "pq_offsets.npy")),
                           np.load(os.path.join(cdir, "pq_pivots.npy")),
                           np.load(os.path.join(cdir, "pq_codes.npy")))
    else:
        out["pq"] = None
    return out


class ClockSampler:
    """nvidia-smi clocks sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = f"/tmp/dk_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    p = [x.strip() for x in line.split(",")]
                    if len(p) >= 9:
                        rows.append(p)
            os.remove(self.path)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(stats, w, l, mean_degree, strategy):
    """Bytes one batch must move (per query, summed): one adjacency row per expanded node
    (length word + ids), one scored item per comparison (a PQ code or a full vector), the
    full vectors of the rerank, the query; plus the PQ pivot table once per batch."""
    hops = stats["hops"].astype(np.float64)
    cmps = stats["cmps"].astype(np.float64)
    d = w["dim"]
    per = hops * (4 + 4 * mean_degree) + d * 4
    if strategy == "full":
        per = per + cmps * d * 4
        extra = 0.0
    else:
        per = per + cmps * w["pq_chunks"] + (l if strategy == "hybrid" else 0) * d * 4
        extra = 256.0 * d * 4
    return float(per.sum() + extra)


def run_ours(args, data, rank, world):
    import torch

    from diskann_b200 import DiskANNIndex, FullPrecision, GpuProvider, Hybrid, Knn, Metric, Quantized
    from diskann_b200.groundtruth import recall_at_k

    w = data["w"]
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    t0 = time.time()
    provider = GpuProvider(data["vectors"], data["adj"], data["deg"], data["n"], Metric.L2,
                           pq=data["pq"], device=dev)
    idx = DiskANNIndex(provider)
    log(f"[ours] index upload {time.time() - t0:.1f}s, {provider.info()['device_bytes'] / 2**20:.0f} MiB")
    strategy = {"hybrid": Hybrid(), "full": FullPrecision(), "quantized": Quantized()}[w["strategy"]]
    queries = data["queries"]
    nq, k = queries.shape[0], w["k"]
    gt = data["gt"]
    dq = torch.from_numpy(queries).to(f"cuda:{dev}")
    ids = torch.empty((nq, k), dtype=torch.int32, device=dq.device)
    dists = torch.empty((nq, k), dtype=torch.float32, device=dq.device)
    stats = torch.empty((nq, 4), dtype=torch.int32, device=dq.device)
    stream = torch.cuda.current_stream(dq.device)

    def search(params, strat):
        idx.search_device(params, strat, dq, ids, dists, stats, stream)

    # Recall sweep: smallest L reaching the target.
    chosen = None
    sweep = {}
    for l in w["l_sweep"]:
        search(Knn(k, l), strategy)
        torch.cuda.synchronize()
        r = recall_at_k(ids.cpu().numpy().view(np.uint32), gt, k)
        sweep[l] = round(r, 4)
        if chosen is None and r >= TARGET_RECALL:
            chosen = l
    if chosen is None:
        chosen = w["l_sweep"][-1]
    log(f"[ours] recall sweep {sweep} -> L={chosen}")
    params = Knn(k, chosen)

    # Plain FP32 path at the same target, for the BF16/PQ-vs-FP32 comparison.
    fp32 = None
    if w["strategy"] != "full":
        for l in [l for l in (50, 75, 100, 150, 200, 300) if l >= k]:
            search(Knn(k, l), FullPrecision())
            torch.cuda.synchronize()
            r = recall_at_k(ids.cpu().numpy().view(np.uint32), gt, k)
            if r >= TARGET_RECALL:
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                search(Knn(k, l), FullPrecision())
                s0.record(stream)
                search(Knn(k, l), FullPrecision())
                s1.record(stream)
                torch.cuda.synchronize()
                fp32 = {"L": l, "recall": round(r, 4), "qps": nq / (s0.elapsed_time(s1) / 1e3)}
                break

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dq.device)  # 256 MiB > 126 MB L2

    for _ in range(args.warmup):
        flush.zero_()
        search(params, strategy)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with ClockSampler(dev) as clocks:
        for s in range(args.steps):
            flush.zero_()
            ev[s][0].record(stream)
            search(params, strategy)
            ev[s][1].record(stream)
        torch.cuda.synchronize()
    barrier(world)
    elapsed_ms = sum(a.elapsed_time(b) for a, b in ev)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    st = stats.cpu().numpy().view(np.uint32)
    stats_np = np.zeros(nq, dtype=[("cmps", np.uint32), ("hops", np.uint32),
                                   ("result_count", np.uint32), ("flags", np.uint32)])
    for i, f in enumerate(("cmps", "hops", "result_count", "flags")):
        stats_np[f] = st[:, i]
    rec = recall_at_k(ids.cpu().numpy().view(np.uint32), gt, k)
    ms_per_step = elapsed_ms / args.steps
    value = world * nq / (ms_per_step / 1e3)

    # End to end through the C ABI with host buffers (pinned host memory).
    hq = torch.from_numpy(queries).pin_memory().numpy()
    e2e_t = []
    for s in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        idx.search(params, strategy, hq)
        t1 = time.perf_counter()
        if s >= args.warmup:
            e2e_t.append(t1 - t0)
    e2e_s = max_over_ranks(float(np.mean(e2e_t)) * 1e3, world) / 1e3
    mean_deg = float(data["deg"][: data["n"]].mean())
    alg = algorithmic_bytes(stats_np, w, chosen, mean_deg, w["strategy"])
    achieved = alg / (ms_per_step / 1e3) / 1e9
    peak, peak_src = hbm_peak()
    cl = clocks.summary()
    return dict(value=value, ms_per_step=ms_per_step, recall=rec, L=chosen, sweep=sweep, fp32=fp32,
                e2e=dict(value=world * nq / e2e_s, unit="queries/s",
                         h2d_bytes_per_step=int(queries.nbytes),
                         d2h_bytes_per_step=int(nq * k * 8 + nq * 16)),
                roofline=dict(bound="hbm", achieved=round(achieved, 1), peak=peak, unit="GB/s",
                              frac=round(achieved / peak, 4), traffic=None,
                              algorithmic_bytes_per_step=int(alg), peak_source=peak_src),
                clocks=cl,
                stats=dict(cmps_mean=float(stats_np["cmps"].mean()),
                           hops_mean=float(stats_np["hops"].mean()),
                           spilled=int((stats_np["flags"] & 1).sum())),
                gpu_launches=2 * args.steps)


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(data, l, threads, min_seconds=2.0, max_reps=5):
    """Oracle (CPU restatement of the reference search) on all host threads."""
    from oracle import oracle as orc

    w = data["w"]
    pq = data["pq"]
    o = orc.OracleIndex(data["vectors"], data["adj"], data["deg"], data["n"], orc.METRIC_L2,
                        *(tuple() if pq is None else (pq.offsets, pq.pivots, pq.codes)))
    strat = {"hybrid": orc.STRATEGY_HYBRID, "full": orc.STRATEGY_FULL_PRECISION,
             "quantized": orc.STRATEGY_QUANTIZED}[w["strategy"]]
    q = data["queries"]
    total, reps, t0 = 0, 0, time.perf_counter()
    res = None
    while reps < max_reps and (time.perf_counter() - t0 < min_seconds or reps == 0):
        res = o.search(q, w["k"], l, 1, strat, threads=threads)
        total += q.shape[0]
        reps += 1
    el = time.perf_counter() - t0
    return total / el, reps, res


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def choose_l_on_cpu(data):
    """Smallest L of the sweep whose oracle recall reaches the target (same rule as ours)."""
    from diskann_b200.groundtruth import recall_at_k
    from oracle import oracle as orc

    w = data["w"]
    pq = data["pq"]
    o = orc.OracleIndex(data["vectors"], data["adj"], data["deg"], data["n"], orc.METRIC_L2,
                        *(tuple() if pq is None else (pq.offsets, pq.pivots, pq.codes)))
    strat = {"hybrid": orc.STRATEGY_HYBRID, "full": orc.STRATEGY_FULL_PRECISION,
             "quantized": orc.STRATEGY_QUANTIZED}[w["strategy"]]
    for l in w["l_sweep"]:
        ids, _, _ = o.search(data["queries"], w["k"], l, 1, strat, threads=os.cpu_count() or 1)
        if recall_at_k(ids, data["gt"], w["k"]) >= TARGET_RECALL:
            return l
    return w["l_sweep"][-1]


def config_of(w, name, l):
    return {
        "workload": (f"{name}: {w['n']:,} x {w['dim']} f32 Gaussian mixture ({w['comps']} comp, "
                     f"sigma {w['sigma']}), Vamana R={w['R']} L_build={w['l_build']} "
                     f"alpha={w['alpha']}" + (f", PQ {w['pq_chunks']}x256" if w["pq_chunks"] else "")
                     + f", {w['nq']:,} queries, k={w['k']}, L={l}, strategy={w['strategy']}"),
        "n_points": w["n"], "dim": w["dim"], "queries_per_step": w["nq"], "k": w["k"], "L": l,
        "strategy": w["strategy"], "metric": "L2", "l2_flush": "256 MiB write before every step",
        "parallelism": "replicas",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pq1m", choices=sorted(WORKLOADS))
    ap.add_argument("--cache", default=os.environ.get("DK_BENCH_CACHE", "/tmp/diskann_b200_bench"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return 0
        data = prepare(args.workload, 0, args.cache)
        w = data["w"]
        l = choose_l_on_cpu(data)
        times = []
        for s in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            qps, _, _ = cpu_baseline(data, l, threads, min_seconds=0.0, max_reps=1)
            if s >= args.warmup:
                times.append(w["nq"] / qps)
        ms = float(np.mean(times)) * 1e3
        value = w["nq"] / (ms / 1e3)
        line = {"impl": "reference", "metric": METRIC_NAME, "value": round(value, 1),
                "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_of(w, args.workload, l),
                "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads,
                                 "kind": "port",
                                 "sample": f"all {w['nq']} queries per step, {threads} threads"},
                "e2e": {"value": round(value, 1), "unit": "queries/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    data = prepare(args.workload, rank, args.cache)
    w = data["w"]
    r = run_ours(args, data, rank, world)
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            qps, reps, _ = cpu_baseline(data, r["L"], threads)
            cpu = {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "port",
                   "sample": f"{reps} x {w['nq']} queries, {threads} threads, L={r['L']}"}
        line = {
            "metric": METRIC_NAME, "value": round(r["value"], 1), "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(r["ms_per_step"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(w, args.workload, r["L"]),
            "recall_at_10": round(r["recall"], 4), "recall_sweep": r["sweep"],
            "fp32_path_at_target": r["fp32"],
            "e2e": {k: (round(v, 1) if isinstance(v, float) else v) for k, v in r["e2e"].items()},
            "gpu_launches": r["gpu_launches"], "roofline": r["roofline"], "cpu_baseline": cpu,
            "clocks": r["clocks"], "search_stats": r["stats"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
