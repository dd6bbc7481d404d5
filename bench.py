"""Benchmark: QPS at recall@10 >= 0.95 of batched greedy beam search on one B200.

Default workload (``pq1m``): 1M x 128 float32 seeded Gaussian mixture (256 components,
sigma 8, means U[0,100], clipped to [0,255]); PQ 32 x 256 trained on a 100k sample; Vamana
R=64, L_build=100, alpha=1.2 (slot width 83); 10,000 queries from the same mixture; k=10.
Every strategy (FP32, BF16, FP8, Hybrid) is timed at the smallest L of its sweep whose
recall@10 against float64 ground truth reaches 0.95; the headline is the plain FP32 path (the
strategy whose results equal the reference's search), the others are reported beside it.

A step = one batched search of all queries.  ``value`` times the search with queries and
outputs resident in HBM (CUDA events on the launching stream, L2 flushed before every step);
``e2e`` times the same search through the C ABI with host buffers (``dk_search``: host->device
copy of the queries, search, device->host copy of ids, distances and stats).

``--impl reference`` times the CPU restatement of the reference search (the oracle, all host
threads) on the same workload, metric and L, on a graph the oracle builds itself (the same
graph; that process loads none of this library).

Multi-GPU (``torchrun --nproc-per-node N``): replicas — each rank holds the whole index and
searches its own copy of the query batch; ``value`` = all ranks' queries / max-over-ranks time.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "pq1m": dict(n=1_000_000, dim=128, comps=256, sigma=8.0, nq=10_000, R=64, l_build=100,
                 alpha=1.2, pq_chunks=32, pq_train=100_000, k=10,
                 l_sweep=[50, 75, 100, 150, 200, 250, 300, 400],
                 strategies=["fp32", "bf16", "fp8", "hybrid"], seed=0xD15CA77 + 1),
    "fp100k": dict(n=100_000, dim=128, comps=64, sigma=10.0, nq=1000, R=32, l_build=50,
                   alpha=1.2, pq_chunks=0, pq_train=0, k=10, l_sweep=[50, 75, 100, 150, 200],
                   strategies=["fp32", "bf16", "fp8"], seed=0xD15CA77),
    # A few thousand points: the CPU-only multi-rank tests and smoke runs.
    "tiny": dict(n=3_000, dim=32, comps=8, sigma=5.0, nq=64, R=16, l_build=32, alpha=1.2,
                 pq_chunks=8, pq_train=3_000, k=10, l_sweep=[20, 40, 80],
                 strategies=["fp32", "bf16", "fp8", "hybrid"], seed=0xD15CA77 + 21),
    "pq100k": dict(n=100_000, dim=128, comps=256, sigma=8.0, nq=10_000, R=64, l_build=100,
                   alpha=1.2, pq_chunks=32, pq_train=100_000, k=10,
                   l_sweep=[50, 75, 100, 150, 200, 250, 300, 400],
                   strategies=["fp32", "bf16", "fp8", "hybrid"], seed=0xD15CA77 + 11),
    # The cosine / inner-product shape with BF16 scoring: 1M x 768, isotropic Gaussian rows
    # L2-normalised, inner product.
    "ip768": dict(n=1_000_000, dim=768, normalized=True, metric=1, comps=0, sigma=0.0,
                  nq=10_000, R=64, l_build=128, alpha=1.2, pq_chunks=0, pq_train=0, k=10,
                  l_sweep=[128, 192, 256, 512, 1024, 2048], strategies=["fp32", "bf16", "fp8"],
                  seed=0xD15CA77 + 3),
    # The same rows under CosineNormalized (1 - dot: the inner-product ranking on normalised
    # rows, with the triangle-inequality prune instead of the occluding one).
    "cosn768": dict(n=1_000_000, dim=768, normalized=True, metric=3, comps=0, sigma=0.0,
                    nq=10_000, R=64, l_build=128, alpha=1.2, pq_chunks=0, pq_train=0, k=10,
                    l_sweep=[128, 192, 256], strategies=["fp32", "bf16", "fp8"],
                    seed=0xD15CA77 + 3),
    # The large FP8 + PQ shape: 20M x 384, a zero-centred 1,024-component mixture (means
    # U[-50, 50]^384, sigma 8) with every row scaled to unit length, inner product, R = 32
    # (L_build 200), PQ 48 x 256.  Held in memory, not cached on disk (31 GB of rows; one rank).
    "ip20m": dict(n=20_000_000, dim=384, normalized=True, metric=1, comps=1024, sigma=8.0,
                  mean_range=(-50.0, 50.0), clip=(-255.0, 255.0),
                  nq=10_000, R=32, l_build=200, alpha=1.2, pq_chunks=48, pq_train=100_000, k=10,
                  l_sweep=[64, 100, 128, 192, 256, 384, 512, 576, 640, 768],
                  strategies=["fp32", "bf16", "fp8", "hybrid"], seed=0xD15CA77 + 5, cache=False,
                  gt_queries=1000, gt_prefilter=256),
    # The large FP8 served shape exactly as specified: 20M x 384 isotropic Gaussian rows scaled
    # to unit length, inner product, R = 32 (L_build 200), FP8 + PQ 48 x 256 codes; L swept to
    # 2,048.  Recall on the first 1,000 queries (exact float64 over a BF16 prefilter of 256).
    "c5": dict(n=20_000_000, dim=384, normalized=True, metric=1, comps=0, sigma=0.0,
               nq=10_000, R=32, l_build=200, alpha=1.2, pq_chunks=48, pq_train=100_000, k=10,
               l_sweep=[128, 256, 512, 1024, 2048], strategies=["fp32", "bf16", "fp8", "hybrid"],
               seed=0xD15CA77 + 7, cache=False, gt_queries=1000, gt_prefilter=256),
    # A 2M-point slice of the 20M x 384 shape (same generator family, R = 32, L_build 200):
    # small enough to prepare in about a minute, for sweeps of the wide-row, long-search regime.
    "ip2m384": dict(n=2_000_000, dim=384, normalized=True, metric=1, comps=1024, sigma=8.0,
                    mean_range=(-50.0, 50.0), clip=(-255.0, 255.0),
                    nq=10_000, R=32, l_build=200, alpha=1.2, pq_chunks=0, pq_train=0, k=10,
                    l_sweep=[64, 100, 128, 192, 256, 384, 512],
                    strategies=["fp32", "bf16", "fp8"], seed=0xD15CA77 + 6),
    # The served-stream shape: 10M x 96 mixture of 1,024 components, R = 48.
    "mix10m": dict(n=10_000_000, dim=96, comps=1024, sigma=8.0, nq=10_000, R=48, l_build=100,
                   alpha=1.2, pq_chunks=0, pq_train=0, k=10, l_sweep=[64, 128, 256, 512],
                   strategies=["fp32", "bf16", "fp8"], seed=0xD15CA77 + 4),
}
TARGET_RECALL = 0.95
PARITY_QUERIES = 1000
SERVE_P99_BOUND_MS = 2.0
METRIC_NAME = "QPS at recall@10>=0.95"


def metric_of(w: dict):
    from diskann_b200 import Metric

    return Metric(w.get("metric", 2))


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_key(w: dict) -> str:
    return hashlib.sha1(json.dumps(w, sort_keys=True).encode()).hexdigest()[:12]


def prepare(name: str, rank: int, cache_root: str, builder: str = "library"):
    """Generate (or load from the per-box cache) data, graph, PQ and ground truth.

    ``builder="library"``: the graph is built by this library (GPU-searched batches when a GPU
    is present) and PQ is trained by it.  ``builder="oracle"``: the CPU reference arm, which
    must not load this library: the graph comes from the oracle's restatement of the same
    construction (the identical graph, tests/test_oracle_build.py and test_gpu_build.py), the
    medoid from the oracle's restatement of the reference's rule, and no PQ is built (that arm
    times the FullPrecision search only).  Each builder keeps its own cache."""
    from diskann_b200 import datasets
    from diskann_b200.groundtruth import knn_f64

    w = WORKLOADS[name]
    cache = w.get("cache", True)
    if not cache and rank != 0:
        raise RuntimeError(f"workload {name} is prepared in memory by one rank only")
    tag = "" if builder == "library" else f"-{builder}"
    cdir = os.path.join(cache_root, f"{name}-{workload_key(w)}{tag}")
    ready = os.path.join(cdir, "READY")
    fresh = {}
    if rank != 0:
        t0 = time.time()
        while not os.path.exists(ready):
            if time.time() - t0 > 1800:
                raise TimeoutError("rank 0 did not finish preparing the workload")
            time.sleep(1.0)
    elif not cache or not os.path.exists(ready):
        t0 = time.time()
        if w.get("normalized") and not w["comps"]:
            base, queries = datasets.normalized_gaussian(w["n"], w["dim"], w["seed"],
                                                         n_queries=w["nq"])
        else:
            base, queries = datasets.gaussian_mixture(
                w["n"], w["dim"], w["comps"], w["sigma"], seed=w["seed"],
                mean_range=w.get("mean_range", (0.0, 100.0)), clip=w.get("clip", (0.0, 255.0)),
                n_queries=w["nq"])
            if w.get("normalized"):
                datasets.normalize_rows(base)
                datasets.normalize_rows(queries)
        log(f"[prepare] data {time.time() - t0:.1f}s")
        t0 = time.time()
        import torch

        dev = 0 if torch.cuda.is_available() else None
        if builder == "oracle":
            from oracle import oracle as orc

            vectors, adj, deg, n = orc.build_vamana(base, int(metric_of(w)), w["R"],
                                                    w["l_build"], w["alpha"])
            how = "oracle, host threads"
        else:
            from diskann_b200 import graph

            # Larger batches search on the GPU when there is one: the same graph as the host
            # build.
            vectors, adj, deg, n = graph.build_vamana(base, metric=metric_of(w),
                                                      pruned_degree=w["R"],
                                                      l_build=w["l_build"], alpha=w["alpha"],
                                                      device=dev)
            how = "GPU searches" if dev is not None else "host"
        log(f"[prepare] vamana build ({how}) {time.time() - t0:.1f}s, "
            f"mean degree {deg[:n].mean():.1f}")
        del base  # the first n rows of `vectors` are the same rows
        fresh = dict(vectors=vectors, queries=queries, adj=adj, deg=deg, pq=None)
        if w["pq_chunks"] and builder == "library":
            from diskann_b200 import graph

            t0 = time.time()
            fresh["pq"] = graph.build_pq(vectors, w["pq_chunks"], w["pq_train"], seed=w["seed"])
            log(f"[prepare] pq {time.time() - t0:.1f}s")
        t0 = time.time()
        # Ground truth for the first gt_queries queries (all by default), optionally through
        # the exact-rerank prefilter for bases too large for a full float64 scan.
        gq = w.get("gt_queries", w["nq"])
        fresh["gt"], _ = knn_f64(vectors[:n], queries[:gq], w["k"], int(metric_of(w)),
                                 prefilter=w.get("gt_prefilter", 0))
        if dev is not None:
            torch.cuda.empty_cache()
        log(f"[prepare] float64 ground truth {time.time() - t0:.1f}s")
        if cache:
            os.makedirs(cdir, exist_ok=True)
            for key in ("vectors", "queries", "adj", "deg", "gt"):
                np.save(os.path.join(cdir, f"{key}.npy"), fresh[key])
            if fresh["pq"] is not None:
                np.save(os.path.join(cdir, "pq_offsets.npy"), fresh["pq"].offsets)
                np.save(os.path.join(cdir, "pq_pivots.npy"), fresh["pq"].pivots)
                np.save(os.path.join(cdir, "pq_codes.npy"), fresh["pq"].codes)
            with open(ready, "w") as f:
                f.write("ok\n")
    out = dict(w=w, n=w["n"])
    if fresh:
        out.update(fresh)
        return out
    for key in ("vectors", "queries", "adj", "deg", "gt"):
        out[key] = np.load(os.path.join(cdir, f"{key}.npy"))
    if w["pq_chunks"] and os.path.exists(os.path.join(cdir, "pq_codes.npy")):
        from diskann_b200 import PQData

        out["pq"] = PQData(np.load(os.path.join(cdir, "pq_offsets.npy")),
                           np.load(os.path.join(cdir, "pq_pivots.npy")),
                           np.load(os.path.join(cdir, "pq_codes.npy")))
    else:
        out["pq"] = None
    return out


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML every 5 ms while the timed region
    runs (the fields of nvidia-smi's clocks line); read-only queries, no settings touched."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.dev = device_index
        self.period = period_s
        self.samples = []
        self.max_mhz = None
        self.error = None
        self._stop = None
        self._thread = None

    def _handle(self, nv):
        import torch

        try:
            p = torch.cuda.get_device_properties(self.dev)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip().isdigit()]
            return nv.nvmlDeviceGetHandleByIndex(int(ids[self.dev]) if self.dev < len(ids) else self.dev)

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]
            self._stop = threading.Event()

            def run():
                while not self._stop.is_set():
                    try:
                        mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(mhz), [n for n, m in masks if r & m]))
                    except Exception as e:  # keep the timed region going
                        self.error = str(e)
                    self._stop.wait(self.period)

            self._thread = threading.Thread(target=run, daemon=True)
            self._thread.start()
        except Exception as e:
            self.error = str(e)
        return self

    def __exit__(self, *exc):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"],
                    "samples": 0, "error": self.error}
        sm = [m for m, _ in self.samples]
        reasons = sorted({n for _, rs in self.samples for n in rs})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples), "source": "NVML, 5 ms period"}


STRATEGY_CODES = ("fp32", "bf16", "fp8", "hybrid")
DTYPE_OF = {"fp32": "f32", "bf16": "bf16 (f32 accumulate, exact f32 rerank)",
            "fp8": "fp8-e4m3 (per-vector f32 scale, f32 accumulate, exact f32 rerank)",
            "hybrid": "u8 PQ codes (f32 ADC table, exact f32 rerank)"}


def strategy_objects():
    from diskann_b200 import BF16, FP8, FullPrecision, Hybrid

    return {"fp32": FullPrecision(), "bf16": BF16(), "fp8": FP8(), "hybrid": Hybrid()}


def algorithmic_bytes(stats, w, l, mean_degree, strategy):
    """Bytes one batch must move (per query, summed): one adjacency row per expanded node
    (length word + ids), one scored item per comparison (a full f32 row, a BF16 or FP8 row
    (+ its f32 scale), or a PQ code), the f32 rows of the exact rerank (at most L), the query;
    plus the PQ pivot table once per batch."""
    hops = stats["hops"].astype(np.float64)
    cmps = stats["cmps"].astype(np.float64)
    d = w["dim"]
    lp = (d + 15) // 16 * 16
    per = hops * (4 + 4 * mean_degree) + d * 4
    extra = 0.0
    if strategy == "fp32":
        per = per + cmps * d * 4
    elif strategy == "bf16":
        per = per + cmps * lp * 2 + l * d * 4
    elif strategy == "fp8":
        per = per + cmps * (lp + 4) + l * d * 4
    else:
        per = per + cmps * w["pq_chunks"] + l * d * 4
        extra = 256.0 * d * 4
    return float(per.sum() + extra)


def max_rel_dist_error(ids, dists, data, metric):
    """Largest relative error of the returned float32 distances against the same pairs'
    distances in float64 (the precision forms rerank with exact FP32 rows, so this is the
    FP32 rounding of the final distances)."""
    rel = rel_dist_errors(ids, dists, data, metric)
    return None if rel is None else float(rel.max())


def rel_dist_errors(ids, dists, data, metric):
    """Relative error of each (query row, id) pair's float32 distance against float64 over the
    original float32 rows (0 for invalid ids); None when no id is valid."""
    import torch

    from diskann_b200 import Metric

    valid = ids != 0xFFFFFFFF
    if not valid.any():
        return None
    q = torch.from_numpy(data["queries"][: ids.shape[0]]).cuda().double()
    rows = torch.from_numpy(data["vectors"][np.where(valid, ids, 0).astype(np.int64)]).cuda().double()
    if metric == Metric.L2:
        d = ((rows - q[:, None, :]) ** 2).sum(-1)
    elif metric == Metric.INNER_PRODUCT:
        d = -(rows * q[:, None, :]).sum(-1)
    elif metric == Metric.COSINE:
        d = 1.0 - (rows * q[:, None, :]).sum(-1) / (rows.norm(dim=-1) * q.norm(dim=-1)[:, None])
    else:
        d = 1.0 - (rows * q[:, None, :]).sum(-1)
    got = torch.from_numpy(dists.astype(np.float64)).cuda()
    rel = (got - d).abs() / d.abs().clamp_min(1e-12)
    rel = torch.where(torch.from_numpy(valid).cuda(), rel, torch.zeros_like(rel))
    return rel.cpu().numpy()


def stats_array(st):
    out = np.zeros(st.shape[0], dtype=[("cmps", np.uint32), ("hops", np.uint32),
                                       ("result_count", np.uint32), ("flags", np.uint32)])
    for i, f in enumerate(("cmps", "hops", "result_count", "flags")):
        out[f] = st[:, i]
    return out


def serve_latency(provider, strategy, queries, gt, k, l, rate, seconds, mixed=False, seed=1,
                  streams=0):
    """Poisson arrivals at `rate` requests/s replayed natively through the serving API
    (dk_server_replay from one host thread); latency = completion seen by the host - scheduled
    arrival.  `mixed`: each request draws k from {10, 50, 100} and L from {64, 128, 256, 512}
    (L >= k), as in the served-stream config; else every request uses (k, l)."""
    from diskann_b200 import SearchServer
    from diskann_b200.groundtruth import recall_at_k

    rng = np.random.default_rng(seed)
    n = max(1, int(rate * seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
    if mixed:
        ks = rng.choice([10, 50, 100], size=n)
        ls = np.maximum(rng.choice([64, 128, 256, 512], size=n), ks)
    else:
        ks = np.full(n, k)
        ls = np.full(n, l)
    srv = SearchServer(provider, strategy, max_k=int(ks.max()), max_l=int(ls.max()),
                       queue_depth=16384, streams=streams)
    srv.replay(queries[:64], ks[:64], ls[:64], np.zeros(64))  # warm-up
    t0 = time.perf_counter()
    lat, ids, _ = srv.replay(queries, ks, ls, arrivals, want_results=True)
    elapsed = time.perf_counter() - t0
    info = srv.info()
    srv.close()
    rows = np.arange(n) % queries.shape[0]
    sel = rows < gt.shape[0]  # requests whose query has ground truth
    rec = recall_at_k(ids[sel, :10], gt[rows[sel]], 10)
    pct = percentiles(lat * 1e3)
    return {"offered_qps": rate, "achieved_qps": round(n / elapsed, 1), "requests": n,
            "stream": "mixed k in {10,50,100}, L in {64,128,256,512}" if mixed else f"k={k}, L={l}",
            "recall_at_10": round(rec, 4),
            "p50_ms": round(pct["median"], 4), "p90_ms": round(pct["p90"], 4),
            "p99_ms": round(pct["p99"], 4), "mean_ms": round(pct["mean"], 4),
            "launches": int(info["launches"]), "streams": int(info["streams"])}


def percentiles(x):
    """The benchmark runner's rule (diskann-benchmark-runner/src/utils/percentiles.rs:59-85):
    sorted; median = middle element or the mean of the two middle ones; p90 = x[min(9n/10,
    n-1)]; p99 = x[min(99n/100, n-1)]."""
    x = np.sort(np.asarray(x, dtype=np.float64))
    n = len(x)
    med = x[n // 2] if n % 2 == 1 else (x[n // 2 - 1] + x[n // 2]) / 2.0
    return {"mean": float(x.mean()), "median": float(med), "p90": float(x[min(9 * n // 10, n - 1)]),
            "p99": float(x[min(99 * n // 100, n - 1)])}


def run_ours(args, data, rank, world):
    import torch

    from diskann_b200 import DiskANNIndex, GpuProvider, Knn, Metric
    from diskann_b200.groundtruth import recall_at_k

    w = data["w"]
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    t0 = time.time()
    provider = GpuProvider(data["vectors"], data["adj"], data["deg"], data["n"], metric_of(w),
                           pq=data["pq"], device=dev, low_precision=("bf16", "fp8"))
    idx = DiskANNIndex(provider)
    log(f"[ours] index upload {time.time() - t0:.1f}s, {provider.info()['device_bytes'] / 2**20:.0f} MiB")
    strategies = strategy_objects()
    queries = data["queries"]
    nq, k = queries.shape[0], w["k"]
    gt = data["gt"]
    dq = torch.from_numpy(queries).to(f"cuda:{dev}")
    ids = torch.empty((nq, k), dtype=torch.int32, device=dq.device)
    dists = torch.empty((nq, k), dtype=torch.float32, device=dq.device)
    stats = torch.empty((nq, 4), dtype=torch.int32, device=dq.device)
    stream = torch.cuda.current_stream(dq.device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dq.device)  # 256 MiB > 126 MB L2

    def search(params, strat):
        idx.search_device(params, strat, dq, ids, dists, stats, stream)

    def timed(params, strat, reps=3):
        ts = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            search(params, strat)
            b.record(stream)
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b))
        return nq / (float(np.median(ts)) / 1e3)

    # Per strategy: the smallest L of the sweep whose recall@10 reaches the target, timed.
    table = {}
    for name in w["strategies"]:
        if name == "hybrid" and data["pq"] is None:
            continue
        strat = strategies[name]
        row = None
        sweep = []
        for l in w["l_sweep"]:
            search(Knn(k, l), strat)
            torch.cuda.synchronize()
            r = recall_at_k(ids.cpu().numpy().view(np.uint32), gt, k)
            sweep.append({"L": l, "recall": round(r, 4), "qps": round(timed(Knn(k, l), strat, 1), 1)})
            row = {"L": l, "recall": round(r, 4), "reached": r >= TARGET_RECALL}
            if r >= TARGET_RECALL:
                break
        row["sweep"] = sweep
        search(Knn(k, row["L"]), strat)
        torch.cuda.synchronize()
        err = max_rel_dist_error(ids.cpu().numpy().view(np.uint32), dists.cpu().numpy(), data,
                                 metric_of(w))
        row["max_rel_dist_err_vs_f64"] = None if err is None else float(f"{err:.3g}")
        if name in ("bf16", "fp8"):
            # The traversal's own (low-precision) distances of the returned pairs, before the
            # FP32 rerank, against float64 over the original rows (first 1,000 queries).
            m = min(PARITY_QUERIES, nq)
            sid = ids[:m].cpu().numpy().view(np.uint32).copy()
            lp = idx.score(strat, queries[:m], sid)
            rel = rel_dist_errors(sid, lp, data, metric_of(w))
            if rel is not None:
                row["scoring_rel_err_vs_f64"] = {"median": float(f"{np.median(rel):.3g}"),
                                                 "p99": float(f"{np.quantile(rel, 0.99):.3g}"),
                                                 "max": float(f"{rel.max():.3g}")}
        row["qps"] = round(timed(Knn(k, row["L"]), strat), 1)
        table[name] = row
        log(f"[ours] {name}: {row}")
    # Headline: the plain FP32 path (the strategy whose results equal the reference's search,
    # and the one the CPU reference arm runs) when it reaches the recall target; the precision
    # forms are reported beside it as QPS ratios.  Otherwise the fastest strategy that does.
    reached = {n: r for n, r in table.items() if r["reached"]}
    pool = reached or table
    head = "fp32" if "fp32" in reached else max(pool, key=lambda n: pool[n]["qps"])
    chosen = table[head]["L"]
    strategy = strategies[head]
    params = Knn(k, chosen)
    log(f"[ours] headline strategy {head} at L={chosen}")

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
    step_ms = [a.elapsed_time(b) for a, b in ev]
    log(f"[ours] timed steps (ms): {[round(x, 3) for x in step_ms]}")
    elapsed_ms = sum(step_ms)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    stats_np = stats_array(stats.cpu().numpy().view(np.uint32))
    rec = recall_at_k(ids.cpu().numpy().view(np.uint32), gt, k)
    ms_per_step = elapsed_ms / args.steps
    value = world * nq / (ms_per_step / 1e3)

    # End to end through the C ABI with host buffers (pinned host memory for the queries and
    # the caller-owned result buffers).
    from diskann_b200 import STATS_DTYPE

    hq = torch.from_numpy(queries).pin_memory().numpy()
    pinned = lambda shape, dt: torch.empty(shape, dtype=dt).pin_memory().numpy()  # noqa: E731
    hout = (pinned((nq, k), torch.int32).view(np.uint32), pinned((nq, k), torch.float32),
            pinned((nq * 16,), torch.uint8).view(STATS_DTYPE))
    e2e_t = []
    for s in range(args.warmup + args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        idx.search(params, strategy, hq, out=hout)
        t1 = time.perf_counter()
        if s >= args.warmup:
            e2e_t.append(t1 - t0)
    e2e_s = max_over_ranks(float(np.mean(e2e_t)) * 1e3, world) / 1e3

    # Serving (N=1 only): per strategy, Poisson arrivals replayed through dk_server_* at
    # offered rates growing 1.5x from a quarter of the strategy's batch QPS until the server
    # saturates (achieved below 90 % of offered, or p99 above the bound: SERVE_P99_BOUND_MS, or
    # twice the p99 at the lightest load when a single search takes longer); capacity = the
    # highest achieved rate whose p99 stays within the bound.  Plus the mixed-k/L stream at
    # 100k requests/s (or the batch QPS / 10 when that is lower).
    serving = None
    if world == 1 and not args.no_serving:
        serving = {}
        for name in ("fp32", "bf16", "fp8"):
            if name not in table:
                continue
            st_obj, ls = strategies[name], table[name]["L"]
            rows, cap = [], 0.0
            rate = float(max(1000, int(table[name]["qps"] / 4 / 1000) * 1000))
            bound = SERVE_P99_BOUND_MS
            while rate <= 8_000_000.0:
                secs = min(args.serve_seconds, 2_000_000.0 / rate)
                row = serve_latency(provider, st_obj, queries, gt, k, ls, rate, secs)
                rows.append(row)
                if len(rows) == 1:  # long searches: twice the p99 of the lightest load
                    bound = max(SERVE_P99_BOUND_MS, 2.0 * row["p99_ms"])
                ok = row["p99_ms"] <= bound
                if ok:
                    cap = max(cap, row["achieved_qps"])
                if not ok or row["achieved_qps"] < 0.9 * rate:
                    break
                rate = float(int(rate * 1.5 / 1000) * 1000)
            mixed = serve_latency(provider, st_obj, queries, gt, k, ls,
                                  min(100_000.0, float(int(table[name]["qps"] / 10))),
                                  args.serve_seconds, mixed=True)
            serving[name] = {"L": ls, "p99_bound_ms": round(bound, 3),
                             "capacity_qps": round(cap, 1), "rates": rows, "mixed": mixed}
            log(f"[ours] serving {name}: capacity {cap:.0f} req/s at p99 <= "
                f"{bound:.3f} ms; {rows} mixed {mixed}")

    mean_deg = float(data["deg"][: data["n"]].mean())
    alg = algorithmic_bytes(stats_np, w, chosen, mean_deg, head)
    achieved = alg / (ms_per_step / 1e3) / 1e9
    peak, peak_src = hbm_peak()
    fp32_row = table.get("fp32")
    fp32_alg = None
    if fp32_row is not None:
        search(Knn(k, fp32_row["L"]), strategies["fp32"])
        torch.cuda.synchronize()
        st32 = stats_array(stats.cpu().numpy().view(np.uint32))
        fp32_alg = algorithmic_bytes(st32, w, fp32_row["L"], mean_deg, "fp32")
        fp32_row = dict(fp32_row, roofline_frac=round(
            fp32_alg * fp32_row["qps"] / nq / 1e9 / peak, 4))
    # GPU results of the first PARITY_QUERIES queries for the strategies whose results are
    # defined bit for bit by the reference's search (FullPrecision, Hybrid), each at its own L;
    # the CPU-baseline leg runs the oracle on the same queries and compares.
    parity_gpu = {}
    if world == 1:
        for name in ("fp32", "hybrid"):
            if name in table:
                lp = table[name]["L"]
                search(Knn(k, lp), strategies[name])
                torch.cuda.synchronize()
                m = min(PARITY_QUERIES, nq)
                parity_gpu[name] = (lp, ids[:m].cpu().numpy().view(np.uint32).copy(),
                                    dists[:m].cpu().numpy().copy(),
                                    stats_array(stats[:m].cpu().numpy().view(np.uint32)))
    return dict(value=value, ms_per_step=ms_per_step, recall=rec, L=chosen, strategy=head,
                strategies=table, fp32=fp32_row, serving=serving, parity_gpu=parity_gpu,
                e2e=dict(value=world * nq / e2e_s, unit="queries/s",
                         h2d_bytes_per_step=int(queries.nbytes),
                         d2h_bytes_per_step=int(nq * k * 8 + nq * 16)),
                roofline=dict(bound="hbm", achieved=round(achieved, 1), peak=peak, unit="GB/s",
                              frac=round(achieved / peak, 4),
                              traffic=traffic_from_profile(args.workload, head, nq),
                              algorithmic_bytes_per_step=int(alg), peak_source=peak_src),
                clocks=clocks.summary(),
                stats=dict(cmps_mean=float(stats_np["cmps"].mean()),
                           hops_mean=float(stats_np["hops"].mean()),
                           spilled=int((stats_np["flags"] & 1).sum())),
                gpu_launches=2 * args.steps)


def traffic_from_profile(workload, strategy, nq):
    """DRAM bytes (read + write) per launch of the headline kernel, from the committed ncu
    summary of the same workload (scaled to `nq` queries), or None when there is none."""
    p = os.path.join(ROOT, "profiles", f"dram_traffic_{workload}.json")
    try:
        with open(p) as f:
            rec = json.load(f)[strategy]
        return int(rec["dram_bytes"] * nq / rec["queries"])
    except Exception:
        return None


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return 6650.0, "fallback"


def oracle_strategy(name):
    from oracle import oracle as orc

    return {"hybrid": orc.STRATEGY_HYBRID, "fp32": orc.STRATEGY_FULL_PRECISION}[name]


def oracle_index(data):
    from oracle import oracle as orc

    pq = data["pq"]
    return orc.OracleIndex(data["vectors"], data["adj"], data["deg"], data["n"],
                           int(metric_of(data["w"])),
                           *(tuple() if pq is None else (pq.offsets, pq.pivots, pq.codes)))


def cpu_baseline(data, strategy, l, threads, min_seconds=2.0, max_reps=5, nq=None):
    """Oracle (CPU restatement of the reference search) on `threads` host threads."""
    w = data["w"]
    o = oracle_index(data)
    q = data["queries"] if nq is None else data["queries"][:nq]
    total, reps, t0 = 0, 0, time.perf_counter()
    res = None
    while reps < max_reps and (time.perf_counter() - t0 < min_seconds or reps == 0):
        res = o.search(q, w["k"], l, 1, oracle_strategy(strategy), threads=threads)
        total += q.shape[0]
        reps += 1
    el = time.perf_counter() - t0
    return total / el, reps, res


def _median_time(fn, reps=3):
    fn()  # warm-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def next_rows(data, threads, build=True):
    """Throughput of the paths beside the k-NN search, on the same index and queries: range
    search, paged search, the diskann-inmem provider (u8 and f16 rows of the same vectors),
    and graph construction on a 100k-point prefix (GPU-searched batches vs host only).  Host
    buffers through the C ABI (copies inside the timing), median of 3 after a warm-up; each
    beside the oracle's single-thread timing on a sample."""
    from diskann_b200 import (DiskANNIndex, FullPrecision, GpuProvider, InmemProvider, Knn,
                              Metric, Range, graph)
    from diskann_b200.index import inmem_rows
    from oracle import oracle as orc

    w = data["w"]
    n, k = data["n"], w["k"]
    q = data["queries"]
    nq = q.shape[0]
    out = {}
    prov = GpuProvider(data["vectors"], data["adj"], data["deg"], n, metric_of(w))
    idx = DiskANNIndex(prov)
    o = oracle_index(data)
    sample = min(300, nq)

    # Range: radius = median distance of the 10th neighbour at L = 50.
    _, d10, _ = idx.search(Knn(k, 50), FullPrecision(), q)
    radius = float(np.median(d10[:, k - 1]))
    rp = Range(50, radius)
    from diskann_b200 import STATS_DTYPE

    rbuf = (np.empty((nq, 2000), np.uint32), np.empty((nq, 2000), np.float32),
            np.zeros(nq, STATS_DTYPE))  # caller-owned result arrays, reused
    res = {}
    t = _median_time(lambda: res.__setitem__(
        "r", idx.range_search_arrays(rp, q, capacity=2000, out=rbuf)))
    counts = res["r"][2]["result_count"]
    t0 = time.perf_counter()
    for i in range(sample):
        o.range_search(q[i], 50, radius, capacity=2000)
    cpu = sample / (time.perf_counter() - t0)
    out["range"] = {"qps": round(nq / t, 1), "cpu_qps": round(cpu, 1), "cpu_cores": 1,
                    "starting_l": 50, "radius": round(radius, 3),
                    "mean_results": round(float(counts.mean()), 2),
                    "second_round": round(float((res["r"][2]["flags"] & 2).astype(bool).mean()), 3)}

    # Paged: one session per query, l_value 50, three pages of 10.
    def paged():
        ps = idx.paged_search(q, 50)
        for _ in range(3):
            ps.next_page_arrays(k)
        ps.close()
    t = _median_time(paged)
    t0 = time.perf_counter()
    for i in range(sample // 3):
        ops = o.paged_search(q[i], 50)
        for _ in range(3):
            ops.next_page(k)
    cpu = 3 * (sample // 3) / (time.perf_counter() - t0)
    out["paged"] = {"pages_per_s": round(3 * nq / t, 1), "cpu_pages_per_s": round(cpu, 1),
                    "cpu_cores": 1, "l_value": 50, "page_size": k, "pages": 3}
    prov.close()

    # diskann-inmem provider: the same graph over u8 / f16 rows, all slots readable.
    total = data["vectors"].shape[0]
    tags = np.full(total, 254, np.uint8)
    tags[n:] = 255
    ext = np.arange(total, dtype=np.uint64)
    ext[n:] = np.uint64(0xFFFFFFFFFFFFFFFF)
    kinds = [("inmem_f16", data["vectors"].astype(np.float16), 1)]
    if not w.get("normalized"):  # values in [0, 255]: the u8 layer holds them after rounding
        kinds.insert(0, ("inmem_u8", np.clip(np.rint(data["vectors"]), 0, 255).astype(np.uint8), 2))
    for name, typed, code in kinds:
        ip = InmemProvider(typed, data["adj"], data["deg"], n, tags, ext, metric_of(w))
        qt = (np.clip(np.rint(q), 0, 255).astype(np.uint8) if code == 2 else q.astype(np.float16))
        res = {}
        t = _median_time(lambda: res.__setitem__("r", ip.search(Knn(k, 50), qt)))
        recall = float(np.mean([len(set(res["r"][0][i].tolist()) & set(data["gt"][i].tolist())) / k
                                for i in range(min(nq, data["gt"].shape[0]))]))
        ip.close()
        oi = orc.OracleIndex(typed.astype(np.float32), data["adj"], data["deg"], n,
                             int(metric_of(w)))
        rows = inmem_rows(typed, tags)
        t0 = time.perf_counter()
        for i in range(sample):
            oi.inmem_search(code, rows, ext, qt[i] if code == 2 else qt[i].astype(np.float32), k, 50)
        cpu = sample / (time.perf_counter() - t0)
        out[name] = {"qps": round(nq / t, 1), "cpu_qps": round(cpu, 1), "cpu_cores": 1, "L": 50,
                     "recall_at_10": round(recall, 4)}

    if not build:
        return out
    # Graph construction on a 100k-point prefix: GPU-searched batches vs host threads only
    # (the same graph, by construction).
    sub = data["vectors"][: min(100_000, n)]
    res = {}
    t0 = time.perf_counter()
    res["g"] = graph.build_vamana(sub, pruned_degree=w["R"], l_build=w["l_build"],
                                  alpha=w["alpha"], device=0)
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    res["h"] = graph.build_vamana(sub, pruned_degree=w["R"], l_build=w["l_build"],
                                  alpha=w["alpha"])
    t_host = time.perf_counter() - t0
    same = bool(np.array_equal(res["g"][2], res["h"][2]) and np.array_equal(res["g"][1], res["h"][1]))
    out["build_100k"] = {"gpu_assisted_s": round(t_gpu, 2), "host_s": round(t_host, 2),
                         "host_threads": threads, "points": int(sub.shape[0]),
                         "identical_graph": same}
    return out


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown CPU"


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Largest value over the ranks (timings are reported as the slowest rank's)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def choose_l_on_cpu(data, strategy):
    """Smallest L of the sweep whose oracle recall reaches the target (same rule as ours)."""
    from diskann_b200.groundtruth import recall_at_k

    w = data["w"]
    o = oracle_index(data)
    for l in w["l_sweep"]:
        ids, _, _ = o.search(data["queries"], w["k"], l, 1, oracle_strategy(strategy),
                             threads=os.cpu_count() or 1)
        if recall_at_k(ids, data["gt"], w["k"]) >= TARGET_RECALL:
            return l
    return w["l_sweep"][-1]


def describe_data(w):
    if w.get("normalized") and not w["comps"]:
        return "isotropic Gaussian rows scaled to unit length"
    lo, hi = w.get("mean_range", (0.0, 100.0))
    mix = f"Gaussian mixture ({w['comps']} comp, means U[{lo:g}, {hi:g}], sigma {w['sigma']})"
    return mix + (", rows scaled to unit length" if w.get("normalized") else "")


def config_of(w, name, l, strategy):
    return {
        "workload": (f"{name}: {w['n']:,} x {w['dim']} f32 {describe_data(w)}, "
                     f"{metric_of(w).name}, Vamana R={w['R']} L_build={w['l_build']} "
                     f"alpha={w['alpha']}" + (f", PQ {w['pq_chunks']}x256" if w["pq_chunks"] else "")
                     + f", {w['nq']:,} queries, k={w['k']}, L={l}, strategy={strategy}"),
        "n_points": w["n"], "dim": w["dim"], "queries_per_step": w["nq"], "k": w["k"], "L": l,
        "strategy": strategy, "metric": metric_of(w).name,
        "l2_flush": "256 MiB write before every step",
        "parallelism": "replicas",
    }


def profile_case(args):
    """Two searches of the workload's query batch with one strategy and L (for ncu -s 1 -c 1),
    or with ``--profile next`` the range / paged / inmem part of the next-rows section."""
    import torch

    from diskann_b200 import DiskANNIndex, GpuProvider, Knn, Metric

    if args.profile == "next":
        data = prepare(args.workload, 0, args.cache)
        torch.cuda.set_device(0)
        log(f"[profile] next rows {next_rows(data, os.cpu_count() or 1, build=False)}")
        return 0
    if args.profile == "build":  # graph construction of a 100k-point prefix on the GPU
        from diskann_b200 import graph

        data = prepare(args.workload, 0, args.cache)
        w = data["w"]
        t0 = time.perf_counter()
        graph.build_vamana(data["vectors"][: min(100_000, data["n"])], metric=metric_of(w),
                           pruned_degree=w["R"], l_build=w["l_build"], alpha=w["alpha"], device=0)
        log(f"[profile] build {time.perf_counter() - t0:.2f}s")
        return 0
    name, l = args.profile.split(":")
    data = prepare(args.workload, 0, args.cache)
    w = data["w"]
    torch.cuda.set_device(0)
    prov = GpuProvider(data["vectors"], data["adj"], data["deg"], data["n"], metric_of(w),
                       pq=data["pq"], low_precision=("bf16", "fp8"))
    idx = DiskANNIndex(prov)
    q = torch.from_numpy(data["queries"]).cuda()
    nq, k = q.shape[0], w["k"]
    ids = torch.empty((nq, k), dtype=torch.int32, device="cuda")
    dists = torch.empty((nq, k), dtype=torch.float32, device="cuda")
    stats = torch.empty((nq, 4), dtype=torch.int32, device="cuda")
    for _ in range(2):
        idx.search_device(Knn(k, int(l)), strategy_objects()[name], q, ids, dists, stats)
    torch.cuda.synchronize()
    log(f"[profile] {name} L={l}: mean cmps {float(stats[:, 0].float().mean()):.1f}")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="pq1m", choices=sorted(WORKLOADS))
    ap.add_argument("--cache", default=os.environ.get("DK_BENCH_CACHE", "/tmp/diskann_b200_bench"))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the range / paged / inmem / build throughput section")
    ap.add_argument("--profile", default=None, metavar="STRATEGY:L",
                    help="profiling case for ncu: upload the workload's index and run two "
                         "batched searches (warm-up, profiled), no timing, no JSON line; "
                         "'next' runs the range / paged / inmem measurements instead, 'build' "
                         "the construction of a 100k-point prefix")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    threads = os.cpu_count() or 1

    if args.profile:
        return profile_case(args)

    if args.impl == "reference":
        # The reference's search on the host cores: the oracle port (the reference is Rust and
        # no Rust toolchain is available to build it), plain FP32 search at the smallest L of
        # the sweep reaching the recall target, all host threads.  Each step is a bounded
        # sample of the query batch.
        if rank != 0:
            return 0
        data = prepare(args.workload, 0, args.cache, builder="oracle")
        w = data["w"]
        l = choose_l_on_cpu(data, "fp32")
        sample = min(w["nq"], 4000)
        times = []
        for s in range(args.warmup + args.steps):
            qps, _, _ = cpu_baseline(data, "fp32", l, threads, min_seconds=0.0, max_reps=1,
                                     nq=sample)
            if s >= args.warmup:
                times.append(sample / qps)
        ms = float(np.mean(times)) * 1e3
        value = sample / (ms / 1e3)
        line = {"impl": "reference", "metric": METRIC_NAME, "value": round(value, 1),
                "unit": "queries/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_of(w, args.workload, l, "fp32"),
                "cpu_baseline": {"value": round(value, 1), "unit": "queries/s", "cores": threads,
                                 "kind": "port",
                                 "sample": f"{sample} of the {w['nq']} queries per step, "
                                           f"{threads} threads, FullPrecision L={l}, "
                                           f"{cpu_model()}"},
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
            cpu_strat = r["strategy"] if r["strategy"] in ("fp32", "hybrid") else "fp32"
            cpu_l = r["L"] if cpu_strat == r["strategy"] else (r["fp32"] or {}).get("L", r["L"])
            sample = min(w["nq"], 4000)
            qps, reps, _ = cpu_baseline(data, cpu_strat, cpu_l, threads, nq=sample)
            cpu = {"value": round(qps, 1), "unit": "queries/s", "cores": threads, "kind": "port",
                   "sample": f"{reps} x {sample} queries, {threads} threads, "
                             f"{cpu_strat} L={cpu_l}, {cpu_model()}"}
            # Parity: the oracle on the first PARITY_QUERIES queries against the GPU's results.
            parity = {}
            o = oracle_index(data)
            for name, (lp, gi, gd, gs) in r["parity_gpu"].items():
                m = gi.shape[0]
                oi, od, ost = o.search(data["queries"][:m], w["k"], lp, 1, oracle_strategy(name),
                                       threads=threads)
                parity[name] = {
                    "L": lp, "of": int(m),
                    "ids_equal": int((gi == oi).all(1).sum()),
                    "dist_bits_equal": int((gd.view(np.uint32) == od.view(np.uint32)).all(1).sum()),
                    "cmps_equal": int((gs["cmps"] == ost["cmps"]).sum()),
                    "hops_equal": int((gs["hops"] == ost["hops"]).sum()),
                    "result_count_equal": int((gs["result_count"] == ost["result_count"]).sum())}
            log(f"[ours] parity vs oracle {parity}")
        line = {
            "metric": METRIC_NAME, "value": round(r["value"], 1), "unit": "queries/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(r["ms_per_step"], 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE_OF[r["strategy"]], "data": "synthetic",
            "config": config_of(w, args.workload, r["L"], r["strategy"]),
            "recall_at_10": round(r["recall"], 4), "strategies": r["strategies"],
            "fp32_path_at_target": r["fp32"],
            # Each precision form's QPS over the plain FP32 path's, both at the smallest L of
            # the sweep reaching the recall target (or their last L when it is not reached).
            "precision_vs_fp32": {n: round(row["qps"] / r["fp32"]["qps"], 3)
                                  for n, row in r["strategies"].items()
                                  if n in ("bf16", "fp8") and r["fp32"]},
            "serving": r["serving"],
            "e2e": {k: (round(v, 1) if isinstance(v, float) else v) for k, v in r["e2e"].items()},
            "gpu_launches": r["gpu_launches"], "roofline": r["roofline"], "cpu_baseline": cpu,
            "clocks": r["clocks"], "search_stats": r["stats"],
        }
        if cpu is not None:
            line["parity"] = parity
        if world == 1 and not args.no_next_rows:
            line["next_rows"] = next_rows(data, threads)
            log(f"[ours] next rows {line['next_rows']}")
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
