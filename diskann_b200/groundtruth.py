"""Exact k-NN ground truth in float64 on the GPU, and recall@k.

This is the measurement oracle for recall (the reference computes recall against exact
ground truth, diskann-benchmark-core/src/recall.rs:146+); float64 is used here and nowhere
on the search path.  Distances follow the reference's metric definitions: squared L2,
negated inner product, 1 - cosine, 1 - dot (normalised cosine).
"""

from __future__ import annotations

import numpy as np


def knn_f64(base: np.ndarray, queries: np.ndarray, k: int, metric: int = 2,
            device: str = "cuda", base_chunk: int = 1 << 18, query_block: int = 2048,
            prefilter: int = 0):
    """Return ``(ids uint32 (nq, k), dists float64 (nq, k))`` of the exact k nearest rows.

    ``prefilter`` = C > 0 (for bases too large to scan in float64, e.g. 20M x 384): each
    query's C best rows by a lower-precision score are taken first, then ranked by their exact
    float64 distances.  The score is a BF16 tensor-core dot product for the angular metrics
    (unit-scale rows) and an FP32 one for L2, whose |x|^2 - 2 q.x on unnormalised rows loses
    too much in BF16.  The k nearest are among the C as long as that rounding cannot move a
    true neighbour below the C-th candidate; with C = 256 and k = 10 the margin between the 10th
    and the 256th best score is far above it on the benchmark shapes, and
    tests/test_gpu_groundtruth.py checks the result equals the full float64 scan."""
    if prefilter:
        return _knn_prefiltered(base, queries, k, metric, device, base_chunk, query_block,
                                prefilter)
    import torch

    if device.startswith("cuda") and not torch.cuda.is_available():
        device = "cpu"
    dev = torch.device(device)
    # The base stays in its own type on the device; each chunk is widened to float64 (exact)
    # when it is used, so a large base needs its own size in memory, not twice that.
    B = torch.as_tensor(np.ascontiguousarray(base), device=dev)
    Q = torch.as_tensor(np.ascontiguousarray(queries), device=dev).to(torch.float64)
    n = B.shape[0]
    out_i = np.empty((Q.shape[0], k), np.uint32)
    out_d = np.empty((Q.shape[0], k), np.float64)
    for q0 in range(0, Q.shape[0], query_block):
        q = Q[q0:q0 + query_block]
        qn = (q * q).sum(1, keepdim=True)
        best_d = None
        best_i = None
        for b0 in range(0, n, base_chunk):
            x = B[b0:b0 + base_chunk].to(torch.float64)
            bn = (x * x).sum(1)
            dot = q @ x.T
            if metric == 2:
                d = qn - 2.0 * dot + bn[None, :]
            elif metric == 1:
                d = -dot
            elif metric == 3:
                d = 1.0 - dot
            else:
                d = 1.0 - dot / (qn.sqrt() * bn.sqrt()[None, :]).clamp_min(1e-300)
            kk = min(k, d.shape[1])
            vd, vi = torch.topk(d, kk, dim=1, largest=False)
            vi = vi + b0
            if best_d is None:
                best_d, best_i = vd, vi
            else:
                cd = torch.cat([best_d, vd], 1)
                ci = torch.cat([best_i, vi], 1)
                best_d, sel = torch.topk(cd, min(k, cd.shape[1]), dim=1, largest=False)
                best_i = torch.gather(ci, 1, sel)
        out_i[q0:q0 + q.shape[0]] = best_i.cpu().numpy().astype(np.uint32)
        out_d[q0:q0 + q.shape[0]] = best_d.cpu().numpy()
    return out_i, out_d


def recall_at_k(ids: np.ndarray, gt: np.ndarray, k: int) -> float:
    """Mean over queries of |ids[:k] ∩ gt[:k]| / k (over the first len(gt) queries when the
    ground truth covers only a prefix of the query set)."""
    m = min(ids.shape[0], gt.shape[0])
    hits = 0
    for a, b in zip(ids[:m, :k], gt[:m, :k]):
        hits += len(set(a.tolist()) & set(b.tolist()))
    return hits / (k * m)


def _knn_prefiltered(base, queries, k, metric, device, base_chunk, query_block, cand):
    import torch

    if device.startswith("cuda") and not torch.cuda.is_available():
        device = "cpu"
    dev = torch.device(device)
    B = torch.as_tensor(np.ascontiguousarray(base), device=dev)
    Q = torch.as_tensor(np.ascontiguousarray(queries), device=dev)
    n = B.shape[0]
    cand = min(cand, n)
    out_i = np.empty((Q.shape[0], k), np.uint32)
    out_d = np.empty((Q.shape[0], k), np.float64)
    low = torch.float32 if metric == 2 else torch.bfloat16
    for q0 in range(0, Q.shape[0], query_block):
        q = Q[q0:q0 + query_block]
        qb = q.to(low)
        best_s = best_i = None
        for b0 in range(0, n, base_chunk):
            x = B[b0:b0 + base_chunk]
            dot = (qb @ x.to(low).T).float()
            if metric == 2:  # smaller |x|^2 - 2 q.x is nearer
                score = (x.float() * x.float()).sum(1)[None, :] - 2.0 * dot
            elif metric == 0:
                score = -dot / x.float().norm(dim=1).clamp_min(1e-30)[None, :]
            else:
                score = -dot
            vs, vi = torch.topk(score, min(cand, score.shape[1]), dim=1, largest=False)
            vi = vi + b0
            if best_s is None:
                best_s, best_i = vs, vi
            else:
                cs, ci = torch.cat([best_s, vs], 1), torch.cat([best_i, vi], 1)
                best_s, sel = torch.topk(cs, min(cand, cs.shape[1]), dim=1, largest=False)
                best_i = torch.gather(ci, 1, sel)
        xc = B[best_i].to(torch.float64)  # (block, cand, dim)
        qd = q.to(torch.float64)[:, None, :]
        dot = (xc * qd).sum(-1)
        if metric == 2:
            d = ((xc - qd) ** 2).sum(-1)
        elif metric == 1:
            d = -dot
        elif metric == 3:
            d = 1.0 - dot
        else:
            d = 1.0 - dot / (xc.norm(dim=-1) * qd.norm(dim=-1)).clamp_min(1e-300)
        vd, sel = torch.topk(d, k, dim=1, largest=False)
        out_i[q0:q0 + q.shape[0]] = torch.gather(best_i, 1, sel).cpu().numpy().astype(np.uint32)
        out_d[q0:q0 + q.shape[0]] = vd.cpu().numpy()
    return out_i, out_d
