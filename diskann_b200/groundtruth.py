"""Exact k-NN ground truth in float64 on the GPU, and recall@k.

This is the measurement oracle for recall (the reference computes recall against exact
ground truth, diskann-benchmark-core/src/recall.rs:146+); float64 is used here and nowhere
on the search path.  Distances follow the reference's metric definitions: squared L2,
negated inner product, 1 - cosine, 1 - dot (normalised cosine).
"""

from __future__ import annotations

import numpy as np


def knn_f64(base: np.ndarray, queries: np.ndarray, k: int, metric: int = 2,
            device: str = "cuda", base_chunk: int = 1 << 18, query_block: int = 2048):
    """Return ``(ids uint32 (nq, k), dists float64 (nq, k))`` of the exact k nearest rows."""
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
    """Mean over queries of |ids[:k] ∩ gt[:k]| / k."""
    hits = 0
    for a, b in zip(ids[:, :k], gt[:, :k]):
        hits += len(set(a.tolist()) & set(b.tolist()))
    return hits / (k * ids.shape[0])
