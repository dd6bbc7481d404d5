// Host side of the batched search: shared-memory planning, visited-set sizing, kernel choice
// and the two-pass launch (first pass with a shared-memory hash, spill pass with a bitmap).
// Device code is in dk_kernels.cuh; per-metric instantiations in dk_search_<metric>.cu.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dk_kernels.cuh"

namespace {

inline uint32_t align_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// Lay out one query's shared-memory state; returns its size in bytes.
uint32_t plan_query_smem(SearchParams& P, bool pq, bool with_hash) {
  uint32_t off = 0;
  auto take = [&](uint32_t bytes) {
    const uint32_t o = off;
    off = align_up(off + bytes, 16);
    return o;
  };
  P.off_query = take(align_up(P.dim, 8) * 4);
  P.off_table = take(pq ? P.pq_chunks * 256u * 4u : 0u);
  P.off_qd0 = take(P.cap * 4);
  P.off_qi0 = take(P.cap * 4);
  P.off_qd1 = take(P.cap * 4);
  P.off_qi1 = take(P.cap * 4);
  P.off_cand_id = take(P.list_cap * 4);
  P.off_cand_d = take(P.list_cap * 4);
  P.off_new_d = take(P.list_cap * 4);
  P.off_new_id = take(P.list_cap * 4);
  P.off_misc = take(sizeof(dk::Misc));
  P.off_hash = take(with_hash ? (4u << P.hash_log2) : 0u);
  return off;
}

uint32_t env_u32(const char* name, uint32_t dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return (uint32_t)strtoul(v, nullptr, 10);
}

}  // namespace

int32_t dk_launch_search(const dk_index* ix, int32_t strategy, const float* queries,
                         uint64_t qstride, uint32_t nq, uint32_t k, uint32_t l, uint32_t beam,
                         uint32_t* ids, float* dists, dk_search_stats* stats,
                         cudaStream_t stream) {
  if (nq == 0) return DK_OK;
  const bool pq = strategy != DK_STRATEGY_FULL_PRECISION;
  SearchParams P{};
  P.vectors = ix->vectors;
  P.adj = ix->adj;
  P.codes = ix->codes;
  P.pivots = ix->pivots;
  P.pivots_cm = ix->pivots_cm;
  P.offsets = ix->offsets;
  P.n = ix->n;
  P.f = ix->f;
  P.dim = ix->dim;
  P.vstride = ix->vstride;
  P.astride = ix->astride;
  P.max_degree = ix->max_degree;
  P.cstride = ix->cstride;
  P.pq_chunks = ix->pq_chunks;
  P.queries = queries;
  P.qstride = qstride;
  P.nq = nq;
  P.k = k;
  P.l = l;
  P.cap = l + ix->f;
  P.beam = beam;
  P.strategy = strategy;
  P.out_ids = ids;
  P.out_dists = dists;
  P.stats = stats;
  P.list_cap = std::max(std::max(beam * ix->max_degree, P.cap), ix->f);

  // Visited-set hash.  |visited| equals the comparison count, which for a given graph grows
  // about linearly with L + F.  The ratio is learned from previous launches on this index
  // (kernels record their largest cmps / (L + F) in mapped host memory); before any launch
  // the prior is half the reference's own upper-bound estimate (scratch.rs:186-193,
  // 1.1 * max_degree * 1.3 * L).  The hash is sized to stay under 3/4 load for the learned
  // ratio plus one hop; a query that needs more re-runs exactly in the bitmap spill pass.
  double ratio = 0.5 * 1.1 * 1.3 * ix->max_degree;
  P.hint = ix->hint_dev;
  if (ix->hint_host) {
    volatile uint32_t* h = ix->hint_host;
    const uint32_t seen = h[0];
    if (seen) {
      h[1] = seen;
      h[0] = 0;
    }
    if (h[1]) ratio = (double)h[1] / 256.0 * 1.15;
  }
  const double est = ratio * (double)P.cap + beam * ix->max_degree + ix->f;
  uint32_t log2h = 9;
  while ((double)(1u << log2h) * 0.75 < est && log2h < 16) ++log2h;
  log2h = env_u32("DK_HASH_LOG2", log2h);
  log2h = std::min<uint32_t>(std::max<uint32_t>(log2h, 6), 20);

  int dev = 0, max_optin = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

  dk::LaunchPlan L{};
  // Kernel choice: one warp per query unless rows are wide (D >= 384) or the beam is wide,
  // where a 128-thread CTA scores more candidates per round.  DK_KERNEL=warp|cta overrides.
  const char* kenv = getenv("DK_KERNEL");
  bool warp = ix->dim < 384 && beam <= 4;
  if (kenv && !strcmp(kenv, "warp")) warp = true;
  if (kenv && !strcmp(kenv, "cta")) warp = false;

  P.hash_log2 = log2h;
  while (true) {
    P.hash_limit = (uint32_t)((1u << P.hash_log2) * 0.75);
    const uint32_t bytes = plan_query_smem(P, pq, true);
    if (warp) {
      P.warp_smem = bytes;
      uint32_t wpc = std::min<uint32_t>(4, (uint32_t)max_optin / std::max<uint32_t>(bytes, 1));
      if (wpc >= 1) {
        L.kind = dk::KernelKind::kWarp;
        L.warps_per_cta = wpc;
        P.smem_bytes = bytes * wpc;
        break;
      }
    } else if (bytes <= (uint32_t)max_optin) {
      L.kind = dk::KernelKind::kCta;
      P.smem_bytes = bytes;
      break;
    }
    if (P.hash_log2 <= 6) {
      dk_set_error(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory (L or PQ too large)");
      return DK_ERR_UNSUPPORTED;
    }
    --P.hash_log2;
  }
  L.p1 = P;

  SearchParams P2 = P;
  P2.hash_limit = 0xFFFFFFFFu;  // the bitmap never fills
  P2.smem_bytes = plan_query_smem(P2, pq, false);
  if (P2.smem_bytes > (uint32_t)max_optin) {
    dk_set_error(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory (L or PQ too large)");
    return DK_ERR_UNSUPPORTED;
  }

  // Spill pass scratch: one bitmap over all ids per spill CTA.
  const uint32_t words = (ix->n + ix->f + 31u) / 32u;
  uint32_t spill_ctas = std::min<uint32_t>(nq, (uint32_t)std::max(1, sms));
  const uint64_t per = (uint64_t)words * 4u;
  const uint64_t budget = 256ull << 20;
  if (per * spill_ctas > budget) spill_ctas = (uint32_t)std::max<uint64_t>(1, budget / per);
  uint32_t* bitmap = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&bitmap), per * spill_ctas, stream);
  if (e != cudaSuccess) {
    dk_set_error(DK_ERR_OUT_OF_MEMORY, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    return DK_ERR_OUT_OF_MEMORY;
  }
  P2.bitmap = bitmap;
  P2.bitmap_words = words;
  L.p2 = P2;
  L.spill_ctas = spill_ctas;

  switch (ix->metric) {
    case DK_METRIC_L2: e = dk_launch_l2(L, pq, stream); break;
    case DK_METRIC_INNER_PRODUCT: e = dk_launch_ip(L, pq, stream); break;
    case DK_METRIC_COSINE: e = dk_launch_cosine(L, pq, stream); break;
    default: e = dk_launch_cosine_normalized(L, pq, stream); break;
  }
  cudaFreeAsync(bitmap, stream);
  if (e != cudaSuccess) {
    dk_set_error(DK_ERR_CUDA, std::string("search launch: ") + cudaGetErrorString(e));
    return DK_ERR_CUDA;
  }
  return DK_OK;
}
