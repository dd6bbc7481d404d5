// Host side of the batched search: shared-memory planning, visited-set sizing, kernel choice,
// occupancy and scratch, then the first pass (warp or CTA kernel) and the spill pass.
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
inline uint64_t align_up64(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

uint32_t env_u32(const char* name, uint32_t dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return (uint32_t)strtoul(v, nullptr, 10);
}

uint32_t log2_at_least(double x, uint32_t lo, uint32_t hi) {
  uint32_t l = lo;
  while (l < hi && (double)(1u << l) < x) ++l;
  return l;
}

int32_t too_big() {
  dk_set_error(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory (L or PQ too large)");
  return DK_ERR_UNSUPPORTED;
}

}  // namespace

namespace dk {

uint32_t plan_query_smem(SearchParams& P, bool pq, bool with_hash) {
  uint32_t off = 0;
  auto take = [&](uint32_t bytes) {
    const uint32_t o = off;
    off = align_up(off + bytes, 16);
    return o;
  };
  P.off_query = take(align_up(P.dim, 16) * 4);
  P.off_table = take(pq ? P.pq_chunks * 256u * 4u : 0u);
  P.off_qd0 = take(P.cap * 4);
  P.off_qi0 = take(P.cap * 4);
  P.off_qd1 = P.single_queue ? P.off_qd0 : take(P.cap * 4);
  P.off_qi1 = P.single_queue ? P.off_qi0 : take(P.cap * 4);
  P.off_cand_id = take(P.list_cap * 4);
  P.off_cand_d = take(P.list_cap * 4);
  P.off_new_d = take(P.list_cap * 4);
  P.off_new_id = take(P.list_cap * 4);
  P.off_misc = take(sizeof(dk::Misc));
  P.off_hash = take(with_hash ? (4u << P.hash_log2) : 0u);
  return off;
}

cudaError_t dispatch(int32_t metric, LaunchPlan& L, int mode, cudaStream_t stream) {
  switch (metric) {
    case DK_METRIC_L2: return dk_launch_l2(L, mode, stream);
    case DK_METRIC_INNER_PRODUCT: return dk_launch_ip(L, mode, stream);
    case DK_METRIC_COSINE: return dk_launch_cosine(L, mode, stream);
    default: return dk_launch_cosine_normalized(L, mode, stream);
  }
}

void base_params(const dk_index* ix, int32_t strategy, uint32_t k, uint32_t l, uint32_t beam,
                 SearchParams& P) {
  P.vectors = ix->vectors;
  P.adj = ix->adj;
  P.codes = ix->codes;
  P.pivots = ix->pivots;
  P.pivots_cm = ix->pivots_cm;
  P.offsets = ix->offsets;
  P.vec_bf16 = ix->vec_bf16;
  P.vec_fp8 = ix->vec_fp8;
  P.bf16_meta = ix->bf16_meta;
  P.fp8_meta = ix->fp8_meta;
  P.lp_stride = ix->lp_stride;
  P.n = ix->n;
  P.f = ix->f;
  P.dim = ix->dim;
  P.vstride = ix->vstride;
  P.astride = ix->astride;
  P.max_degree = ix->max_degree;
  P.cstride = ix->cstride;
  P.pq_chunks = ix->pq_chunks;
  P.k = k;
  P.l = l;
  P.cap = l + ix->f;
  P.beam = beam;
  P.strategy = strategy;
  // One hop's candidates (or the start points).  The rerank of the queue (up to L + F entries)
  // uses the queue's second buffer, free once the last merge is done.
  P.list_cap = std::max(beam * ix->max_degree, ix->f);
}

void visited_estimates(dk_index* ix, const SearchParams& P, double& est, double& est_mean,
                       bool absorb) {
  // |visited| equals the comparison count, which for a given graph grows about linearly with
  // L + F.  The largest and the mean ratio are learned from previous launches on this index
  // (see dk_index::hint_dev); before any launch the prior is half the reference's own
  // upper-bound estimate (scratch.rs:186-193, 1.1 * max_degree * 1.3 * L).  Only performance
  // depends on these sizes: a query whose visited set outgrows them re-runs exactly in the
  // bitmap spill pass.
  double ratio = 0.5 * 1.1 * 1.3 * ix->max_degree;
  double mean_ratio = ratio;
  {
    if (absorb) {
      volatile uint32_t* h = ix->hint_stage;  // written by the previous launch's async copy
      const uint32_t seen = h[0], sum = h[1], cnt = h[2];
      if (seen) ix->hint_max = seen;
      if (cnt) ix->hint_mean = (uint32_t)(((uint64_t)sum + cnt - 1) / cnt);
    }
    if (ix->hint_max) ratio = (double)ix->hint_max / 256.0 * 1.15;
    if (ix->hint_mean) mean_ratio = (double)ix->hint_mean / 256.0;
  }
  est = ratio * (double)P.cap + P.beam * ix->max_degree + ix->f;
  est_mean = mean_ratio * (double)P.cap + P.beam * ix->max_degree + ix->f;
}

int32_t plan_warp(dk_index* ix, SearchParams& P, LaunchPlan& L, int mode, double est,
                  double est_mean, uint64_t max_warps, cudaStream_t stream) {
  const bool pq = mode == kModePQ;
  int dev = 0, max_optin = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // Shared level: room for 1.3x the mean visited set at <= 3/4 load, within a per-warp
  // shared-memory budget; the global level takes what a longer search adds.
  P.hash_log2 = 0;
  // One queue buffer: the merge works in place, and a rerank's list (up to L + F ids and
  // distances) goes into the shared visited level, which the search no longer needs by then.
  P.single_queue = 1u;
  const uint32_t base = plan_query_smem(P, pq, false);
  // Per-warp budget (measured on the 1M x 128 and 2M x 384 workloads): the kernels are fastest
  // with a shared level holding ~1.1x the mean visited set at load 3/4 (12-32 KB per warp),
  // which keeps nearly every probe out of the global level, rather than with more resident
  // warps (2M x 384 at L = 512: 342k QPS with 20 KB per warp, 371k with 28 KB); beyond 32 KB
  // see below.  PQ traversal keeps its 32 KB-class ADC table beside a level sized the same
  // way, up to 96 KB per warp: with a 1 KB level the 1M x 128 Hybrid search at L = 400 sent
  // nearly every probe to the global level (4.8 GB of DRAM writes per launch) and ran 145k QPS;
  // with a 74 KB slice, 186k.  DK_WARP_SMEM overrides.
  uint32_t dflt = 12288;
  if (mode == kModePQ) {
    dflt = std::min<uint32_t>(base + (uint32_t)(4.0 * est_mean * 1.1 / 0.75), 98304);
  } else {
    dflt = base + (uint32_t)(4.0 * est_mean * 1.1 / 0.75);
    // A visited set too large for a 32 KB slice goes mostly to the global level whatever the
    // slice, and then more resident warps pay more than a larger shared level: 20M x 384 at
    // L = 512 (8.4k visited ids) ran 150k QPS with 32 KB per warp, 131k with 48 KB, 185k with
    // 24 KB, 233k with 16 KB and 245k with 14 KB (16 warps per SM, the register limit at 128
    // registers).
    dflt = dflt > 32768 ? std::max<uint32_t>(14336, base + 2048) : std::max<uint32_t>(dflt, 12288);
  }
  const uint32_t budget = std::max<uint32_t>(env_u32("DK_WARP_SMEM", dflt), base + 1024);
  uint32_t slots = align_up((uint32_t)(est_mean * 1.3 / 0.75) + 1, 32);
  slots = std::min<uint32_t>(slots, ((budget - base) / 4) & ~31u);
  if (const uint32_t hl = env_u32("DK_HASH_LOG2", 0)) slots = 1u << std::min<uint32_t>(hl, 16);
  slots = std::max<uint32_t>(slots, 64);
  // The rerank list needs 2 (L + F) slots; a second queue buffer would have taken as much.
  if (strategy_reranks(P.strategy)) slots = std::max<uint32_t>(slots, align_up(2u * P.cap, 32));
  P.hash_slots = slots;
  P.hash_limit = slots * 3 / 4;
  // One global round trip per adjacency row for every mode: measured faster than one per
  // 32-id round for FP32 too (1M x 128 L = 50 +2.3 %, 2M x 384 L = 512 +4 %, 20M x 384
  // L = 512 +6.6 %).  DK_ROW_PROBES=0 restores one round trip per round.
  P.row_probes = env_u32("DK_ROW_PROBES", 1u) ? 1u : 0u;
  P.hash_log2 = log2_at_least(slots, 6, 16);  // only sizes the shared-memory carve-up below
  P.warp_smem = base + align_up(slots * 4, 16);
  plan_query_smem(P, pq, false);
  P.off_hash = base;
  if (P.warp_smem > (uint32_t)max_optin) return too_big();
  // Global level: open addressing probed one CAS per step, so its load stays low (a warp waits
  // for the longest of its 32 lanes' probe chains).  DK_GTABLE_LOAD (percent) overrides.
  const double gload = std::min(0.75, std::max(0.05, env_u32("DK_GTABLE_LOAD", 75) / 100.0));
  P.gtable_log2 = log2_at_least(std::max(est, 2.0 * P.hash_limit) / gload, 10, 22);
  P.gtable_log2 = std::min<uint32_t>(std::max<uint32_t>(env_u32("DK_GTABLE_LOG2", P.gtable_log2), 6), 24);
  P.gtable_limit = (uint32_t)((1u << P.gtable_log2) * gload);
  // Warps per CTA: the packing with the most resident warps per SM.
  int best_warps = 0;
  for (uint32_t wpc : {4u, 2u, 1u}) {
    if (P.warp_smem * wpc > (uint32_t)max_optin) continue;
    LaunchPlan Q{};
    Q.kind = KernelKind::kWarp;
    Q.p1 = P;
    Q.score_u = L.score_u;
    Q.warps_per_cta = wpc;
    Q.query_only = true;
    const cudaError_t e = dispatch(ix->metric, Q, mode, stream);
    if (e != cudaSuccess) {
      dk_set_error(DK_ERR_CUDA, std::string("occupancy query: ") + cudaGetErrorString(e));
      return DK_ERR_CUDA;
    }
    if (Q.blocks_per_sm * (int)wpc > best_warps) {
      best_warps = Q.blocks_per_sm * (int)wpc;
      L.warps_per_cta = wpc;
      L.blocks_per_sm = Q.blocks_per_sm;
    }
  }
  if (best_warps == 0) return too_big();
  const uint64_t want = (max_warps + L.warps_per_cta - 1) / L.warps_per_cta;
  L.grid = (uint32_t)std::min<uint64_t>(want, (uint64_t)L.blocks_per_sm * (uint64_t)sms);
  return DK_OK;
}

}  // namespace dk

int32_t dk_launch_search(dk_index* ix, int32_t strategy, const float* queries,
                         uint64_t qstride, uint32_t nq, uint32_t k, uint32_t l, uint32_t beam,
                         uint32_t* ids, float* dists, dk_search_stats* stats,
                         cudaStream_t stream, const SearchRecord* record, bool keep_start) {
  if (nq == 0) return DK_OK;
  const int mode = mode_of_strategy(strategy);
  const bool pq = mode == kModePQ;
  SearchParams P{};
  dk::base_params(ix, strategy, k, l, beam, P);
  P.queries = queries;
  P.qstride = qstride;
  P.nq = nq;
  P.out_ids = ids;
  P.out_dists = dists;
  P.stats = stats;
  P.hint = ix->hint_dev;
  P.keep_start = keep_start ? 1u : 0u;
  if (record) {
    P.rec_ids = record->ids;
    P.rec_d = record->dists;
    P.rec_cap = record->cap;
  }
  double est = 0, est_mean = 0;
  dk::visited_estimates(ix, P, est, est_mean);

  int dev = 0, max_optin = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);

  // Kernel choice: one warp per query unless the beam is wide (> 4), where a 128-thread CTA
  // scores more candidates per round.  Wide rows stay on the warp kernel too: on 1M x 768 at
  // L = 256 it ran 5.7x faster than the CTA kernel, whose shared visited hash leaves one query
  // per SM.  DK_KERNEL=warp|cta overrides.
  const char* kenv = getenv("DK_KERNEL");
  bool warp = beam <= 4;
  if (kenv && !strcmp(kenv, "warp")) warp = true;
  if (kenv && !strcmp(kenv, "cta")) warp = false;

  dk::LaunchPlan L{};
  L.score_u = env_u32("DK_SCORE_U", mode == kModeFP32 ? 4u : 2u);
  uint64_t gtable_bytes = 0;
  cudaError_t e = cudaSuccess;
  if (warp) {
    L.kind = dk::KernelKind::kWarp;
    const int32_t rc = dk::plan_warp(ix, P, L, mode, est, est_mean, nq, stream);
    if (rc != DK_OK) return rc;
    gtable_bytes = (uint64_t)L.grid * L.warps_per_cta * (4ull << P.gtable_log2);
  } else {
    L.kind = dk::KernelKind::kCta;
    uint32_t log2h = log2_at_least(est / 0.75, 9, 16);
    log2h = env_u32("DK_HASH_LOG2", log2h);
    P.hash_log2 = std::min<uint32_t>(std::max<uint32_t>(log2h, 6), 20);
    while (true) {
      P.hash_limit = (uint32_t)((1u << P.hash_log2) * 0.75);
      P.smem_bytes = dk::plan_query_smem(P, pq, true);
      if (P.smem_bytes <= (uint32_t)max_optin) break;
      if (P.hash_log2 <= 6) return too_big();
      --P.hash_log2;
    }
  }

  SearchParams P2 = P;
  P2.single_queue = 0;  // the spill pass (CTA kernel) merges into its second queue buffer
  P2.hash_limit = 0xFFFFFFFFu;  // the bitmap never fills
  P2.smem_bytes = dk::plan_query_smem(P2, pq, false);
  if (P2.smem_bytes > (uint32_t)max_optin) return too_big();

  // Scratch, one stream-ordered allocation: work counter | global tables | spill bitmaps.
  // Spill pass: up to eight CTAs per SM (it exits at once when nothing spilled; a workload whose
  // visited sets outgrow the shared hash runs mostly here), each with a bitmap, within 256 MiB.
  const uint32_t words = (ix->n + ix->f + 31u) / 32u;
  uint32_t spill_ctas = std::min<uint32_t>(nq, 8u * (uint32_t)std::max(1, sms));
  const uint64_t per = (uint64_t)words * 4u;
  const uint64_t budget = 256ull << 20;
  if (per * spill_ctas > budget) spill_ctas = (uint32_t)std::max<uint64_t>(1, budget / per);
  const uint64_t off_gtable = 256;
  const uint64_t off_bitmap = align_up64(off_gtable + gtable_bytes, 256);
  const uint64_t total = off_bitmap + per * spill_ctas;
  unsigned char* scratch = nullptr;
  e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch), total, ix->pool, stream);
  if (e != cudaSuccess) {
    dk_set_error(DK_ERR_OUT_OF_MEMORY, std::string("scratch allocation: ") + cudaGetErrorString(e));
    return DK_ERR_OUT_OF_MEMORY;
  }
  e = cudaMemsetAsync(scratch, 0, 256, stream);
  P.work_counter = reinterpret_cast<uint32_t*>(scratch);
  P.spill_count = reinterpret_cast<uint32_t*>(scratch) + 1;  // zeroed with the counter
  P.gtable = reinterpret_cast<uint32_t*>(scratch + off_gtable);
  P2.bitmap = reinterpret_cast<uint32_t*>(scratch + off_bitmap);
  P2.spill_count = P.spill_count;
  P2.bitmap_words = words;
  L.p1 = P;
  L.p2 = P2;
  L.spill_ctas = spill_ctas;
  if (e == cudaSuccess) e = dk::dispatch(ix->metric, L, mode, stream);
  cudaFreeAsync(scratch, stream);
  // Stage this launch's visited-size statistics for the next launch's planning, then reset.
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(ix->hint_stage, ix->hint_dev, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ix->hint_dev, 0, 3 * sizeof(uint32_t), stream);
  if (e != cudaSuccess) {
    dk_set_error(DK_ERR_CUDA, std::string("search launch: ") + cudaGetErrorString(e));
    return DK_ERR_CUDA;
  }
  return DK_OK;
}
