// Device code of the batched greedy beam search (sm_100a).
//
// Two kernels run the reference's `search_internal` loop (diskann/src/graph/index.rs:
// 1938-2005) for a batch of queries, each query's state resident in shared memory:
//
//  * k_search_warp — one WARP per query, several queries per CTA, no block barriers.  A
//    hop's work is small (one adjacency row, a few to a few dozen candidates), so the kernel
//    is bound by dependent memory latency; one warp per query keeps many queries in flight
//    per SM and every phase is warp-synchronous (ballots, shuffles, __syncwarp).
//  * k_search_cta — one CTA (128 threads) per query: more lanes per hop for wide beams.  Its
//    bitmap variant is the spill pass (below).
//
// Query state:
//   * the candidate queue (diskann/src/neighbor/queue.rs:68-519): sorted (distance, id) arrays
//     with capacity L + #start points, visited flag in the id's top bit, double-buffered so a
//     hop's candidates merge in one parallel pass;
//   * the visited set (diskann/src/graph/search/scratch.rs:41-48, glue.rs:524-561): an
//     open-addressing u32 hash in shared memory; a query that would load it past 3/4 is
//     abandoned and re-run by the spill pass with an exact bitmap over all ids in global
//     memory, so results never depend on the hash size;
//   * the query vector and, for PQ traversal, the per-query ADC table
//     (diskann-providers/src/model/pq/fixed_chunk_pq_table.rs:149-215).
//
// Full-precision scoring uses 8-lane subgroups: lane s reads float4 pieces at offsets
// 32*b + 4*s of the row, which makes it own exactly accumulator lanes 4s..4s+3 of the
// reference's x86-64-v3 kernel (four f32x8 accumulators over 32-float blocks,
// diskann-vector/src/distance/simd.rs:321-363, 686-745).  The reduction then reproduces
// the reference's rounding sequence bit for bit: (s0+s1)+(s2+s3) lane-wise, masked
// remainder, sum_tree (diskann-wide/src/arch/x86_64/v3/f32x8_.rs:187-212).
//
// Merge: the reference inserts a hop's candidates one by one in adjacency order; `insert`
// (queue.rs:130-171) places an item before existing equal distances, drops it when the queue
// is full and its distance exceeds the last, and evicts the last otherwise.  That is the
// first `cap` entries of the union ordered by (distance, newest first), which the merge
// computes directly: new items are ranked among themselves by (distance ascending, adjacency
// position descending) and placed before old items of equal distance.  NaN distances are
// scored and counted but never inserted (queue.rs:131-135).
#pragma once

#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "dk_internal.cuh"

namespace dk {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;

constexpr uint32_t kVisited = 0x80000000u;
constexpr uint32_t kIdMask = 0x7FFFFFFFu;
constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr int kCtaThreads = 128;

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ----------------------------------------------------------------------------------------
// Visited sets.
// ----------------------------------------------------------------------------------------

struct SmemHashSet {
  uint32_t* slots;
  uint32_t mask;
  uint32_t shift;

  __device__ void clear(uint32_t tid, uint32_t nt) const {
    for (uint32_t i = tid; i <= mask; i += nt) slots[i] = kEmpty;
  }
  // True if `id` was absent (and is now present).  Callers keep the load at most 3/4, so
  // the probe always ends.  Linear probing over 16-byte buckets of four slots, one shared
  // read per bucket; slots fill in probe order and are never removed, so the first empty slot
  // ends a lookup.  Threads may insert the same id at once: a lost CAS re-reads the bucket.
  __device__ bool insert(uint32_t id) const {
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(slots);
    const uint32_t bmask = mask >> 2;
    uint32_t b = ((id * 2654435761u) >> shift) >> 2;
    while (true) {
      uint32_t v[4];
      asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                   : "r"(base + 16u * b));
      if (v[0] == id || v[1] == id || v[2] == id || v[3] == id) return false;
      const uint32_t j = v[0] == kEmpty ? 0u : v[1] == kEmpty ? 1u : v[2] == kEmpty ? 2u
                                                              : v[3] == kEmpty ? 3u : 4u;
      if (j < 4u) {
        const uint32_t old = atomicCAS(&slots[4u * b + j], kEmpty, id);
        if (old == kEmpty) return true;
        if (old == id) return false;
        continue;  // another id took the slot: read the bucket again
      }
      b = (b + 1u) & bmask;
    }
  }
};

struct BitmapSet {
  uint32_t* words;
  uint32_t nwords;

  __device__ void clear(uint32_t tid, uint32_t nt) const {
    for (uint32_t i = tid; i < nwords; i += nt) words[i] = 0u;
  }
  __device__ bool insert(uint32_t id) const {
    const uint32_t bit = 1u << (id & 31u);
    const uint32_t old = atomicOr(&words[id >> 5], bit);
    return (old & bit) == 0u;
  }
};

// Exact visited set of one warp, in two levels: a small shared-memory hash takes the first
// `slimit` ids; after it holds that many it never changes again, and every later new id goes
// to a larger open-addressing hash in global memory owned by the warp.  Because the shared
// level is frozen once full, "absent from the shared level" followed by a global probe is an
// exact membership test.  The warp inserts up to 32 distinct ids at a time (adjacency lists
// are de-duplicated when the index is built and beam rows are filtered one after another);
// the counters are warp-uniform registers updated from ballots.
struct WarpVisited {
  uint32_t* s;
  uint32_t ssize, slimit;  // shared level: any size (multiply-high hashing), at most slimit ids
  uint32_t* g;
  uint32_t gmask, gshift;
  uint32_t scount = 0;  // ids in the shared level
  uint32_t gcount = 0;  // ids in the global level

  __device__ __forceinline__ void reset(uint32_t lane) {
    for (uint32_t i = lane; i < ssize; i += 32u) s[i] = kEmpty;
    scount = 0u;
    gcount = 0u;
  }
  __device__ __forceinline__ uint32_t next(uint32_t h) const { return h + 1 == ssize ? 0u : h + 1; }
  // Shared-level half of an insert.  Every lane calls; lanes with `want` test `id`.  Returns
  // true if the id was new and went into the shared level; `global` is set when the id is not
  // in the frozen shared level and must be tested against the global level.
  // The shared level probes linearly, four slots (one 16-byte bucket) per read: slots fill in
  // probe order and nothing is ever removed, so the first empty slot ends a lookup.
  __device__ __forceinline__ bool shared_step(bool want, uint32_t id, bool& global) {
    volatile uint32_t* vs = s;
    bool present = false;
    const uint32_t nbk = ssize >> 2;
    uint32_t b = __umulhi(id * 2654435761u, nbk);
    uint32_t h = 0;
    if (want) {
      const uint32_t base = (uint32_t)__cvta_generic_to_shared(s);
      while (true) {
        uint32_t v0, v1, v2, v3;
        asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(v0), "=r"(v1), "=r"(v2), "=r"(v3)
                     : "r"(base + 16u * b));
        if (v0 == id || v1 == id || v2 == id || v3 == id) { present = true; break; }
        if (v0 == kEmpty) { h = 4u * b; break; }
        if (v1 == kEmpty) { h = 4u * b + 1u; break; }
        if (v2 == kEmpty) { h = 4u * b + 2u; break; }
        if (v3 == kEmpty) { h = 4u * b + 3u; break; }
        b = b + 1u == nbk ? 0u : b + 1u;
      }
    }
    const bool absent = want && !present;
    const uint32_t m = __ballot_sync(kFull, absent);
    const uint32_t rank = __popc(m & lanemask_lt());
    const uint32_t room = scount < slimit ? slimit - scount : 0u;
    bool fresh = false;
    if (absent && rank < room) {
      // Take the first empty slot from the probe's end; other lanes only add other ids.
      while (atomicCAS(&s[h], kEmpty, id) != kEmpty) {
        do { h = next(h); } while (vs[h] != kEmpty);
      }
      fresh = true;
    }
    scount += min((uint32_t)__popc(m), room);
    global = absent && rank >= room;
    return fresh;
  }

  __device__ __forceinline__ uint32_t ghash(uint32_t id) const {
    return ((id ^ 0x5bd1e995u) * 0x9E3779B1u) >> gshift;
  }

  // Global-level probe continued from the id's home slot, whose CAS returned `old`: true if
  // `id` was new.
  __device__ __forceinline__ bool global_finish(uint32_t id, uint32_t old) {
    uint32_t hg = ghash(id);
    while (true) {
      if (old == kEmpty) return true;
      if (old == id) return false;
      hg = (hg + 1) & gmask;
      old = atomicCAS(&g[hg], kEmpty, id);  // one round trip per step
    }
  }

  // Every lane calls; lanes with `want` test-and-insert their `id`.  True if it was new.
  __device__ __forceinline__ bool insert(bool want, uint32_t id) {
    bool global;
    bool fresh = shared_step(want, id, global);
    if (__any_sync(kFull, global)) {
      if (global) {
        fresh = global_finish(id, atomicCAS(&g[ghash(id)], kEmpty, id));
      }
      gcount += __popc(__ballot_sync(kFull, global && fresh));
    }
    return fresh;
  }

  // The ids of one adjacency row, up to 128, lane `l` holding entries l, l+32, l+64, l+96:
  // the shared level is updated round by round (in row order), then the first global-level
  // probes of all rounds are issued together, so a row costs one global round trip, not one
  // per round.  Ids of one row are distinct.
  __device__ __forceinline__ void insert_row(const uint32_t (&id)[4], uint32_t deg, uint32_t lane,
                                             bool (&fresh)[4]) {
    bool glob[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      glob[r] = false;
      fresh[r] = false;
      if (32u * r < deg) fresh[r] = shared_step(32u * r + lane < deg, id[r], glob[r]);
    }
    if (__any_sync(kFull, glob[0] || glob[1] || glob[2] || glob[3])) {
      uint32_t old[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) old[r] = glob[r] ? atomicCAS(&g[ghash(id[r])], kEmpty, id[r]) : kEmpty;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (glob[r]) fresh[r] = global_finish(id[r], old[r]);
        gcount += __popc(__ballot_sync(kFull, glob[r] && fresh[r]));
      }
    }
  }
};

// ----------------------------------------------------------------------------------------
// Small helpers.
// ----------------------------------------------------------------------------------------

// Exclusive prefix of a 0/1 flag over the block, in thread order; `total` = block sum.
template <int NT>
__device__ __forceinline__ uint32_t block_scan(bool flag, uint32_t* warp_sums, uint32_t& total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t b = __ballot_sync(kFull, flag);
  const uint32_t pre = __popc(b & lanemask_lt());
  if (lane == 0) warp_sums[warp] = __popc(b);
  __syncthreads();
  uint32_t base = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) {
    const uint32_t s = warp_sums[w];
    base += (w < (int)warp) ? s : 0u;
    tot += s;
  }
  __syncthreads();
  total = tot;
  return base + pre;
}

// Entries of sorted a[0..n) that are < d / <= d.
__device__ __forceinline__ uint32_t count_less(const float* a, uint32_t n, float d) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < d) lo = mid + 1; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ uint32_t count_less_equal(const float* a, uint32_t n, float d) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= d) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// ----------------------------------------------------------------------------------------
// Distances.
// ----------------------------------------------------------------------------------------

__device__ __forceinline__ float tree4(float u0, float u1, float u2, float u3) {
  // Each lane holds q_i = t_i + t_{i+4} (i = 0..3); sum_tree: (q0+q2) + (q1+q3).
  const float d0 = u0 + u2, d1 = u1 + u3;
  return d0 + d1;
}

template <int METRIC>
__device__ __forceinline__ void acc4(float4 a, float4 v, float* acc) {
  if (METRIC == DK_METRIC_L2) {
    const float c0 = a.x - v.x, c1 = a.y - v.y, c2 = a.z - v.z, c3 = a.w - v.w;
    acc[0] = __fmaf_rn(c0, c0, acc[0]);
    acc[1] = __fmaf_rn(c1, c1, acc[1]);
    acc[2] = __fmaf_rn(c2, c2, acc[2]);
    acc[3] = __fmaf_rn(c3, c3, acc[3]);
  } else {
    acc[0] = __fmaf_rn(a.x, v.x, acc[0]);
    acc[1] = __fmaf_rn(a.y, v.y, acc[1]);
    acc[2] = __fmaf_rn(a.z, v.z, acc[2]);
    acc[3] = __fmaf_rn(a.w, v.w, acc[3]);
  }
}

// Row elements as floats: FP32 rows directly, FP16 rows (the diskann-inmem f16 layer) through
// the exact f16 -> f32 conversion.  ld4 reads elements 4i..4i+3, ld1 element i.
__device__ __forceinline__ float4 ld4(const float* r, uint32_t i) {
  return __ldg(reinterpret_cast<const float4*>(r) + i);
}
__device__ __forceinline__ float4 ld4(const __half* r, uint32_t i) {
  const uint2 w = __ldg(reinterpret_cast<const uint2*>(r) + i);
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float ld1(const float* r, uint32_t i) { return __ldg(r + i); }
__device__ __forceinline__ float ld1(const __half* r, uint32_t i) { return __half2float(r[i]); }

// Distances of U rows to the shared-memory query `q` (zero padded to a multiple of 8
// floats) computed by the 8 lanes of a subgroup; rows are padded to 4 elements and aligned to
// 4 elements.  All 8 lanes return the results.  L2, inner product, normalised cosine.  FP16
// rows take the same path: the reference's f32-by-f16 kernels (simd.rs:1121-1156, 1878-1912,
// Strategy4x2) feed the same vectors to the same accumulators in the same order as
// Strategy4x1, after an exact conversion.
template <int METRIC, int DIM, int U, class RowT = float>
__device__ __forceinline__ void subgroup_distances(const RowT* const (&rows)[U],
                                                   const float* __restrict__ q, uint32_t dim_rt,
                                                   uint32_t s, unsigned gmask, float (&out)[U]) {
  const uint32_t dim = DIM > 0 ? (uint32_t)DIM : dim_rt;
  const uint32_t rem = dim & 7u;
  const uint32_t full = dim - rem;
  const float4* q4 = reinterpret_cast<const float4*>(q);
  float acc[U][4];
#pragma unroll
  for (int u = 0; u < U; ++u) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0f;
  if (DIM > 0 && DIM % 32 == 0) {
    // The 16-byte pieces of the U rows are requested CH blocks at a time (at most 16 pieces
    // per lane in flight) before their FMAs, so a row of up to 16·32 floats costs one memory
    // latency and a 768-float row two.  The FMAs run in the reference's block order.
    constexpr int NB = DIM > 0 ? DIM / 32 : 1;
    constexpr int CH = (16 / U) < NB ? (16 / U) : NB;
#pragma unroll
    for (int c0 = 0; c0 < NB; c0 += CH) {
      float4 v[U][CH];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int j = 0; j < CH; ++j)
          if (c0 + j < NB) v[u][j] = ld4(rows[u], 8 * (c0 + j) + s);
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        if (c0 + j >= NB) break;
        const float4 a = q4[8 * (c0 + j) + s];
#pragma unroll
        for (int u = 0; u < U; ++u) acc4<METRIC>(a, v[u][j], acc[u]);
      }
    }
  } else {
#pragma unroll 4
    for (uint32_t base = 4u * s; base < full; base += 32u) {
      const float4 a = q4[base >> 2];
      float4 v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = ld4(rows[u], base >> 2);
#pragma unroll
      for (int u = 0; u < U; ++u) acc4<METRIC>(a, v[u], acc[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      acc[u][i] += __shfl_xor_sync(gmask, acc[u][i], 2, 8);  // s0+s1 / s2+s3
      acc[u][i] += __shfl_xor_sync(gmask, acc[u][i], 4, 8);  // (s0+s1)+(s2+s3)
    }
  if (rem) {
    const uint32_t e = full + 4u * (s & 1u);
    if (e < dim) {
      const float4 a = q4[e >> 2];
      const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const float4 v = ld4(rows[u], e >> 2);
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          if (e + i < dim) {
            if (METRIC == DK_METRIC_L2) {
              const float c = av[i] - vv[i];
              acc[u][i] = __fmaf_rn(c, c, acc[u][i]);
            } else {
              acc[u][i] = __fmaf_rn(av[i], vv[i], acc[u][i]);
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[u][i] += __shfl_xor_sync(gmask, acc[u][i], 1, 8);
    const float r = tree4(acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
    out[u] = METRIC == DK_METRIC_L2 ? r : (METRIC == DK_METRIC_INNER_PRODUCT ? -r : 1.0f - r);
  }
}

// Cosine (CosineStateless, simd.rs:2430-2460) on x86-64-v3 runs Strategy2x4
// (simd.rs:422-482): three accumulators (x*x, y*y, x*y) in two sets, full 8-wide vectors in
// order alternating between the sets (vector k -> set k % 2), combined as set0 + set1, then a
// masked remainder.  Lane s of the subgroup is SIMD lane s: it runs both sets' FMA chains for
// element 8k + s.  sum (simd.rs:2327-2361): sum_tree of each accumulator (xor 4, 2, 1 over the
// 8 lanes gives (t_i + t_{i+4}), then (q0 + q2) + (q1 + q3)); zero similarity if a norm is
// below f32::MIN_POSITIVE, else clamp(prod / (sqrt(nx) * sqrt(ny))); distance 1 - similarity.
template <int DIM, class RowT = float>
__device__ __forceinline__ float subgroup_cosine(const RowT* __restrict__ row,
                                                 const float* __restrict__ q, uint32_t dim_rt,
                                                 uint32_t s, unsigned gmask) {
  const uint32_t dim = DIM > 0 ? (uint32_t)DIM : dim_rt;
  const uint32_t nvec = dim >> 3;
  float x0 = 0.f, y0 = 0.f, p0 = 0.f, x1 = 0.f, y1 = 0.f, p1 = 0.f;
  uint32_t k = 0;
#pragma unroll 8
  for (; k + 1u < nvec; k += 2u) {
    const float b0 = ld1(row, 8u * k + s), b1 = ld1(row, 8u * k + 8u + s);
    const float a0 = q[8u * k + s], a1 = q[8u * k + 8u + s];
    x0 = __fmaf_rn(a0, a0, x0);
    y0 = __fmaf_rn(b0, b0, y0);
    p0 = __fmaf_rn(a0, b0, p0);
    x1 = __fmaf_rn(a1, a1, x1);
    y1 = __fmaf_rn(b1, b1, y1);
    p1 = __fmaf_rn(a1, b1, p1);
  }
  if (k < nvec) {
    const float b0 = ld1(row, 8u * k + s), a0 = q[8u * k + s];
    x0 = __fmaf_rn(a0, a0, x0);
    y0 = __fmaf_rn(b0, b0, y0);
    p0 = __fmaf_rn(a0, b0, p0);
  }
  float tx = x0 + x1, ty = y0 + y1, tp = p0 + p1;
  if (s < (dim & 7u)) {
    const float b = ld1(row, 8u * nvec + s), a = q[8u * nvec + s];
    tx = __fmaf_rn(a, a, tx);
    ty = __fmaf_rn(b, b, ty);
    tp = __fmaf_rn(a, b, tp);
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    tx += __shfl_xor_sync(gmask, tx, o, 8);
    ty += __shfl_xor_sync(gmask, ty, o, 8);
    tp += __shfl_xor_sync(gmask, tp, o, 8);
  }
  const float denom = __fmul_rn(__fsqrt_rn(tx), __fsqrt_rn(ty));
  float sim;
  if (tx < 1.17549435e-38f || ty < 1.17549435e-38f) sim = 0.0f;
  else sim = fmaxf(-1.0f, fminf(1.0f, __fdiv_rn(tp, denom)));
  return 1.0f - sim;
}

// Score candidates ids[0..count) into d[...] with subgroup `sg` of `nsub` subgroups; U rows
// per subgroup are loaded together.  Lanes of a subgroup must be converged.
template <class RowT>
__device__ __forceinline__ const RowT* row_of(const SearchParams& P, uint32_t id);
template <>
__device__ __forceinline__ const float* row_of<float>(const SearchParams& P, uint32_t id) {
  return P.vectors + (size_t)id * P.vstride;
}
template <>
__device__ __forceinline__ const __half* row_of<__half>(const SearchParams& P, uint32_t id) {
  return reinterpret_cast<const __half*>(P.raw + (size_t)id * P.raw_stride);
}

template <int METRIC, int DIM, int U, class RowT = float>
__device__ __forceinline__ void score_fp(const SearchParams& P, const float* q,
                                         const uint32_t* ids, float* d, uint32_t count,
                                         uint32_t sg, uint32_t nsub, uint32_t s, unsigned gmask) {
  // Wide rows (one per subgroup per round, so a hop takes several rounds): the rows scored
  // after the first round are requested into L2 first (no registers held), so the later rounds
  // find them on chip instead of each waiting a full memory latency.  Measured on 2M x 384
  // rows: +9 % at L = 128, +11 % at L = 512; with four 128-float rows per subgroup per round
  // (1M x 128) the prefetches delayed the first round and cost 12 %, so narrow rows skip it.
  if constexpr (sizeof(RowT) == 4 && U == 1) {
    const uint32_t first = METRIC == DK_METRIC_COSINE ? nsub : nsub * U;
    if (count > first) {
      const uint32_t lines = (P.vstride * 4u + 127u) / 128u;
      const uint32_t total = (count - first) * lines;
      for (uint32_t e = sg * 8u + s; e < total; e += nsub * 8u) {
        const float* r = P.vectors + (size_t)ids[first + e / lines] * P.vstride + (e % lines) * 32u;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(r));
      }
    }
  }
  if (METRIC == DK_METRIC_COSINE) {
    for (uint32_t i = sg; i < count; i += nsub) {
      const float r = subgroup_cosine<DIM>(row_of<RowT>(P, ids[i]), q, P.dim, s, gmask);
      if (s == 0) d[i] = r;
    }
    return;
  }
  const uint32_t step = nsub * U;
  for (uint32_t base = 0; base < count; base += step) {
    const RowT* rows[U];
    uint32_t idx[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      idx[u] = base + sg + u * nsub;
      const uint32_t j = idx[u] < count ? idx[u] : count - 1;  // a valid row; result unused
      rows[u] = row_of<RowT>(P, ids[j]);
    }
    float out[U];
    subgroup_distances<METRIC, DIM, U>(rows, q, P.dim, s, gmask, out);
    if (s == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (idx[u] < count) d[idx[u]] = out[u];
    }
  }
}

// Integer rows (the diskann-inmem u8 / i8 layers): the reference accumulates x*x, y*y, x*y or
// (x-y)^2 exactly in i32 lanes (simd.rs:1192-1227, 1370-1405, 1947-1981, 2109-2145,
// 2790-2829, 2996-3035) and converts the sums to f32 once, so the order of the additions does
// not matter.  Lane s of a subgroup takes 4-byte words s, s+8, ... of the row and the packed
// query (both zero padded) with dp4a; L2 = xx + yy - 2xy in 64-bit, exact.  The f32 post-ops
// are the reference's: L2 the sum, inner product its negation, cosine 1 - clamp(xy / (sqrt(xx)
// sqrt(yy))) with zero similarity below f32::MIN_POSITIVE (simd.rs:2327-2363).  Exact while
// no i32 sum of the reference wraps (dim <= 33,000 for u8).
template <int METRIC, bool SIGNED>
__device__ __forceinline__ void score_int(const SearchParams& P, const float* q,
                                          const uint32_t* ids, float* d, uint32_t count,
                                          uint32_t sg, uint32_t nsub, uint32_t s, unsigned gmask) {
  const uint32_t* qw = reinterpret_cast<const uint32_t*>(q);
  const uint32_t nw = (P.dim + 3u) >> 2;
  for (uint32_t i = sg; i < count; i += nsub) {
    const uint32_t* row = reinterpret_cast<const uint32_t*>(P.raw + (size_t)ids[i] * P.raw_stride);
    long long xx, yy, xy;
    if (SIGNED) {
      int a2 = 0, b2 = 0, ab = 0;
      for (uint32_t w = s; w < nw; w += 8u) {
        const int a = (int)qw[w], b = (int)__ldg(row + w);
        a2 = __dp4a(a, a, a2);
        b2 = __dp4a(b, b, b2);
        ab = __dp4a(a, b, ab);
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        a2 += __shfl_xor_sync(gmask, a2, o, 8);
        b2 += __shfl_xor_sync(gmask, b2, o, 8);
        ab += __shfl_xor_sync(gmask, ab, o, 8);
      }
      xx = a2;
      yy = b2;
      xy = ab;
    } else {
      unsigned a2 = 0u, b2 = 0u, ab = 0u;
      for (uint32_t w = s; w < nw; w += 8u) {
        const unsigned a = qw[w], b = __ldg(row + w);
        a2 = __dp4a(a, a, a2);
        b2 = __dp4a(b, b, b2);
        ab = __dp4a(a, b, ab);
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) {
        a2 += __shfl_xor_sync(gmask, a2, o, 8);
        b2 += __shfl_xor_sync(gmask, b2, o, 8);
        ab += __shfl_xor_sync(gmask, ab, o, 8);
      }
      xx = a2;
      yy = b2;
      xy = ab;
    }
    if (s != 0) continue;
    float r;
    if (METRIC == DK_METRIC_L2) {
      r = __ll2float_rn(xx + yy - 2 * xy);
    } else if (METRIC == DK_METRIC_INNER_PRODUCT) {
      r = -__ll2float_rn(xy);
    } else {  // cosine; the layers map CosineNormalized to cosine for integer data
      const float nx = __ll2float_rn(xx), ny = __ll2float_rn(yy), p = __ll2float_rn(xy);
      const float denom = __fmul_rn(__fsqrt_rn(nx), __fsqrt_rn(ny));
      float sim;
      if (nx < 1.17549435e-38f || ny < 1.17549435e-38f) sim = 0.0f;
      else sim = fmaxf(-1.0f, fminf(1.0f, __fdiv_rn(p, denom)));
      r = 1.0f - sim;
    }
    d[i] = r;
  }
}

// Low-precision candidate scoring (BF16 rows, or FP8-E4M3 rows times a per-row scale), FP32
// accumulation.  Lane s of a subgroup reads 16-byte pieces s, s+8, s+16, ... of each row
// (8 BF16 or 16 FP8 elements per piece); partial sums meet in a butterfly over the 8 lanes.
// These distances steer the traversal only: the strategies re-rank with exact FP32 rows.
__device__ __forceinline__ void bf16x8(const uint4 w, float (&x)[8]) {
  const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    x[2 * i] = __uint_as_float(ws[i] << 16);
    x[2 * i + 1] = __uint_as_float(ws[i] & 0xFFFF0000u);
  }
}

__device__ __forceinline__ void fp8x16(const uint4 w, float (&x)[16]) {
  const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const __nv_fp8x2_storage_t pair = (__nv_fp8x2_storage_t)((ws[i] >> (16 * h)) & 0xFFFFu);
      const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2(pair, __NV_E4M3);
      const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&hr));
      x[4 * i + 2 * h] = f.x;
      x[4 * i + 2 * h + 1] = f.y;
    }
  }
}

// Low-precision distance from the row's dot product with the query and its (scale, norm):
// L2 |q|^2 + norm - 2 s (q.x); inner product -s (q.x); normalised cosine 1 - s (q.x); cosine
// 1 - clamp(s (q.x) / (|q| sqrt(norm))), similarity 0 if a norm is below f32::MIN_POSITIVE.
template <int METRIC>
__device__ __forceinline__ float lp_distance(float dot, float2 meta, float qq) {
  const float sd = meta.x * dot;
  if (METRIC == DK_METRIC_L2) return __fmaf_rn(-2.0f, sd, qq + meta.y);
  if (METRIC == DK_METRIC_INNER_PRODUCT) return -sd;
  if (METRIC == DK_METRIC_COSINE_NORMALIZED) return 1.0f - sd;
  if (qq < 1.17549435e-38f || meta.y < 1.17549435e-38f) return 1.0f;
  return 1.0f - fmaxf(-1.0f, fminf(1.0f, sd / (sqrtf(qq) * sqrtf(meta.y))));
}

// |q|^2 over the pieces lane s of a subgroup owns (pieces s, s+8, ...), summed over the 8 lanes.
template <uint32_t kPer>
__device__ __forceinline__ float subgroup_qq(const float* q, uint32_t pieces, uint32_t s,
                                            unsigned gmask) {
  float qq = 0.0f;
  for (uint32_t p = s; p < pieces; p += 8u) {
    const float4* q4 = reinterpret_cast<const float4*>(q + p * kPer);
#pragma unroll
    for (uint32_t i = 0; i < kPer / 4; ++i) {
      const float4 t = q4[i];
      qq = __fmaf_rn(t.x, t.x, qq);
      qq = __fmaf_rn(t.y, t.y, qq);
      qq = __fmaf_rn(t.z, t.z, qq);
      qq = __fmaf_rn(t.w, t.w, qq);
    }
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) qq += __shfl_xor_sync(gmask, qq, o, 8);
  return qq;
}

// Dot product of one 16-byte piece of a low-precision row with the matching query floats.
template <int MODE>
__device__ __forceinline__ float piece_dot(uint4 w, const float* qp, float acc) {
  constexpr uint32_t kPer = MODE == kModeBF16 ? 8u : 16u;
  float x[kPer];
  if (MODE == kModeBF16) bf16x8(w, *reinterpret_cast<float(*)[8]>(x));
  else fp8x16(w, *reinterpret_cast<float(*)[16]>(x));
  const float4* q4 = reinterpret_cast<const float4*>(qp);
#pragma unroll
  for (uint32_t i = 0; i < kPer / 4; ++i) {
    const float4 t = q4[i];
    acc = __fmaf_rn(t.x, x[4 * i], acc);
    acc = __fmaf_rn(t.y, x[4 * i + 1], acc);
    acc = __fmaf_rn(t.z, x[4 * i + 2], acc);
    acc = __fmaf_rn(t.w, x[4 * i + 3], acc);
  }
  return acc;
}

template <int MODE>
__device__ __forceinline__ const unsigned char* lp_rows(const SearchParams& P) {
  return MODE == kModeBF16 ? reinterpret_cast<const unsigned char*>(P.vec_bf16)
                           : reinterpret_cast<const unsigned char*>(P.vec_fp8);
}

template <int MODE>
__device__ __forceinline__ const float2* lp_meta(const SearchParams& P) {
  return MODE == kModeBF16 ? P.bf16_meta : P.fp8_meta;
}

template <int METRIC, int MODE, int U>
__device__ __forceinline__ void score_lp(const SearchParams& P, const float* q, const uint32_t* ids,
                                         float* d, uint32_t count, uint32_t sg, uint32_t nsub,
                                         uint32_t s, unsigned gmask) {
  constexpr uint32_t kPer = MODE == kModeBF16 ? 8u : 16u;  // elements per 16-byte piece
  const uint32_t pieces = P.lp_stride / kPer;
  const uint32_t row_bytes = P.lp_stride * (MODE == kModeBF16 ? 2u : 1u);
  const unsigned char* base = lp_rows<MODE>(P);
  const float2* meta = lp_meta<MODE>(P);
  const float qq = (METRIC == DK_METRIC_L2 || METRIC == DK_METRIC_COSINE)
                       ? subgroup_qq<kPer>(q, pieces, s, gmask) : 0.0f;
  const uint32_t step = nsub * U;
  for (uint32_t b0 = 0; b0 < count; b0 += step) {
    const uint4* rows[U];
    uint32_t idx[U], rid[U];
    float acc[U];
    float2 mt[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      idx[u] = b0 + sg + u * nsub;
      rid[u] = ids[idx[u] < count ? idx[u] : count - 1];
      rows[u] = reinterpret_cast<const uint4*>(base + (size_t)rid[u] * row_bytes);
      mt[u] = __ldg(meta + rid[u]);
      acc[u] = 0.0f;
    }
    for (uint32_t p = s; p < pieces; p += 8u) {
      uint4 w[U];
#pragma unroll
      for (int u = 0; u < U; ++u) w[u] = __ldg(rows[u] + p);
#pragma unroll
      for (int u = 0; u < U; ++u) acc[u] = piece_dot<MODE>(w[u], q + p * kPer, acc[u]);
    }
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
      for (int u = 0; u < U; ++u) acc[u] += __shfl_xor_sync(gmask, acc[u], o, 8);
    }
    if (s == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (idx[u] < count) d[idx[u]] = lp_distance<METRIC>(acc[u], mt[u], qq);
    }
  }
}

// Row geometry of the low-precision copies for a compile-time dimension: 16-byte pieces per
// row, pieces each lane of an 8-lane subgroup loads per row (kNP), and rows per subgroup per
// round (kU) chosen so a lane has about eight 16-byte loads in flight.
template <int MODE, int DIM>
struct LpShape {
  static constexpr uint32_t kPer = MODE == kModeBF16 ? 8u : 16u;
  static constexpr uint32_t kStride = (uint32_t)(DIM + 15) / 16u * 16u;
  static constexpr uint32_t kPieces = kStride / kPer;
  static constexpr uint32_t kNP = (kPieces + 7u) / 8u;
  static constexpr int kU = kNP >= 8u ? 1 : (int)(8u / kNP);
};

// score_lp for a compile-time dimension, in wide rounds: every 16-byte piece of a round's rows
// (kU rows per subgroup) and their (scale, norm) are requested before the first conversion, so
// a hop's ~40 FP8 rows cost two memory latencies instead of five.  Per-lane sums and the
// butterfly run in the same order as score_lp, so both give identical distances.
template <int METRIC, int MODE, int DIM>
__device__ __forceinline__ void score_lp_wide(const SearchParams& P, const float* q,
                                              const uint32_t* ids, float* d, uint32_t count,
                                              uint32_t sg, uint32_t nsub, uint32_t s,
                                              unsigned gmask) {
  using Sh = LpShape<MODE, DIM>;
  constexpr uint32_t kPer = Sh::kPer;
  constexpr int U = Sh::kU;
  constexpr int NP = (int)Sh::kNP;
  constexpr uint32_t row_bytes = Sh::kStride * (MODE == kModeBF16 ? 2u : 1u);
  const unsigned char* base = lp_rows<MODE>(P);
  const float2* meta = lp_meta<MODE>(P);
  const float qq = (METRIC == DK_METRIC_L2 || METRIC == DK_METRIC_COSINE)
                       ? subgroup_qq<kPer>(q, Sh::kPieces, s, gmask) : 0.0f;
  const uint32_t step = nsub * U;
  if constexpr (U == 1) {
    // Wide rows (one per subgroup per round): the rows of the later rounds are requested into
    // L2 first, as the FP32 scorer does for its wide rows.
    if (count > step) {
      const uint32_t lines = (row_bytes + 127u) / 128u;
      const uint32_t total = (count - step) * lines;
      for (uint32_t e = sg * 8u + s; e < total; e += nsub * 8u) {
        const unsigned char* r = base + (size_t)ids[step + e / lines] * row_bytes + (e % lines) * 128u;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(r));
      }
    }
  }
  for (uint32_t b0 = 0; b0 < count; b0 += step) {
    uint32_t idx[U], rid[U];
    uint4 w[U][NP];
    float2 mt[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      idx[u] = b0 + sg + u * nsub;
      rid[u] = ids[idx[u] < count ? idx[u] : count - 1];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint4* row = reinterpret_cast<const uint4*>(base + (size_t)rid[u] * row_bytes);
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        const uint32_t p = s + 8u * j;
        w[u][j] = p < Sh::kPieces ? __ldg(row + p) : make_uint4(0u, 0u, 0u, 0u);
      }
      mt[u] = __ldg(meta + rid[u]);
    }
    // Two to four rows per subgroup per round: once the first round's loads are out, the later
    // rounds' rows and (scale, norm) pairs are requested into L2, so those rounds find them on
    // chip.  Measured: BF16 1M x 128 +7-11 %, FP8 2M x 384 +8-12 %; with eight rows per round
    // (FP8 at 128 dimensions, where a hop's second round holds a few rows) it cost 1-7 %.
    if constexpr (U > 1 && U <= 4) {
      if (b0 == 0u && count > step) {
        constexpr uint32_t lines = (row_bytes + 127u) / 128u;
        const uint32_t total = (count - step) * (lines + 1u);
        for (uint32_t e = sg * 8u + s; e < total; e += nsub * 8u) {
          const uint32_t r = ids[step + e / (lines + 1u)], l = e % (lines + 1u);
          const void* a = l < lines ? static_cast<const void*>(base + (size_t)r * row_bytes + l * 128u)
                                    : static_cast<const void*>(meta + r);
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
        }
      }
    }
    float acc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) acc[u] = 0.0f;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const uint32_t p = s + 8u * j;
      if (p >= Sh::kPieces) continue;
#pragma unroll
      for (int u = 0; u < U; ++u) acc[u] = piece_dot<MODE>(w[u][j], q + p * kPer, acc[u]);
    }
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
#pragma unroll
      for (int u = 0; u < U; ++u) acc[u] += __shfl_xor_sync(gmask, acc[u], o, 8);
    }
    if (s == 0) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (idx[u] < count) d[idx[u]] = lp_distance<METRIC>(acc[u], mt[u], qq);
    }
  }
}

// One thread's restatement of the reference kernel for a short slice (PQ chunk distances):
// same accumulator assignment and reduction, lanes walked serially.
__device__ __forceinline__ float thread_chunk_distance(const float* __restrict__ x,
                                                       const float* __restrict__ y, uint32_t len,
                                                       bool ip) {
  const uint32_t trip = len / 32u;
  const uint32_t epi = (len - 32u * trip) / 8u;
  const uint32_t rem = len & 7u;
  const uint32_t base = len - rem;
  float t[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    float s[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t b = 0; b < trip; ++b) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const uint32_t e = 32u * b + 8u * j + l;
        if (ip) s[j] = __fmaf_rn(x[e], __ldg(y + e), s[j]);
        else { const float c = x[e] - __ldg(y + e); s[j] = __fmaf_rn(c, c, s[j]); }
      }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if ((uint32_t)j < epi) {
        const uint32_t e = 32u * trip + 8u * j + l;
        if (ip) s[j] = __fmaf_rn(x[e], __ldg(y + e), s[j]);
        else { const float c = x[e] - __ldg(y + e); s[j] = __fmaf_rn(c, c, s[j]); }
      }
    }
    float v = (s[0] + s[1]) + (s[2] + s[3]);
    if ((uint32_t)l < rem) {
      const uint32_t e = base + l;
      if (ip) v = __fmaf_rn(x[e], __ldg(y + e), v);
      else { const float c = x[e] - __ldg(y + e); v = __fmaf_rn(c, c, v); }
    }
    t[l] = v;
  }
  const float r = tree4(t[0] + t[4], t[1] + t[5], t[2] + t[6], t[3] + t[7]);
  return ip ? -r : r;
}

// pq_dist_lookup_single (fixed_chunk_pq_table.rs:79-95): sequential f32 sum, m ascending.
// The code row's 16-byte words are all loaded before the first lookup.
__device__ __forceinline__ float pq_distance(const uint8_t* __restrict__ code,
                                             const float* __restrict__ table, uint32_t m_count) {
  const uint4* c4 = reinterpret_cast<const uint4*>(code);
  float acc = 0.0f;
  if (m_count <= 64) {
    uint4 w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
      w[i] = (16u * i < m_count) ? __ldg(c4 + i) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (uint32_t m = 0; m < 64; ++m) {
      if (m < m_count) {
        const uint4 ww = w[m >> 4];
        const uint32_t word = ((m >> 2) & 3u) == 0 ? ww.x : ((m >> 2) & 3u) == 1 ? ww.y
                              : ((m >> 2) & 3u) == 2 ? ww.z : ww.w;
        acc += table[m * 256u + ((word >> (8u * (m & 3u))) & 0xFFu)];
      }
    }
    return acc;
  }
  for (uint32_t m0 = 0; m0 < m_count; m0 += 16u) {
    const uint4 ww = __ldg(c4 + (m0 >> 4));
    const uint32_t words[4] = {ww.x, ww.y, ww.z, ww.w};
#pragma unroll
    for (uint32_t j = 0; j < 16u; ++j)
      if (m0 + j < m_count)
        acc += table[(m0 + j) * 256u + ((words[j >> 2] >> (8u * (j & 3u))) & 0xFFu)];
  }
  return acc;
}

// Per-query ADC table (fixed_chunk_pq_table.rs:149-215): L2 table for L2 and
// CosineNormalized, -dot table for InnerProduct (pq/distance/dynamic.rs:64-84).  Pivots are
// read chunk-major (chunk m, centre c, len_m floats), so consecutive threads read
// consecutive 16-byte pieces.
// PQ with the Cosine metric (`DirectCosine`, pq/distance/cosine.rs:27-70 →
// fixed_chunk_pq_table.rs:32-56, 233-243): per chunk m, one CosineStateless pass (the
// Strategy2x4 order of `subgroup_cosine`) over (query chunk, pivot[code[m]] chunk) from zero,
// folded lane by lane into a running accumulator; the cosine of the total, distance 1 - sim.
// One 8-lane subgroup per candidate; lane s is SIMD lane s.
__device__ __forceinline__ float subgroup_pq_cosine(const SearchParams& P, const float* q,
                                                    const uint8_t* __restrict__ code, uint32_t s,
                                                    unsigned gmask) {
  float tx = 0.f, ty = 0.f, tp = 0.f;
  for (uint32_t m = 0; m < P.pq_chunks; ++m) {
    const uint32_t start = __ldg(P.offsets + m), stop = __ldg(P.offsets + m + 1);
    const uint32_t len = stop - start, nvec = len >> 3;
    const float* pv = P.pivots + (size_t)__ldg(code + m) * P.dim + start;
    const float* qq = q + start;
    float x0 = 0.f, y0 = 0.f, p0 = 0.f, x1 = 0.f, y1 = 0.f, p1 = 0.f;
    uint32_t k = 0;
    for (; k + 1u < nvec; k += 2u) {
      const float b0 = __ldg(pv + 8u * k + s), b1 = __ldg(pv + 8u * k + 8u + s);
      const float a0 = qq[8u * k + s], a1 = qq[8u * k + 8u + s];
      x0 = __fmaf_rn(a0, a0, x0);
      y0 = __fmaf_rn(b0, b0, y0);
      p0 = __fmaf_rn(a0, b0, p0);
      x1 = __fmaf_rn(a1, a1, x1);
      y1 = __fmaf_rn(b1, b1, y1);
      p1 = __fmaf_rn(a1, b1, p1);
    }
    if (k < nvec) {
      const float b0 = __ldg(pv + 8u * k + s), a0 = qq[8u * k + s];
      x0 = __fmaf_rn(a0, a0, x0);
      y0 = __fmaf_rn(b0, b0, y0);
      p0 = __fmaf_rn(a0, b0, p0);
    }
    float cx = x0 + x1, cy = y0 + y1, cp = p0 + p1;
    if (s < (len & 7u)) {
      const float b = __ldg(pv + 8u * nvec + s), a = qq[8u * nvec + s];
      cx = __fmaf_rn(a, a, cx);
      cy = __fmaf_rn(b, b, cy);
      cp = __fmaf_rn(a, b, cp);
    }
    tx = tx + cx;
    ty = ty + cy;
    tp = tp + cp;
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    tx += __shfl_xor_sync(gmask, tx, o, 8);
    ty += __shfl_xor_sync(gmask, ty, o, 8);
    tp += __shfl_xor_sync(gmask, tp, o, 8);
  }
  const float denom = __fmul_rn(__fsqrt_rn(tx), __fsqrt_rn(ty));
  float sim;
  if (tx < 1.17549435e-38f || ty < 1.17549435e-38f) sim = 0.0f;
  else sim = fmaxf(-1.0f, fminf(1.0f, __fdiv_rn(tp, denom)));
  return 1.0f - sim;
}

// PQ scoring of ids[0..count): table lookups, or DirectCosine by 8-lane subgroups.
template <int METRIC>
__device__ __forceinline__ void score_pq(const SearchParams& P, const float* q, const float* table,
                                         const uint32_t* ids, float* d, uint32_t count,
                                         uint32_t tid, uint32_t nt) {
  if constexpr (METRIC == DK_METRIC_COSINE) {
    const uint32_t s = tid & 7u;
    const unsigned gmask = 0xFFu << (8u * ((tid & 31u) >> 3));
    for (uint32_t i = tid >> 3; i < count; i += nt >> 3) {
      const float r = subgroup_pq_cosine(P, q, P.codes + (size_t)ids[i] * P.cstride, s, gmask);
      if (s == 0) d[i] = r;
    }
  } else {
    for (uint32_t i = tid; i < count; i += nt)
      d[i] = pq_distance(P.codes + (size_t)ids[i] * P.cstride, table, P.pq_chunks);
  }
}

template <int METRIC>
__device__ __forceinline__ void build_table(const SearchParams& P, const float* q, float* table,
                                            uint32_t tid, uint32_t nt) {
  const bool ip = METRIC == DK_METRIC_INNER_PRODUCT;
  const uint32_t total = P.pq_chunks * 256u;
#pragma unroll 4
  for (uint32_t idx = tid; idx < total; idx += nt) {
    const uint32_t m = idx >> 8, c = idx & 255u;
    const uint32_t start = __ldg(P.offsets + m), stop = __ldg(P.offsets + m + 1);
    const uint32_t len = stop - start;
    table[idx] = thread_chunk_distance(q + start, P.pivots_cm + (size_t)start * 256u + c * len,
                                       len, ip);
  }
}

// ----------------------------------------------------------------------------------------
// Shared-memory state of one query (both kernels).
// ----------------------------------------------------------------------------------------

struct Misc {
  uint32_t size, cursor, cur, nbeam, nvalid, inserted, overflow, result_count;
  uint32_t scount, gcount, pad0, pad1;  // warp kernel: two-level visited-set counters
  uint32_t beam[64];
  uint32_t warp_sums[32];
};

struct State {
  float* q;
  float* table;
  float* qd[2];
  uint32_t* qi[2];
  uint32_t* cand_id;
  float* cand_d;
  float* new_d;
  uint32_t* new_id;
  uint32_t* hash;
  Misc* misc;
};

__device__ __forceinline__ State carve(unsigned char* base, const SearchParams& P) {
  State S;
  S.q = reinterpret_cast<float*>(base + P.off_query);
  S.table = reinterpret_cast<float*>(base + P.off_table);
  S.qd[0] = reinterpret_cast<float*>(base + P.off_qd0);
  S.qd[1] = reinterpret_cast<float*>(base + P.off_qd1);
  S.qi[0] = reinterpret_cast<uint32_t*>(base + P.off_qi0);
  S.qi[1] = reinterpret_cast<uint32_t*>(base + P.off_qi1);
  S.cand_id = reinterpret_cast<uint32_t*>(base + P.off_cand_id);
  S.cand_d = reinterpret_cast<float*>(base + P.off_cand_d);
  S.new_d = reinterpret_cast<float*>(base + P.off_new_d);
  S.new_id = reinterpret_cast<uint32_t*>(base + P.off_new_id);
  S.hash = reinterpret_cast<uint32_t*>(base + P.off_hash);
  S.misc = reinterpret_cast<Misc*>(base + P.off_misc);
  return S;
}

__device__ __forceinline__ void record_hint(const SearchParams& P, uint32_t cmps, uint32_t cap) {
  if (P.hint) {  // device memory: L2 atomics
    const uint32_t r = (uint32_t)(((uint64_t)cmps << 8) / cap);
    atomicMax(P.hint, r);
    atomicAdd(P.hint + 1, r);
    atomicAdd(P.hint + 2, 1u);
  }
}

// Rerank order (inmem/full_precision.rs:357-404 sorts by the exact distance): ascending
// distance, equal distances in queue order.  The reference's comparator calls a NaN equal to
// everything, which leaves its place unspecified; here NaN distances sort after every number,
// in queue order.  True when entry (a, ai) precedes entry (b, bi).
__device__ __forceinline__ bool rerank_before(float a, uint32_t ai, float b, uint32_t bi) {
  const bool an = a != a, bn = b != b;
  if (an != bn) return bn;
  if (an) return ai < bi;
  return a < b || (a == b && ai < bi);
}

// The first k entries of a rerank list (ids `rid`, exact distances `rd`, `count` entries) in
// rerank order, by one warp.  Ranking every entry against the whole list costs O(count * k)
// dependent shared-memory reads per lane when the low-precision queue order differs from the
// exact order (FP8 on 2M x 384 at L = 512: ~4 % of a search).  Instead: T = the k-th smallest
// key of a 32-entry sample (at first the first 32 entries), so at least k keys are <= T and the
// k smallest all are; the keys <= T are gathered one per lane, and each one's rank among them
// is its rank in the whole list (every smaller key is <= T too).  More than 32 keys <= T: the
// first 32 of them become the sample and T shrinks; after 8 rounds, or when T is NaN, or for
// short lists, every entry is ranked against the list.  Returns min(count, k).
__device__ __forceinline__ uint32_t warp_rerank_select(const uint32_t* rid, const float* rd,
                                                       uint32_t count, uint32_t k,
                                                       uint32_t* out_ids, float* out_d,
                                                       uint32_t lane) {
  if (count >= 64u && k >= 1u && k <= 32u) {
    float sd = rd[lane];  // sample: one key per lane
    uint32_t si = lane;
    for (int round = 0; round < 8; ++round) {
      uint32_t r = 0;
      for (uint32_t m = 0; m < 32u; ++m)
        r += rerank_before(__shfl_sync(kFull, sd, m), __shfl_sync(kFull, si, m), sd, si);
      const uint32_t src = __ffs(__ballot_sync(kFull, r == k - 1u)) - 1u;
      const float td = __shfl_sync(kFull, sd, src);
      const uint32_t ti = __shfl_sync(kFull, si, src);
      if (td != td) break;
      uint32_t nc = 0;  // keys <= T gathered so far; lane t holds the t-th
      float cd = 0.0f;
      uint32_t ci = 0;
      for (uint32_t t0 = 0; t0 < count && nc <= 32u; t0 += 32u) {
        const uint32_t i = t0 + lane;
        const float d = i < count ? rd[i] : 0.0f;
        const uint32_t m = __ballot_sync(kFull, i < count && !rerank_before(td, ti, d, i));
        if (m == 0u) continue;
        // Lane nc + q takes the q-th set lane of m (as many as fit in 32).
        uint32_t from = lane;
        const bool take = lane >= nc && lane - nc < (uint32_t)__popc(m);
        if (take) {
          uint32_t mm = m;
          for (uint32_t q = lane - nc; q > 0u; --q) mm &= mm - 1u;
          from = __ffs(mm) - 1u;
        }
        const float gd = __shfl_sync(kFull, d, from);
        const uint32_t gi = __shfl_sync(kFull, i, from);
        if (take) {
          cd = gd;
          ci = gi;
        }
        nc += __popc(m);
      }
      if (nc > 32u) {  // too many keys <= T: the first 32 of them are the next sample
        sd = cd;
        si = ci;
        continue;
      }
      uint32_t rank = 0;
      for (uint32_t m = 0; m < nc; ++m)
        rank += rerank_before(__shfl_sync(kFull, cd, m), __shfl_sync(kFull, ci, m), cd, ci);
      if (lane < nc && rank < k) {
        out_ids[rank] = rid[ci];
        out_d[rank] = cd;
      }
      return k;
    }
  }
  for (uint32_t i = lane; i < count; i += 32u) {
    const float d = rd[i];
    uint32_t r = 0;
    for (uint32_t j = 0; j < count && r < k; ++j) r += rerank_before(rd[j], j, d, i);
    if (r < k) { out_ids[r] = rid[i]; out_d[r] = d; }
  }
  return min(count, k);
}

// ========================================================================================
// CTA-per-query kernel.
// ========================================================================================

template <int NT, int METRIC, int MODE, int DIM>
__device__ __forceinline__ void cta_score(const SearchParams& P, const State& S, const uint32_t* ids,
                                          float* d, uint32_t count) {
  const uint32_t tid = threadIdx.x;
  if (MODE == kModePQ) {
    score_pq<METRIC>(P, S.q, S.table, ids, d, count, tid, NT);
  } else {
    const unsigned gmask = 0xFFu << (8u * ((tid & 31u) >> 3));
    if constexpr (MODE == kModeFP32) {
      score_fp<METRIC, DIM, 1>(P, S.q, ids, d, count, tid >> 3, NT / 8, tid & 7u, gmask);
    } else if constexpr (MODE == kModeF16) {
      score_fp<METRIC, DIM, 1, __half>(P, S.q, ids, d, count, tid >> 3, NT / 8, tid & 7u, gmask);
    } else if constexpr (MODE == kModeU8 || MODE == kModeI8) {
      score_int<METRIC, MODE == kModeI8>(P, S.q, ids, d, count, tid >> 3, NT / 8, tid & 7u, gmask);
    } else if constexpr (DIM > 0) {
      score_lp_wide<METRIC, MODE, DIM>(P, S.q, ids, d, count, tid >> 3, NT / 8, tid & 7u, gmask);
    } else {
      score_lp<METRIC, MODE, 1>(P, S.q, ids, d, count, tid >> 3, NT / 8, tid & 7u, gmask);
    }
  }
}

template <int NT>
__device__ __forceinline__ void cta_merge(const SearchParams& P, const State& S, uint32_t count) {
  const uint32_t tid = threadIdx.x;
  Misc* M = S.misc;
  uint32_t my_valid = 0;
  // Items that cannot enter are dropped: NaN, and above the last entry of a full queue.
  const float tail = M->size == P.cap ? S.qd[M->cur][M->size - 1u] : INFINITY;
  for (uint32_t i = tid; i < count; i += NT) {
    const float d = S.cand_d[i];
    if (d != d || d > tail) continue;
    uint32_t r = 0;
    for (uint32_t j = 0; j < count; ++j) {
      const float dj = S.cand_d[j];
      r += (dj < d) || (dj == d && j > i);
    }
    S.new_d[r] = d;
    S.new_id[r] = S.cand_id[i];
    ++my_valid;
  }
  if (my_valid) atomicAdd(&M->nvalid, my_valid);
  __syncthreads();
  const uint32_t nvalid = M->nvalid;
  const uint32_t size = M->size, cur = M->cur, nxt = cur ^ 1u;
  const uint32_t cap = P.cap;
  const uint32_t new_size = min(size + nvalid, cap);
  const float* od = S.qd[cur];
  const uint32_t* oi = S.qi[cur];
  float* wd = S.qd[nxt];
  uint32_t* wi = S.qi[nxt];
  // Entries before the first insertion point keep their positions; the rest are ranked.
  const uint32_t p0 = nvalid ? count_less(od, size, S.new_d[0]) : size;
  for (uint32_t o = tid; o < p0; o += NT) {
    wd[o] = od[o];
    wi[o] = oi[o];
  }
  for (uint32_t o = p0 + tid; o < size; o += NT) {
    const float d = od[o];
    const uint32_t pos = o + count_less_equal(S.new_d, nvalid, d);
    if (pos < cap) { wd[pos] = d; wi[pos] = oi[o]; }
  }
  for (uint32_t r = tid; r < nvalid; r += NT) {
    const float d = S.new_d[r];
    const uint32_t pos = r + p0 + count_less(od + p0, size - p0, d);
    if (pos < cap) { wd[pos] = d; wi[pos] = S.new_id[r]; }
  }
  __syncthreads();
  if (tid == 0) {
    const uint32_t c = M->cursor;
    uint32_t nc = new_size;
    if (c < size) nc = min(nc, c + count_less_equal(S.new_d, nvalid, od[c]));
    if (nvalid > 0) nc = min(nc, count_less(od, size, S.new_d[0]));
    M->cursor = nc;
    M->size = new_size;
    M->cur = nxt;
    M->nvalid = 0;
  }
  __syncthreads();
}

template <int NT, int METRIC, int DIM>
__device__ void cta_post_process(const SearchParams& P, const State& S, uint32_t qid) {
  const uint32_t tid = threadIdx.x;
  Misc* M = S.misc;
  const uint32_t size = M->size;
  const float* qd = S.qd[M->cur];
  const uint32_t* qi = S.qi[M->cur];
  // The rerank list (up to L + F entries) lives in the queue's other buffer, free after the
  // last merge.
  uint32_t* rid = S.qi[M->cur ^ 1u];
  float* rd = S.qd[M->cur ^ 1u];
  uint32_t* out_ids = P.out_ids + (size_t)qid * P.k;
  float* out_d = P.out_dists + (size_t)qid * P.k;
  uint32_t written;
  uint32_t base = 0;
  for (uint32_t t0 = 0; t0 < size; t0 += NT) {
    const uint32_t i = t0 + tid;
    const uint32_t id = i < size ? (qi[i] & kIdMask) : 0u;
    const bool keep = i < size && (id < P.n || P.keep_start);  // FilterStartPoints (glue.rs:730-773)
    uint32_t total;
    const uint32_t pos = base + block_scan<NT>(keep, M->warp_sums, total);
    if (keep) {
      if (strategy_reranks(P.strategy)) rid[pos] = id;
      else if (pos < P.k) { out_ids[pos] = id; out_d[pos] = qd[i]; }
    }
    base += total;
  }
  if (!strategy_reranks(P.strategy)) {
    written = min(base, P.k);
  } else {
    // Rerank (inmem/full_precision.rs:357-404): exact distances, stable sort, first k.
    const uint32_t count = base;
    __syncthreads();
    cta_score<NT, METRIC, kModeFP32, DIM>(P, S, rid, rd, count);
    __syncthreads();
    for (uint32_t i = tid; i < count; i += NT) {
      const float d = rd[i];
      uint32_t r = 0;
      for (uint32_t j = 0; j < count && r < P.k; ++j) r += rerank_before(rd[j], j, d, i);
      if (r < P.k) { out_ids[r] = rid[i]; out_d[r] = d; }
    }
    written = min(count, P.k);
  }
  for (uint32_t j = written + tid; j < P.k; j += NT) {
    out_ids[j] = DK_INVALID_ID;
    out_d[j] = INFINITY;
  }
  if (tid == 0) M->result_count = written;
}

// The whole search of one query by one CTA.  Returns false if the visited set overflowed.
template <int NT, int METRIC, int MODE, int DIM, class VSet>
__device__ bool cta_search(const SearchParams& P, const State& S, const VSet& vset, uint32_t qid,
                           uint32_t& cmps_out, uint32_t& hops_out) {
  const uint32_t tid = threadIdx.x;
  Misc* M = S.misc;
  const float* qsrc = P.queries + (size_t)qid * P.qstride;
  const uint32_t dpad = (P.dim + 15u) & ~15u;  // zero padded: FP8 pieces hold 16 elements
  for (uint32_t i = tid; i < dpad; i += NT) S.q[i] = i < P.dim ? qsrc[i] : 0.0f;
  vset.clear(tid, NT);
  if (tid == 0) {
    M->size = M->cursor = M->cur = M->inserted = M->overflow = M->nvalid = 0;
  }
  __syncthreads();
  if (MODE == kModePQ && METRIC != DK_METRIC_COSINE) {
    build_table<METRIC>(P, S.q, S.table, tid, NT);
    __syncthreads();
  }
  if (P.f + P.beam * P.max_degree > P.hash_limit) return false;
  // Start points (index.rs:1956-1963): visited, scored and inserted in order.
  for (uint32_t s = tid; s < P.f; s += NT) {
    S.cand_id[s] = P.n + s;
    vset.insert(P.n + s);
  }
  if (tid == 0) M->inserted = P.f;
  __syncthreads();
  cta_score<NT, METRIC, MODE, DIM>(P, S, S.cand_id, S.cand_d, P.f);
  __syncthreads();
  cta_merge<NT>(P, S, P.f);
  uint32_t cmps = P.f, hops = 0;
  while (true) {
    if (tid == 0) {  // closest_notvisited x beam (queue.rs:297-313)
      uint32_t nb = 0, c = M->cursor;
      const uint32_t size = M->size;
      uint32_t* qi = S.qi[M->cur];
      while (nb < P.beam && c < size) {
        if (P.rec_ids && hops + nb < P.rec_cap) {
          P.rec_ids[(size_t)qid * P.rec_cap + hops + nb] = qi[c] & kIdMask;
          P.rec_d[(size_t)qid * P.rec_cap + hops + nb] = S.qd[M->cur][c];
        }
        M->beam[nb++] = qi[c] & kIdMask;
        qi[c] |= kVisited;
        ++c;
        while (c < size && (qi[c] & kVisited)) ++c;
      }
      M->cursor = c;
      M->nbeam = nb;
      if (nb && M->inserted + nb * P.max_degree > P.hash_limit) M->overflow = 1;
    }
    __syncthreads();
    const uint32_t nb = M->nbeam;
    if (nb == 0) break;
    if (M->overflow) return false;
    uint32_t count = 0;
    for (uint32_t b = 0; b < nb; ++b) {
      const uint32_t* row = P.adj + (size_t)M->beam[b] * P.astride;
      const uint32_t deg = __ldg(row);
      for (uint32_t t0 = 0; t0 < deg; t0 += NT) {
        const uint32_t t = t0 + tid;
        bool fresh = false;
        uint32_t id = 0;
        if (t < deg) {
          id = __ldg(row + 1 + t);
          fresh = vset.insert(id);
          // diskann-inmem (provider.rs:451-473): a slot whose tag is not readable stays in the
          // visited set but is not scored.  Only set with the exact bitmap visited set, so
          // `inserted` (hash load) needs no count of these.
          if (fresh && P.readable) fresh = (__ldg(P.readable + (id >> 5)) >> (id & 31u)) & 1u;
        }
        uint32_t total;
        const uint32_t pos = block_scan<NT>(fresh, M->warp_sums, total);
        if (fresh) S.cand_id[count + pos] = id;
        count += total;
      }
    }
    if (tid == 0) M->inserted += count;
    __syncthreads();
    cta_score<NT, METRIC, MODE, DIM>(P, S, S.cand_id, S.cand_d, count);
    __syncthreads();
    cta_merge<NT>(P, S, count);
    cmps += count;
    hops += nb;
  }
  cmps_out = cmps;
  hops_out = hops;
  return true;
}

template <int NT, int METRIC, int MODE, int DIM>
__global__ void __launch_bounds__(NT) k_search_cta(const SearchParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const State S = carve(smem, P);
  SmemHashSet vset{S.hash, (1u << P.hash_log2) - 1u, 32u - P.hash_log2};
  const uint32_t qid = blockIdx.x;
  if (qid >= P.nq) return;
  uint32_t cmps = 0, hops = 0;
  if (!cta_search<NT, METRIC, MODE, DIM>(P, S, vset, qid, cmps, hops)) {
    if (threadIdx.x == 0) {
      P.stats[qid] = dk_search_stats{0u, 0u, 0u, kFlagSpilled};
      if (P.spill_count) atomicAdd(P.spill_count, 1u);
    }
    return;
  }
  cta_post_process<NT, METRIC, DIM>(P, S, qid);
  __syncthreads();
  if (threadIdx.x == 0) {
    P.stats[qid] = dk_search_stats{cmps, hops, S.misc->result_count, 0u};
    record_hint(P, cmps, P.cap);
  }
}

// Spill pass: each CTA owns one bitmap slice and re-runs the queries the first pass flagged.
template <int NT, int METRIC, int MODE, int DIM>
__global__ void __launch_bounds__(NT) k_search_spill(const SearchParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const State S = carve(smem, P);
  BitmapSet vset{P.bitmap + (size_t)blockIdx.x * P.bitmap_words, P.bitmap_words};
  if (P.spill_count && *(volatile const uint32_t*)P.spill_count == 0u) return;  // nothing spilled
  for (uint32_t qid = blockIdx.x; qid < P.nq; qid += gridDim.x) {
    if (!(P.stats[qid].flags & kFlagSpilled)) continue;
    __syncthreads();
    uint32_t cmps = 0, hops = 0;
    cta_search<NT, METRIC, MODE, DIM>(P, S, vset, qid, cmps, hops);
    cta_post_process<NT, METRIC, DIM>(P, S, qid);
    __syncthreads();
    if (threadIdx.x == 0) {
      P.stats[qid] = dk_search_stats{cmps, hops, S.misc->result_count, kFlagSpilled};
      record_hint(P, cmps, P.cap);
    }
    __syncthreads();
  }
}

// ========================================================================================
// Warp-per-query kernel.
// ========================================================================================

// Order key of a scored candidate at position i: distance ascending (an order-preserving
// integer image of the float), then position descending (the later insert goes first);
// NaN and padding sort after every valid key.
__device__ __forceinline__ uint64_t new_item_key(const float* d, uint32_t i, uint32_t count,
                                                 float tail) {
  if (i >= count) return ~0ull;
  const float x = d[i];
  if (x != x || x > tail) return ~0ull - 1u;
  uint32_t u = __float_as_uint(x);
  u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  return ((uint64_t)u << 32) | (uint32_t)~i;
}

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, uint32_t m) {
  const uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  const uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}

// Sort the hop's scored candidates into new_{d,id}[0..nvalid) by (distance ascending,
// position descending) — the order the reference's one-by-one inserts produce among
// themselves.  Items that cannot enter the queue are dropped first: NaN distances, and,
// when the queue is full, distances above its last entry `tail` (every queue entry precedes
// them, so the merged top L+F is unchanged).  At most 32 kept: each lane counts the smaller
// keys in shared memory (measured 3.5 % faster for FP8 traversal than a bitonic network of
// shuffles, whose 15 stages form one dependent chain); 33 to 64: a bitonic network over two
// keys per lane; beyond 64 a counting rank.  Returns nvalid.
__device__ __forceinline__ uint32_t warp_order_new(const State& S, uint32_t count, uint32_t lane,
                                                   float tail) {
  uint32_t nvalid = 0;
  if (count <= 64u) {
    uint64_t k0 = new_item_key(S.cand_d, lane, count, tail);
    uint64_t k1 = new_item_key(S.cand_d, lane + 32u, count, tail);
    const bool v0 = k0 < ~0ull - 1u, v1 = k1 < ~0ull - 1u;
    const uint32_t m0 = __ballot_sync(kFull, v0), m1 = __ballot_sync(kFull, v1);
    nvalid = __popc(m0) + __popc(m1);
    if (nvalid == 0u) {
      // nothing to place
    } else if (nvalid <= 32u) {
      // Compact the kept keys to one per lane (through new_d / new_id as scratch), sort 32.
      uint32_t* hi = reinterpret_cast<uint32_t*>(S.new_d);
      if (v0) {
        const uint32_t r = __popc(m0 & lanemask_lt());
        hi[r] = (uint32_t)(k0 >> 32);
        S.new_id[r] = (uint32_t)k0;
      }
      if (v1) {
        const uint32_t r = __popc(m0) + __popc(m1 & lanemask_lt());
        hi[r] = (uint32_t)(k1 >> 32);
        S.new_id[r] = (uint32_t)k1;
      }
      __syncwarp();
      // Each lane's rank among the kept keys (all distinct: the low word holds the candidate's
      // index), counted from shared memory: no dependent chain of shuffle stages.
      const uint64_t k = lane < nvalid ? (((uint64_t)hi[lane] << 32) | S.new_id[lane]) : ~0ull;
      uint32_t r = 0;
      for (uint32_t j = 0; j < nvalid; ++j) {
        const uint64_t kj = ((uint64_t)hi[j] << 32) | S.new_id[j];
        r += kj < k;
      }
      __syncwarp();
      if (lane < nvalid) {
        const uint32_t i = ~(uint32_t)k;
        S.new_d[r] = S.cand_d[i];
        S.new_id[r] = S.cand_id[i];
      }
    } else {
      for (uint32_t size = 2; size <= 64u; size <<= 1) {
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
          if (stride == 32u) {  // index lane vs index lane+32, both in this lane; ascending
            const uint64_t a = min(k0, k1), b = max(k0, k1);
            k0 = a;
            k1 = b;
          } else {
            const bool lower = (lane & stride) == 0u;
            const bool asc0 = size == 64u || (lane & size) == 0u;
            const bool asc1 = size == 64u || ((lane + 32u) & size) == 0u;
            const uint64_t o0 = shfl_xor64(k0, stride), o1 = shfl_xor64(k1, stride);
            k0 = (lower == asc0) ? min(k0, o0) : max(k0, o0);
            k1 = (lower == asc1) ? min(k1, o1) : max(k1, o1);
          }
        }
      }
      if (lane < nvalid) {
        const uint32_t i = ~(uint32_t)k0;
        S.new_d[lane] = S.cand_d[i];
        S.new_id[lane] = S.cand_id[i];
      }
      if (lane + 32u < nvalid) {
        const uint32_t i = ~(uint32_t)k1;
        S.new_d[lane + 32u] = S.cand_d[i];
        S.new_id[lane + 32u] = S.cand_id[i];
      }
    }
  } else {
    for (uint32_t i0 = 0; i0 < count; i0 += 32u) {
      const uint32_t i = i0 + lane;
      const float d = i < count ? S.cand_d[i] : 0.0f;
      const bool valid = i < count && d == d && !(d > tail);
      if (valid) {
        uint32_t r = 0;
        for (uint32_t j = 0; j < count; ++j) {
          const float dj = S.cand_d[j];
          r += (dj < d) || (dj == d && j > i);
        }
        S.new_d[r] = d;
        S.new_id[r] = S.cand_id[i];
      }
      nvalid += __popc(__ballot_sync(kFull, valid));
    }
  }
  __syncwarp();
  return nvalid;
}

// Last entry of a full queue (items above it cannot enter), else +infinity.
__device__ __forceinline__ float queue_tail(uint32_t cap, const State& S, uint32_t size,
                                            uint32_t cur) {
  return size == cap ? S.qd[cur][size - 1u] : INFINITY;
}

// Position of the first unvisited entry after merging the ordered new items (the next node
// to expand) and that node's id, or kEmpty when the queue will hold no unvisited entry.
__device__ __forceinline__ uint32_t warp_next_cursor(uint32_t cap, const State& S,
                                                     uint32_t nvalid, uint32_t size,
                                                     uint32_t cursor, uint32_t cur,
                                                     uint32_t& next_id) {
  const uint32_t new_size = min(size + nvalid, cap);
  const float* od = S.qd[cur];
  uint32_t nc = new_size;
  next_id = kEmpty;
  if (cursor < size) {
    const uint32_t p = cursor + count_less_equal(S.new_d, nvalid, od[cursor]);
    if (p < nc) { nc = p; next_id = S.qi[cur][cursor] & kIdMask; }
  }
  if (nvalid > 0) {
    const uint32_t p = count_less(od, size, S.new_d[0]);
    if (p < nc) { nc = p; next_id = S.new_id[0]; }
  }
  return nc;
}

// Merge the ordered new items into the queue in place (see the file comment for the order
// rule).  Entries before the first insertion point p0 stay where they are; each later entry
// moves right by the number of new items at or below its distance (a new item goes before
// old items of equal distance), handled 32 at a time from the back, so every entry is read
// before anything is written over it (the destinations keep their order); entries pushed past
// the capacity drop.  The new items' final positions are taken first, from the queue as it
// was.  Before this in-place form every hop rewrote the whole queue into a second buffer; at
// L = 512 that copy was the largest part of a hop.
__device__ __forceinline__ void warp_commit_merge(uint32_t cap, const State& S,
                                                  uint32_t nvalid, uint32_t nc, uint32_t lane,
                                                  uint32_t& size, uint32_t& cursor,
                                                  uint32_t& cur) {
  const uint32_t new_size = min(size + nvalid, cap);
  float* qd = S.qd[cur];
  uint32_t* qi = S.qi[cur];
  if (nvalid > 0u) {
    const uint32_t p0 = count_less(qd, size, S.new_d[0]);
    // The hop's candidate list is consumed: it holds the new items' final positions.
    for (uint32_t r = lane; r < nvalid; r += 32u)
      S.cand_id[r] = r + p0 + count_less(qd + p0, size - p0, S.new_d[r]);
    __syncwarp();
    for (int32_t c0 = (int32_t)size - 32; c0 + 32 > (int32_t)p0; c0 -= 32) {
      const int32_t o = c0 + (int32_t)lane;
      const bool live = o >= (int32_t)p0 && o < (int32_t)size;
      float d = 0.0f;
      uint32_t id = 0u, pos = cap;
      if (live) {
        d = qd[o];
        id = qi[o];
        pos = (uint32_t)o + count_less_equal(S.new_d, nvalid, d);
      }
      __syncwarp();
      if (live && pos < cap) {
        qd[pos] = d;
        qi[pos] = id;
      }
      __syncwarp();
    }
    for (uint32_t r = lane; r < nvalid; r += 32u) {
      const uint32_t pos = S.cand_id[r];
      if (pos < cap) {
        qd[pos] = S.new_d[r];
        qi[pos] = S.new_id[r];
      }
    }
  }
  cursor = nc;
  size = new_size;
  (void)cur;  // the queue stays in buffer `cur`; the other buffer is the rerank's scratch
  __syncwarp();
}

__device__ __forceinline__ void warp_merge(uint32_t cap, const State& S, uint32_t count,
                                           uint32_t lane, uint32_t& size, uint32_t& cursor,
                                           uint32_t& cur) {
  const uint32_t nvalid = warp_order_new(S, count, lane, queue_tail(cap, S, size, cur));
  uint32_t next_id;
  const uint32_t nc = warp_next_cursor(cap, S, nvalid, size, cursor, cur, next_id);
  warp_commit_merge(cap, S, nvalid, nc, lane, size, cursor, cur);
}

// One query's inputs and outputs (a batch row, or a serving request).
struct QueryIO {
  const float* query;
  uint32_t k;
  uint32_t cap;  // L + F
  uint32_t* ids;
  float* dists;
  dk_search_stats* stats;
  uint32_t* rec_ids;  // graph construction: expanded nodes (P.rec_cap), or null
  float* rec_d;
};

template <int METRIC, int MODE, int DIM, int U>
__device__ __forceinline__ void warp_score(const SearchParams& P, const State& S,
                                           const uint32_t* ids, float* d, uint32_t count,
                                           uint32_t lane) {
  if (MODE == kModePQ) {
    score_pq<METRIC>(P, S.q, S.table, ids, d, count, lane, 32u);
  } else {
    const unsigned gmask = 0xFFu << (8u * (lane >> 3));
    if constexpr (MODE == kModeFP32) {
      score_fp<METRIC, DIM, U>(P, S.q, ids, d, count, lane >> 3, 4u, lane & 7u, gmask);
    } else if constexpr (DIM > 0) {
      score_lp_wide<METRIC, MODE, DIM>(P, S.q, ids, d, count, lane >> 3, 4u, lane & 7u, gmask);
    } else {
      score_lp<METRIC, MODE, 2>(P, S.q, ids, d, count, lane >> 3, 4u, lane & 7u, gmask);
    }
  }
  __syncwarp();
}

template <int METRIC, int DIM, int U>
__device__ void warp_post_process(const SearchParams& P, const State& S, const QueryIO& io,
                                  uint32_t lane, uint32_t size, uint32_t cur,
                                  uint32_t& result_count) {
  const float* qd = S.qd[cur];
  const uint32_t* qi = S.qi[cur];
  // The rerank list (up to L + F ids and distances) lives in the shared visited level when the
  // queue has one buffer (the planner sizes the level for it; every query clears the level
  // before its search), else in the queue's other buffer, free after the last merge.
  uint32_t* rid = P.single_queue ? S.hash : S.qi[cur ^ 1u];
  float* rd = P.single_queue ? reinterpret_cast<float*>(S.hash + P.cap) : S.qd[cur ^ 1u];
  uint32_t* out_ids = io.ids;
  float* out_d = io.dists;
  const uint32_t k = io.k;
  const bool hybrid = strategy_reranks(P.strategy);
  uint32_t base = 0;
  for (uint32_t t0 = 0; t0 < size; t0 += 32u) {
    if (!hybrid && base >= k) break;
    const uint32_t i = t0 + lane;
    const uint32_t id = i < size ? (qi[i] & kIdMask) : 0u;
    const bool keep = i < size && (id < P.n || P.keep_start);  // FilterStartPoints (glue.rs:730-773)
    const uint32_t m = __ballot_sync(kFull, keep);
    const uint32_t pos = base + __popc(m & lanemask_lt());
    if (keep) {
      if (hybrid) rid[pos] = id;
      else if (pos < k) { out_ids[pos] = id; out_d[pos] = qd[i]; }
    }
    base += __popc(m);
  }
  uint32_t written;
  if (!hybrid) {
    written = min(base, k);
  } else {
    // Rerank (inmem/full_precision.rs:357-404): exact distances, stable sort, first k.
    const uint32_t count = base;
    __syncwarp();
    warp_score<METRIC, kModeFP32, DIM, U>(P, S, rid, rd, count, lane);
    written = warp_rerank_select(rid, rd, count, k, out_ids, out_d, lane);
  }
  for (uint32_t j = written + lane; j < k; j += 32u) {
    out_ids[j] = DK_INVALID_ID;
    out_d[j] = INFINITY;
  }
  result_count = written;
}

// One query, run by one warp.  Writes the query's outputs and stats (or the spill flag).
template <int METRIC, int MODE, int DIM, int U>
__device__ __forceinline__ void warp_query(const SearchParams& P, const State& S,
                                           WarpVisited& vset, const QueryIO& io, uint32_t lane) {
  const float* qsrc = io.query;
  const uint32_t cap = io.cap;
  const uint32_t dpad = (P.dim + 15u) & ~15u;  // zero padded: FP8 pieces hold 16 elements
  for (uint32_t i = lane; i < dpad; i += 32u) S.q[i] = i < P.dim ? qsrc[i] : 0.0f;
  vset.reset(lane);
  __syncwarp();
  if (MODE == kModePQ && METRIC != DK_METRIC_COSINE) {
    build_table<METRIC>(P, S.q, S.table, lane, 32u);
    __syncwarp();
  }
  if (P.f + P.beam * P.max_degree > P.gtable_limit) {
    if (lane == 0) {
      *io.stats = dk_search_stats{0u, 0u, 0u, kFlagSpilled};
      if (P.spill_count) atomicAdd(P.spill_count, 1u);
    }
    return;
  }
  uint32_t size = 0, cursor = 0, cur = 0;
  for (uint32_t s0 = 0; s0 < P.f; s0 += 32u) {
    const uint32_t s = s0 + lane;
    if (s < P.f) S.cand_id[s] = P.n + s;
    vset.insert(s < P.f, P.n + s);
  }
  __syncwarp();
  warp_score<METRIC, MODE, DIM, U>(P, S, S.cand_id, S.cand_d, P.f, lane);
  warp_merge(cap, S, P.f, lane, size, cursor, cur);
  uint32_t cmps = P.f, hops = 0;
  uint32_t* beam = S.misc->beam;
  // Adjacency row of the next node, fetched while the previous hop's merge runs (beam 1:
  // the next node is known as soon as the hop's candidates are scored).
  uint32_t pf_node = kEmpty, pf_deg = 0, pf_ids[4] = {0u, 0u, 0u, 0u};

  while (cursor < size) {
    // closest_notvisited x beam (queue.rs:297-313); `cursor` is the first unvisited entry.
    uint32_t nb = 0, c = cursor;
    uint32_t* qi = S.qi[cur];
    while (c < size) {
      const uint32_t idx = c + lane;
      const bool unv = idx < size && !(qi[idx] & kVisited);
      uint32_t m = __ballot_sync(kFull, unv);
      if (nb < P.beam) {
        const uint32_t take = min((uint32_t)__popc(m), P.beam - nb);
        const uint32_t rank = __popc(m & lanemask_lt());
        if (unv && rank < take) {
          beam[nb + rank] = qi[idx] & kIdMask;
          qi[idx] |= kVisited;
          if (io.rec_ids && hops + nb + rank < P.rec_cap) {
            io.rec_ids[hops + nb + rank] = qi[idx] & kIdMask;
            io.rec_d[hops + nb + rank] = S.qd[cur][idx];
          }
        }
        nb += take;
        for (uint32_t t = 0; t < take; ++t) m &= m - 1u;
      }
      if (m) {
        c += __ffs(m) - 1u;
        break;
      }
      c += 32u;
    }
    cursor = min(c, size);
    __syncwarp();
    // The global level must keep room for a whole hop going there; otherwise spill.
    if (vset.gcount + nb * P.max_degree > P.gtable_limit) {
      if (lane == 0) {
      *io.stats = dk_search_stats{0u, 0u, 0u, kFlagSpilled};
      if (P.spill_count) atomicAdd(P.spill_count, 1u);
    }
      return;
    }
    // Expand: adjacency rows in beam order, ids through the visited set in order.
    uint32_t count = 0;
    for (uint32_t b = 0; b < nb; ++b) {
      const uint32_t node = beam[b];
      const uint32_t* row = P.adj + (size_t)node * P.astride;
      uint32_t deg;
      uint32_t ids[4];
      if (b == 0 && node == pf_node) {
        deg = pf_deg;
#pragma unroll
        for (int r = 0; r < 4; ++r) ids[r] = pf_ids[r];
      } else {
        deg = __ldg(row);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const uint32_t t = 32u * r + lane;
          ids[r] = t < P.max_degree ? __ldg(row + 1 + t) : 0u;
        }
      }
      // A row's global-level probes go out together (one round trip per row): always for the
      // low-precision traversal, and for the other modes unless P.row_probes is cleared.
      if ((MODE == kModeBF16 || MODE == kModeFP8 || P.row_probes) && deg <= 128u) {
        bool fresh[4];
        vset.insert_row(ids, deg, lane, fresh);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          if (32u * r >= deg) break;
          const uint32_t m = __ballot_sync(kFull, fresh[r]);
          if (fresh[r]) S.cand_id[count + __popc(m & lanemask_lt())] = ids[r];
          count += __popc(m);
        }
      } else {
        for (uint32_t t0 = 0; t0 < deg; t0 += 32u) {
          const uint32_t t = t0 + lane;
          uint32_t id;
          if (t0 < 128u) {
            const uint32_t r = t0 >> 5;
            id = r == 0 ? ids[0] : r == 1 ? ids[1] : r == 2 ? ids[2] : ids[3];
          } else {
            id = t < deg ? __ldg(row + 1 + t) : 0u;
          }
          const bool fresh = vset.insert(t < deg, id);
          const uint32_t m = __ballot_sync(kFull, fresh);
          if (fresh) S.cand_id[count + __popc(m & lanemask_lt())] = id;
          count += __popc(m);
        }
      }
    }
    __syncwarp();
    warp_score<METRIC, MODE, DIM, U>(P, S, S.cand_id, S.cand_d, count, lane);
    const uint32_t nvalid = warp_order_new(S, count, lane, queue_tail(cap, S, size, cur));
    uint32_t next_id;
    const uint32_t nc = warp_next_cursor(cap, S, nvalid, size, cursor, cur, next_id);
    pf_node = P.beam == 1 ? next_id : kEmpty;
    if (pf_node != kEmpty) {
      const uint32_t* row = P.adj + (size_t)pf_node * P.astride;
      pf_deg = __ldg(row);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint32_t t = 32u * r + lane;
        pf_ids[r] = t < P.max_degree ? __ldg(row + 1 + t) : 0u;
      }
    }
    warp_commit_merge(cap, S, nvalid, nc, lane, size, cursor, cur);
    cmps += count;
    hops += nb;
  }
  uint32_t result_count = 0;
  warp_post_process<METRIC, DIM, U>(P, S, io, lane, size, cur, result_count);
  if (lane == 0) {
    *io.stats = dk_search_stats{cmps, hops, result_count, 0u};
    record_hint(P, cmps, cap);
  }
}

// Persistent grid: every warp owns a shared-memory slice and a global overflow table and
// takes queries from a work counter until the batch is done.
template <int METRIC, int MODE, int DIM, int U>
// Register budget.  The compiler's own choice for `__launch_bounds__(128)` alone is 96
// registers with heavy spills (~1.6x slower).  FP32 / BF16 / FP8: a minimum of four resident
// blocks caps them at 128 registers (FP32 at D = 128 with four rows per subgroup spills 12
// bytes; no other variant spills), measured 2 % (FP32) and 5-9 % (BF16 / FP8) faster on a
// 1M-point graph than with the ~160-170 registers of a one-block minimum.  PQ keeps the
// one-block minimum (up to 255 registers).  (A six-block minimum for rows wider than 128
// elements, 85 registers, let 24 warps stay resident on long searches but measured 5-8 % slower
// on 2M x 384 and 11 % slower for BF16 on 20M x 384, for 1 % on FP32 there.)
__global__ void __launch_bounds__(128, (MODE == kModePQ) ? 1 : 4)
    k_search_warp(const SearchParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t slot = blockIdx.x * (blockDim.x >> 5) + warp;
  const State S = carve(smem + (size_t)warp * P.warp_smem, P);
  WarpVisited vset;
  vset.s = S.hash;
  vset.ssize = P.hash_slots;
  vset.slimit = P.hash_limit;
  vset.g = P.gtable + ((size_t)slot << P.gtable_log2);
  vset.gmask = (1u << P.gtable_log2) - 1u;
  vset.gshift = 32u - P.gtable_log2;
  bool gdirty = true;  // the overflow table starts as uninitialised memory
  while (true) {
    uint32_t qid = 0;
    if (lane == 0) qid = atomicAdd(P.work_counter, 1u);
    qid = __shfl_sync(kFull, qid, 0);
    if (qid >= P.nq) break;
    if (gdirty) {
      for (uint32_t i = lane; i <= vset.gmask; i += 32u) vset.g[i] = kEmpty;
      __syncwarp();
    }
    const uint32_t qk = P.req_kl ? P.req_kl[2 * qid] : P.k;
    const uint32_t qcap = P.req_kl ? P.req_kl[2 * qid + 1] + P.f : P.cap;
    const QueryIO io{P.queries + (size_t)qid * P.qstride, qk, qcap,
                     P.out_ids + (size_t)qid * P.k, P.out_dists + (size_t)qid * P.k,
                     P.stats + qid,
                     P.rec_ids ? P.rec_ids + (size_t)qid * P.rec_cap : nullptr,
                     P.rec_ids ? P.rec_d + (size_t)qid * P.rec_cap : nullptr};
    warp_query<METRIC, MODE, DIM, U>(P, S, vset, io, lane);
    if (P.done_flags) {  // serving: publish this request (results first, then its flag)
      __threadfence_system();
      __syncwarp();
      if (lane == 0) {
        __threadfence_system();
        *reinterpret_cast<volatile uint32_t*>(P.done_flags + qid) = P.done_value;
      }
    }
    __syncwarp();
    gdirty = vset.gcount != 0u;
  }
}

// ========================================================================================
// Launch helpers (host).
// ========================================================================================

enum class KernelKind { kWarp, kCta };

struct LaunchPlan {
  SearchParams p1;     // first pass (warp or CTA layout, with hash)
  SearchParams p2;     // spill pass (CTA layout, bitmap)
  KernelKind kind;
  uint32_t warps_per_cta;
  uint32_t grid;       // warp kernel: persistent grid size
  uint32_t spill_ctas;
  uint32_t score_u;    // warp kernel, D <= 128: FP32 rows per subgroup per round (2 or 4; the
                       // FP32 rerank of the low-precision kernels uses it too)
  bool query_only;     // warp kernel: only report `blocks_per_sm` for `warps_per_cta`
  bool skip_spill;     // serving launches: spilled requests are re-run by the host
  int blocks_per_sm;
};

template <int METRIC, int MODE, int DIM, int U>
cudaError_t launch_warp(LaunchPlan& L, cudaStream_t stream) {
  auto k1 = k_search_warp<METRIC, MODE, DIM, U>;
  const uint32_t bytes = L.p1.warp_smem * L.warps_per_cta;
  cudaError_t e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  if (L.query_only)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&L.blocks_per_sm, k1, 32 * L.warps_per_cta,
                                                         bytes);
  k1<<<L.grid, 32 * L.warps_per_cta, bytes, stream>>>(L.p1);
  return cudaGetLastError();
}

template <int METRIC, int MODE, int DIM>
cudaError_t launch_variant(LaunchPlan& L, cudaStream_t stream) {
  cudaError_t e;
  if (L.kind == KernelKind::kWarp) {
    // Rows scored together per 8-lane subgroup: more rows in flight per round for narrow rows.
    if (DIM > 0 && DIM <= 128 && L.score_u >= 4) e = launch_warp<METRIC, MODE, DIM, 4>(L, stream);
    else if (DIM > 0 && DIM <= 128) e = launch_warp<METRIC, MODE, DIM, 2>(L, stream);
    else e = launch_warp<METRIC, MODE, DIM, 1>(L, stream);
    if (e != cudaSuccess || L.query_only || L.skip_spill) return e;
  } else {
    auto k1 = k_search_cta<kCtaThreads, METRIC, MODE, DIM>;
    e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.p1.smem_bytes);
    if (e != cudaSuccess) return e;
    k1<<<L.p1.nq, kCtaThreads, L.p1.smem_bytes, stream>>>(L.p1);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  auto k2 = k_search_spill<kCtaThreads, METRIC, MODE, DIM>;
  e = cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.p2.smem_bytes);
  if (e != cudaSuccess) return e;
  k2<<<L.spill_ctas, kCtaThreads, L.p2.smem_bytes, stream>>>(L.p2);
  return cudaGetLastError();
}

template <int METRIC, int MODE>
cudaError_t launch_dims(LaunchPlan& L, cudaStream_t stream) {
  switch (L.p1.dim) {
    case 96: return launch_variant<METRIC, MODE, 96>(L, stream);
    case 128: return launch_variant<METRIC, MODE, 128>(L, stream);
    case 384: return launch_variant<METRIC, MODE, 384>(L, stream);
    case 768: return launch_variant<METRIC, MODE, 768>(L, stream);
    default: return launch_variant<METRIC, MODE, 0>(L, stream);
  }
}

}  // namespace dk

// Per-metric entry points (one translation unit each, compiled in parallel).
cudaError_t dk_launch_l2(dk::LaunchPlan& L, int mode, cudaStream_t stream);
cudaError_t dk_launch_ip(dk::LaunchPlan& L, int mode, cudaStream_t stream);
cudaError_t dk_launch_cosine(dk::LaunchPlan& L, int mode, cudaStream_t stream);
cudaError_t dk_launch_cosine_normalized(dk::LaunchPlan& L, int mode, cudaStream_t stream);

namespace dk {
// Host planning shared by the batch path and the serving path (dk_search.cu).
// Lay out one query's shared-memory state in `P`; returns its size in bytes.
uint32_t plan_query_smem(SearchParams& P, bool pq, bool with_hash);
// Fill the index and list fields of `P` for k, L (capacity L + F) and the beam width.
void base_params(const dk_index* ix, int32_t strategy, uint32_t k, uint32_t l, uint32_t beam,
                 SearchParams& P);
// Visited-set size estimates (largest, mean) for the queue capacity in `P`.  `absorb`: first
// take in the values the last launch staged (false: read the index's current estimate only).
void visited_estimates(dk_index* ix, const SearchParams& P, double& est, double& est_mean,
                       bool absorb = true);
// Plan a warp-per-query launch (shared level, global level, warps per CTA, and a grid of at
// most `max_warps` warps, capped at the resident maximum); returns a dk_status.
int32_t plan_warp(dk_index* ix, SearchParams& P, LaunchPlan& L, int mode, double est,
                  double est_mean, uint64_t max_warps, cudaStream_t stream);
cudaError_t dispatch(int32_t metric, LaunchPlan& L, int mode, cudaStream_t stream);

// All scoring modes of one metric.
template <int METRIC>
cudaError_t launch_modes(LaunchPlan& L, int mode, cudaStream_t stream) {
  switch (mode) {
    case kModePQ: return launch_dims<METRIC, kModePQ>(L, stream);
    case kModeBF16: return launch_dims<METRIC, kModeBF16>(L, stream);
    case kModeFP8: return launch_dims<METRIC, kModeFP8>(L, stream);
    default: return launch_dims<METRIC, kModeFP32>(L, stream);
  }
}
}  // namespace dk
