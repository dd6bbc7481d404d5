// Paged search (the reference's `PagedSearch`, diskann/src/graph/search/paged.rs, created by
// DiskANNIndex::paged_search / paged_search_with_init_ids, diskann/src/graph/index.rs:2080-2160)
// with the FullPrecision accessor, for a batch of sessions that page together.
//
// Each session keeps its whole search state in device memory between calls: the resizable
// queue (every scored id is kept, sorted by distance, with the visited flag in the id's top
// bit; only the first L + F entries are searched and iterated), an exact visited bitmap over
// all N + F ids, the page cache (`computed_result`, at most L entries) and the running
// comparison / hop counters.  One 128-thread CTA owns one session at a time; the grid is
// persistent over the batch.  The queue lives in global memory (it grows past any shared
// memory budget) and is merged in place: a batch of new items ranked in shared memory, the
// old entries from the first insertion point moved right from the back in CTA-wide chunks,
// then the new items written to their final positions.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "dk_kernels.cuh"

namespace {

using namespace dk;

constexpr uint32_t kPagedCapacityReached = 4u;  // dk_search_stats::flags bit 2

struct PagedSession {
  uint32_t size, cursor, cache_n, cache_next, cmps, hops, flags, pad;
};

struct PagedParams {
  PagedSession* sess;
  const float* query;  // nq x dim, compact
  uint32_t* q_ids;     // nq x qcap: the resizable queue
  float* q_d;
  uint32_t* cache_ids;  // nq x l_value: computed_result
  float* cache_d;
  uint32_t* bitmap;  // nq x bitmap_words
  uint32_t bitmap_words;
  uint32_t qcap;
  uint32_t l_value;  // PagedSearch::search_param_l
  uint32_t lq;       // the queue's search_param_l: l_value + F
  uint32_t k;
  const uint32_t* init_ids;  // creation only: nq x n_init, or null for the start points
  uint32_t n_init;
  uint32_t* out_ids;  // nq x k
  float* out_d;
  dk_search_stats* stats;
};

struct PagedShared {
  uint32_t size, cursor, cache_n, cache_next, cmps, hops, flags;
  uint32_t node, nb, nvalid, total;
};

// Inserts cand_id/cand_d[0..count) (adjacency order) into the session's queue with the
// resizable queue's rules (queue.rs:130-171 with auto_resizable): NaN dropped, each item
// before existing equal distances, later items before earlier equal ones, the cursor moved to
// the first insertion point if that is lower.  A queue at `qcap` keeps its best qcap entries
// and flags the session (the reference grows without bound).
template <int NT>
__device__ void paged_insert(const State& S, PagedShared& T, uint32_t* qi, float* qd,
                             uint32_t qcap, uint32_t count) {
  const uint32_t tid = threadIdx.x;
  uint32_t my_valid = 0;
  for (uint32_t i = tid; i < count; i += NT) {
    const float d = S.cand_d[i];
    if (d != d) continue;
    uint32_t r = 0;
    for (uint32_t j = 0; j < count; ++j) {
      const float dj = S.cand_d[j];
      r += (dj < d) || (dj == d && j > i);  // NaN compares false: not counted
    }
    S.new_d[r] = d;
    S.new_id[r] = S.cand_id[i];
    ++my_valid;
  }
  if (tid == 0) T.nvalid = 0;
  __syncthreads();
  if (my_valid) atomicAdd(&T.nvalid, my_valid);
  __syncthreads();
  const uint32_t nv = T.nvalid;
  if (nv == 0) return;
  const uint32_t size = T.size;
  // Final positions of the new items, taken before the old entries move (cand_id is free).
  for (uint32_t r = tid; r < nv; r += NT) S.cand_id[r] = r + count_less(qd, size, S.new_d[r]);
  const uint32_t p0 = count_less(qd, size, S.new_d[0]);
  __syncthreads();
  // Old entries from p0 on move right by the number of new items <= them, back to front.
  for (uint32_t hi = size; hi > p0;) {
    const uint32_t lo = hi - p0 > NT ? hi - NT : p0;
    const uint32_t o = lo + tid;
    uint32_t id = 0, pos = 0xFFFFFFFFu;
    float d = 0.0f;
    if (o < hi) {
      d = qd[o];
      id = qi[o];
      pos = o + count_less_equal(S.new_d, nv, d);
    }
    __syncthreads();
    if (pos < qcap) {
      qd[pos] = d;
      qi[pos] = id;
    }
    __syncthreads();
    hi = lo;
  }
  for (uint32_t r = tid; r < nv; r += NT) {
    const uint32_t pos = S.cand_id[r];
    if (pos < qcap) {
      qd[pos] = S.new_d[r];
      qi[pos] = S.new_id[r];
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (size + nv > qcap) T.flags |= kPagedCapacityReached;
    T.size = min(size + nv, qcap);
    T.cursor = min(T.cursor, p0);
  }
  __syncthreads();
}

// One node's expansion: its adjacency row in stored order, retained by the visited bitmap
// (glue.rs:524-561 NotInMut), scored; returns the number of scored ids.
template <int NT, int METRIC, int DIM>
__device__ uint32_t paged_expand(const SearchParams& P, const State& S, const BitmapSet& vset,
                                 uint32_t node) {
  const uint32_t tid = threadIdx.x;
  const uint32_t* row = P.adj + (size_t)node * P.astride;
  const uint32_t deg = __ldg(row);
  uint32_t count = 0;
  for (uint32_t t0 = 0; t0 < deg; t0 += NT) {
    const uint32_t t = t0 + tid;
    bool fresh = false;
    uint32_t id = 0;
    if (t < deg) {
      id = __ldg(row + 1 + t);
      fresh = vset.insert(id);
    }
    uint32_t total;
    const uint32_t pos = block_scan<NT>(fresh, S.misc->warp_sums, total);
    if (fresh) S.cand_id[count + pos] = id;
    count += total;
  }
  __syncthreads();
  cta_score<NT, METRIC, kModeFP32, DIM>(P, S, S.cand_id, S.cand_d, count);
  __syncthreads();
  return count;
}

// Creation (INIT) or one next_page call for every session of the batch.
template <int NT, int METRIC, int DIM, bool INIT>
__global__ void __launch_bounds__(NT) k_paged(const SearchParams P, const PagedParams G) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ PagedShared T;
  const State S = carve(smem, P);
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  const uint32_t dpad = (P.dim + 15u) & ~15u;
  for (uint32_t s = blockIdx.x; s < P.nq; s += gridDim.x) {
    __syncthreads();
    const BitmapSet vset{G.bitmap + (size_t)s * G.bitmap_words, G.bitmap_words};
    uint32_t* qi = G.q_ids + (size_t)s * G.qcap;
    float* qd = G.q_d + (size_t)s * G.qcap;
    uint32_t* cache_i = G.cache_ids + (size_t)s * G.l_value;
    float* cache_d = G.cache_d + (size_t)s * G.l_value;
    const float* qsrc = G.query + (size_t)s * P.dim;
    for (uint32_t i = tid; i < dpad; i += NT) S.q[i] = i < P.dim ? qsrc[i] : 0.0f;
    if (INIT) {
      vset.clear(tid, NT);
      if (tid == 0) T = PagedShared{};
      __syncthreads();
      // index.rs:2117-2146: the init ids (default: the start points) enter the visited set,
      // then their neighbours are expanded in order and inserted; no counter moves.
      const uint32_t n_init = G.init_ids ? G.n_init : P.f;
      const uint32_t* init = G.init_ids ? G.init_ids + (size_t)s * G.n_init : nullptr;
      for (uint32_t j = tid; j < n_init; j += NT) vset.insert(init ? init[j] : P.n + j);
      __syncthreads();
      for (uint32_t j = 0; j < n_init; ++j) {
        const uint32_t count = paged_expand<NT, METRIC, DIM>(P, S, vset, init ? init[j] : P.n + j);
        paged_insert<NT>(S, T, qi, qd, G.qcap, count);
      }
      if (tid == 0) G.sess[s] = PagedSession{T.size, T.cursor, 0u, 0u, 0u, 0u, T.flags, 0u};
      continue;
    }
    if (tid == 0) {
      const PagedSession ss = G.sess[s];
      T.size = ss.size;
      T.cursor = ss.cursor;
      T.cache_n = ss.cache_n;
      T.cache_next = ss.cache_next;
      T.cmps = ss.cmps;
      T.hops = ss.hops;
      T.flags = ss.flags;
    }
    __syncthreads();
    uint32_t* out_i = G.out_ids + (size_t)s * G.k;
    float* out_d = G.out_d + (size_t)s * G.k;
    // paged.rs:71-87: drain the cached page first.
    const uint32_t from_cache = min(G.k, T.cache_n - T.cache_next);
    for (uint32_t i = tid; i < from_cache; i += NT) {
      out_i[i] = cache_i[T.cache_next + i];
      out_d[i] = cache_d[T.cache_next + i];
    }
    uint32_t n_out = from_cache;
    __syncthreads();
    if (tid == 0) T.cache_next += from_cache;
    if (n_out < G.k) {
      // paged.rs:89-97: resume search_internal (beam 1; the visited set is not empty).
      while (true) {
        if (warp == 0) {  // closest_notvisited (queue.rs:297-313), the scan by ballots
          uint32_t c = T.cursor, node = 0, nb = 0;
          const uint32_t size = T.size, lim = min(G.lq, size);
          if (c < lim) {
            node = qi[c] & kIdMask;
            nb = 1;
            __syncwarp();
            if (lane == 0) qi[c] |= kVisited;
            ++c;
            while (c < size) {
              const uint32_t i = c + lane;
              const bool unv = i < size && !(qi[i] & kVisited);
              const uint32_t b = __ballot_sync(kFull, unv);
              if (b) { c += __ffs(b) - 1; break; }
              c = min(c + 32u, size);
            }
          }
          if (lane == 0) {
            T.cursor = c;
            T.node = node;
            T.nb = nb;
          }
        }
        __syncthreads();
        if (T.nb == 0) break;
        const uint32_t count = paged_expand<NT, METRIC, DIM>(P, S, vset, T.node);
        paged_insert<NT>(S, T, qi, qd, G.qcap, count);
        if (tid == 0) {
          T.cmps += count;
          T.hops += 1;
        }
      }
      __syncthreads();
      // filter_search_candidates (paged.rs:128-151): the first page_size non-start entries of
      // the iterated prefix, and how many entries were looked at.
      const uint32_t lim = min(G.lq, T.size);
      if (tid == 0) T.total = lim;
      uint32_t found = 0;
      for (uint32_t i0 = 0; i0 < lim && found < G.k; i0 += NT) {
        const uint32_t i = i0 + tid;
        const uint32_t id = i < lim ? (qi[i] & kIdMask) : 0u;
        const bool keep = i < lim && id < P.n;
        uint32_t total;
        const uint32_t pos = found + block_scan<NT>(keep, S.misc->warp_sums, total);
        if (keep && pos < G.k) {
          cache_i[pos] = id;
          cache_d[pos] = qd[i];
          if (pos == G.k - 1) T.total = i + 1;
        }
        found += total;
      }
      __syncthreads();
      const uint32_t cache_n = min(found, G.k), drained = T.total;
      // drain_best (queue.rs:174-181): shift left by `drained`, front to back.
      const uint32_t size = T.size, rest = size - drained;
      for (uint32_t lo = 0; lo < rest; lo += NT) {
        const uint32_t o = lo + tid;
        uint32_t id = 0;
        float d = 0.0f;
        if (o < rest) {
          id = qi[o + drained];
          d = qd[o + drained];
        }
        __syncthreads();
        if (o < rest) {
          qi[o] = id;
          qd[o] = d;
        }
        __syncthreads();
      }
      // paged.rs:105-121: the new page goes to the cache; what this call still needs from it.
      const uint32_t leftover = min(G.k - n_out, cache_n);
      for (uint32_t i = tid; i < leftover; i += NT) {
        out_i[n_out + i] = cache_i[i];
        out_d[n_out + i] = cache_d[i];
      }
      n_out += leftover;
      __syncthreads();
      if (tid == 0) {
        T.size = rest;
        T.cursor = 0;
        T.cache_n = cache_n;
        T.cache_next = leftover;
      }
    }
    for (uint32_t j = n_out + tid; j < G.k; j += NT) {
      out_i[j] = DK_INVALID_ID;
      out_d[j] = INFINITY;
    }
    __syncthreads();
    if (tid == 0) {
      G.sess[s] = PagedSession{T.size, T.cursor, T.cache_n, T.cache_next, T.cmps, T.hops, T.flags, 0u};
      if (G.stats) G.stats[s] = dk_search_stats{T.cmps, T.hops, n_out, T.flags};
    }
  }
}

// Launches the kernel, or with `occupancy` set only reports its resident CTAs per SM.
template <int METRIC, int DIM>
cudaError_t launch_paged(const SearchParams& P, const PagedParams& G, bool init, uint32_t grid,
                         cudaStream_t stream, int* occupancy) {
  auto k = init ? k_paged<kCtaThreads, METRIC, DIM, true> : k_paged<kCtaThreads, METRIC, DIM, false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_bytes);
  if (e != cudaSuccess) return e;
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, k, kCtaThreads, P.smem_bytes);
  k<<<grid, kCtaThreads, P.smem_bytes, stream>>>(P, G);
  return cudaGetLastError();
}

template <int METRIC>
cudaError_t paged_dims(const SearchParams& P, const PagedParams& G, bool init, uint32_t grid,
                       cudaStream_t stream, int* occupancy) {
  switch (P.dim) {
    case 96: return launch_paged<METRIC, 96>(P, G, init, grid, stream, occupancy);
    case 128: return launch_paged<METRIC, 128>(P, G, init, grid, stream, occupancy);
    case 384: return launch_paged<METRIC, 384>(P, G, init, grid, stream, occupancy);
    case 768: return launch_paged<METRIC, 768>(P, G, init, grid, stream, occupancy);
    default: return launch_paged<METRIC, 0>(P, G, init, grid, stream, occupancy);
  }
}

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

struct dk_paged {
  dk_index* ix = nullptr;
  uint32_t nq = 0, l_value = 0, qcap = 0;
  cudaStream_t stream = nullptr;
  unsigned char* buf = nullptr;  // sessions, queries, queues, caches, bitmaps, outputs
  SearchParams P{};
  PagedParams G{};
  uint32_t grid = 0;
};

namespace {

cudaError_t paged_launch(dk_paged* ps, bool init, int* occupancy = nullptr) {
  switch (ps->ix->metric) {
    case DK_METRIC_L2:
      return paged_dims<DK_METRIC_L2>(ps->P, ps->G, init, ps->grid, ps->stream, occupancy);
    case DK_METRIC_INNER_PRODUCT:
      return paged_dims<DK_METRIC_INNER_PRODUCT>(ps->P, ps->G, init, ps->grid, ps->stream, occupancy);
    case DK_METRIC_COSINE:
      return paged_dims<DK_METRIC_COSINE>(ps->P, ps->G, init, ps->grid, ps->stream, occupancy);
    default:
      return paged_dims<DK_METRIC_COSINE_NORMALIZED>(ps->P, ps->G, init, ps->grid, ps->stream, occupancy);
  }
}

void paged_release(dk_paged* ps) {
  if (ps->buf) cudaFreeAsync(ps->buf, ps->stream);
  if (ps->stream) {
    cudaStreamSynchronize(ps->stream);
    cudaStreamDestroy(ps->stream);
  }
  delete ps;
}

}  // namespace

extern "C" int32_t dk_paged_search_create(dk_index* ix, const float* queries,
                                          uint64_t query_stride, uint32_t nq, uint32_t l_value,
                                          const uint32_t* init_ids, uint32_t n_init,
                                          uint32_t queue_capacity, dk_paged** out) {
  if (!ix || !out) return fail(DK_ERR_INVALID_ARGUMENT, "index and out are required");
  *out = nullptr;
  if (nq == 0) return fail(DK_ERR_INVALID_ARGUMENT, "a paged search needs at least one query");
  if (!queries) return fail(DK_ERR_INVALID_ARGUMENT, "queries are required");
  if (query_stride < ix->dim) return fail(DK_ERR_DIMENSION_MISMATCH, "query stride below dim");
  if (n_init && !init_ids) return fail(DK_ERR_INVALID_ARGUMENT, "init_ids is null");
  const uint64_t ids_total = (uint64_t)ix->n + ix->f;
  for (uint64_t i = 0; i < (uint64_t)nq * n_init; ++i)
    if (init_ids[i] >= ids_total) return fail(DK_ERR_INVALID_ARGUMENT, "init id out of range");
  const uint32_t qcap = queue_capacity ? queue_capacity : (uint32_t)ids_total;
  if ((uint64_t)l_value + ix->f > 16384u)
    return fail(DK_ERR_UNSUPPORTED, "l_value above 16383 is not supported");
  dk::DeviceGuard guard(ix->device);
  auto* ps = new dk_paged;
  ps->ix = ix;
  ps->nq = nq;
  ps->l_value = l_value;
  ps->qcap = qcap;
  cudaError_t e = cudaStreamCreateWithFlags(&ps->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ps;
    return fail(DK_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  const uint32_t words = (uint32_t)((ids_total + 31u) / 32u);
  const uint32_t lcap = std::max<uint32_t>(l_value, 1u);
  const size_t o_sess = 0;
  const size_t o_query = o_sess + align256((size_t)nq * sizeof(PagedSession));
  const size_t o_qi = o_query + align256((size_t)nq * ix->dim * 4);
  const size_t o_qd = o_qi + align256((size_t)nq * qcap * 4);
  const size_t o_ci = o_qd + align256((size_t)nq * qcap * 4);
  const size_t o_cd = o_ci + align256((size_t)nq * lcap * 4);
  const size_t o_bm = o_cd + align256((size_t)nq * lcap * 4);
  const size_t o_oi = o_bm + align256((size_t)nq * words * 4);
  const size_t o_od = o_oi + align256((size_t)nq * lcap * 4);
  const size_t o_st = o_od + align256((size_t)nq * lcap * 4);
  const size_t o_init = o_st + align256((size_t)nq * sizeof(dk_search_stats));
  const size_t total = o_init + align256((size_t)nq * n_init * 4);
  e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ps->buf), total, ix->pool, ps->stream);
  if (e != cudaSuccess) {
    ps->buf = nullptr;
    paged_release(ps);
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("paged search state: ") + cudaGetErrorString(e));
  }
  unsigned char* b = ps->buf;
  SearchParams& P = ps->P;
  dk::base_params(ix, DK_STRATEGY_FULL_PRECISION, 1, l_value, 1, P);
  P.cap = 0;  // the queue lives in global memory
  P.nq = nq;
  P.smem_bytes = dk::plan_query_smem(P, false, false);
  PagedParams& G = ps->G;
  G.sess = reinterpret_cast<PagedSession*>(b + o_sess);
  G.query = reinterpret_cast<const float*>(b + o_query);
  G.q_ids = reinterpret_cast<uint32_t*>(b + o_qi);
  G.q_d = reinterpret_cast<float*>(b + o_qd);
  G.cache_ids = reinterpret_cast<uint32_t*>(b + o_ci);
  G.cache_d = reinterpret_cast<float*>(b + o_cd);
  G.bitmap = reinterpret_cast<uint32_t*>(b + o_bm);
  G.bitmap_words = words;
  G.qcap = qcap;
  G.l_value = l_value;
  G.lq = l_value + ix->f;
  G.out_ids = reinterpret_cast<uint32_t*>(b + o_oi);
  G.out_d = reinterpret_cast<float*>(b + o_od);
  G.stats = reinterpret_cast<dk_search_stats*>(b + o_st);
  G.init_ids = n_init ? reinterpret_cast<const uint32_t*>(b + o_init) : nullptr;
  G.n_init = n_init;
  // Persistent grid of every resident CTA (each session owns its bitmap, so no cap here).
  int sms = 0, occ = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  e = paged_launch(ps, false, &occ);
  if (e != cudaSuccess) {
    paged_release(ps);
    return fail(DK_ERR_CUDA, std::string("paged occupancy: ") + cudaGetErrorString(e));
  }
  ps->grid = std::min<uint32_t>(nq, (uint32_t)std::max(1, occ) * (uint32_t)std::max(1, sms));
  if (query_stride == ix->dim)
    e = cudaMemcpyAsync(b + o_query, queries, (size_t)nq * ix->dim * 4, cudaMemcpyHostToDevice, ps->stream);
  else
    e = cudaMemcpy2DAsync(b + o_query, ix->dim * 4, queries, query_stride * 4, ix->dim * 4, nq,
                          cudaMemcpyHostToDevice, ps->stream);
  if (e == cudaSuccess && n_init)
    e = cudaMemcpyAsync(b + o_init, init_ids, (size_t)nq * n_init * 4, cudaMemcpyHostToDevice, ps->stream);
  if (e == cudaSuccess) e = paged_launch(ps, true);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ps->stream);
  if (e != cudaSuccess) {
    paged_release(ps);
    return fail(DK_ERR_CUDA, std::string("paged search create: ") + cudaGetErrorString(e));
  }
  G.init_ids = nullptr;
  *out = ps;
  return DK_OK;
}

extern "C" int32_t dk_paged_search_next(dk_paged* ps, uint32_t k, uint32_t* ids, float* dists,
                                        dk_search_stats* stats) {
  if (!ps) return fail(DK_ERR_INVALID_ARGUMENT, "paged search is null");
  if (k > ps->l_value)
    return fail(DK_ERR_INVALID_ARGUMENT, "k should be less than or equal to search_param_l");
  if (k == 0) return fail(DK_ERR_INVALID_ARGUMENT, "k should be greater than 0");
  if (!ids || !dists) return fail(DK_ERR_INVALID_ARGUMENT, "ids and dists are required");
  dk::DeviceGuard guard(ps->ix->device);
  ps->G.k = k;
  cudaError_t e = paged_launch(ps, false);
  const size_t obytes = (size_t)ps->nq * k * 4;
  if (e == cudaSuccess) e = cudaMemcpyAsync(ids, ps->G.out_ids, obytes, cudaMemcpyDeviceToHost, ps->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dists, ps->G.out_d, obytes, cudaMemcpyDeviceToHost, ps->stream);
  if (e == cudaSuccess && stats)
    e = cudaMemcpyAsync(stats, ps->G.stats, (size_t)ps->nq * sizeof(dk_search_stats),
                        cudaMemcpyDeviceToHost, ps->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ps->stream);
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("paged search next: ") + cudaGetErrorString(e));
  return DK_OK;
}

extern "C" int32_t dk_paged_search_destroy(dk_paged* ps) {
  if (!ps) return DK_OK;
  dk::DeviceGuard guard(ps->ix->device);
  paged_release(ps);
  return DK_OK;
}
