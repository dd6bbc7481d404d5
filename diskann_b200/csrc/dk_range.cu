// Range search (the reference's `Range`, diskann/src/graph/search/range_search.rs) with the
// FullPrecision accessor, in two launches per batch.
//
// Round one is the k-NN search itself (dk_launch_search, the warp-per-query kernel) with
// L = k = starting_l and the start points kept in its output: the queue's first starting_l
// entries, in order, which is what range_search.rs:179-193 reads.  k_range_rest then, one
// 128-thread CTA per query (persistent, each CTA owning an exact bitmap): in_range is those
// entries with distance <= radius, written straight into the caller's output row; when
// |in_range| >= (starting_l as f32 * initial_slack) and |in_range| < max_returned, the second
// round (range_search_internal, range_search.rs:331-389) starts from a visited set holding
// exactly in_range and walks a FIFO frontier - in_range itself, in order - popping beam_width
// nodes, expanding them through the visited set and appending every scored neighbour with
// distance <= radius * range_slack while |in_range| < max_returned.  The post-processor drops
// start points and keeps inner_radius < distance <= radius, in order.  Stats follow the
// reference: cmps of the first round; with a second round, hops = first-round hops +
// (first-round hops + second-round hops) (the scratch counter carries the first round's hops).
//
// in_range lives in the caller's output rows (capacity entries per query) and is compacted in
// place at the end.  With max_returned unlimited the capacity bounds it instead; a query that
// reaches the capacity then reports flags bit 2 (its results may be incomplete).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "dk_kernels.cuh"

namespace {

using namespace dk;

struct RangeParams {
  float radius;
  float inner_radius;  // NaN: none
  float initial_slack;
  float range_slack;
  uint32_t starting_l;
  uint32_t max_returned;  // 0: unlimited (bounded by capacity)
  uint32_t capacity;      // output entries per query
  // Round one's output: starting_l entries per query, and its stats.
  const uint32_t* first_ids;
  const float* first_d;
  const dk_search_stats* first_stats;
};

template <int NT, int METRIC, int DIM>
__global__ void __launch_bounds__(NT) k_range_rest(const SearchParams P, const RangeParams R) {
  extern __shared__ __align__(16) unsigned char smem[];
  const State S = carve(smem, P);
  const uint32_t tid = threadIdx.x;
  Misc* M = S.misc;
  BitmapSet vset{P.bitmap + (size_t)blockIdx.x * P.bitmap_words, P.bitmap_words};
  const uint32_t max_ret = R.max_returned ? R.max_returned : R.capacity;
  const float limit = R.radius * R.range_slack;
  const uint32_t dpad = (P.dim + 15u) & ~15u;
  for (uint32_t qid = blockIdx.x; qid < P.nq; qid += gridDim.x) {
    uint32_t* out_ids = P.out_ids + (size_t)qid * R.capacity;
    float* out_d = P.out_dists + (size_t)qid * R.capacity;
    const uint32_t* fi = R.first_ids + (size_t)qid * R.starting_l;
    const float* fd = R.first_d + (size_t)qid * R.starting_l;
    const dk_search_stats first = R.first_stats[qid];
    __syncthreads();
    // in_range: the first starting_l queue entries within the radius, in queue order.
    const uint32_t n_iter = min(first.result_count, R.starting_l);
    uint32_t n_in = 0;
    for (uint32_t i0 = 0; i0 < n_iter; i0 += NT) {
      const uint32_t i = i0 + tid;
      const bool in = i < n_iter && fd[i] <= R.radius;
      uint32_t total;
      const uint32_t pos = block_scan<NT>(in, M->warp_sums, total);
      if (in && n_in + pos < max_ret) {
        out_ids[n_in + pos] = fi[i];
        out_d[n_in + pos] = fd[i];
      }
      n_in = min(n_in + total, max_ret);
    }
    __syncthreads();
    const bool second = n_in >= (uint32_t)((float)R.starting_l * R.initial_slack) && n_in < max_ret;
    uint32_t range_hops = 0;
    if (second) {
      const float* qsrc = P.queries + (size_t)qid * P.qstride;
      for (uint32_t i = tid; i < dpad; i += NT) S.q[i] = i < P.dim ? qsrc[i] : 0.0f;
      vset.clear(tid, NT);
      __syncthreads();
      for (uint32_t i = tid; i < n_in; i += NT) vset.insert(out_ids[i]);
      __syncthreads();
      uint32_t front = 0;
      while (front < n_in && n_in < max_ret) {
        const uint32_t nb = min(P.beam, n_in - front);
        uint32_t count = 0;
        for (uint32_t b = 0; b < nb; ++b) {
          const uint32_t* row = P.adj + (size_t)out_ids[front + b] * P.astride;
          const uint32_t deg = __ldg(row);
          for (uint32_t t0 = 0; t0 < deg; t0 += NT) {
            const uint32_t t = t0 + tid;
            bool fresh = false;
            uint32_t id = 0;
            if (t < deg) {
              id = __ldg(row + 1 + t);
              fresh = vset.insert(id);
            }
            uint32_t total;
            const uint32_t pos = block_scan<NT>(fresh, M->warp_sums, total);
            if (fresh) S.cand_id[count + pos] = id;
            count += total;
          }
        }
        front += nb;
        __syncthreads();
        cta_score<NT, METRIC, kModeFP32, DIM>(P, S, S.cand_id, S.cand_d, count);
        __syncthreads();
        // Append, in expansion order, the neighbours within radius * range_slack while room.
        for (uint32_t i0 = 0; i0 < count; i0 += NT) {
          const uint32_t i = i0 + tid;
          const bool in = i < count && S.cand_d[i] <= limit;
          uint32_t total;
          const uint32_t pos = block_scan<NT>(in, M->warp_sums, total);
          if (in && n_in + pos < max_ret) {
            out_ids[n_in + pos] = S.cand_id[i];
            out_d[n_in + pos] = S.cand_d[i];
          }
          n_in = min(n_in + total, max_ret);
        }
        range_hops += nb;
        __syncthreads();
      }
    }
    // Post-process: FilterStartPoints, then inner_radius < distance <= radius, in order,
    // compacted in place (every element of a chunk is read before the chunk's writes).
    uint32_t written = 0;
    for (uint32_t i0 = 0; i0 < n_in; i0 += NT) {
      const uint32_t i = i0 + tid;
      uint32_t id = 0;
      float d = 0.0f;
      bool keep = false;
      if (i < n_in) {
        id = out_ids[i];
        d = out_d[i];
        keep = id < P.n && d <= R.radius && !(R.inner_radius == R.inner_radius && d <= R.inner_radius);
      }
      uint32_t total;
      const uint32_t pos = block_scan<NT>(keep, M->warp_sums, total);
      if (keep) {
        out_ids[written + pos] = id;
        out_d[written + pos] = d;
      }
      written += total;
      __syncthreads();
    }
    for (uint32_t j = written + tid; j < R.capacity; j += NT) {
      out_ids[j] = DK_INVALID_ID;
      out_d[j] = INFINITY;
    }
    if (tid == 0) {
      const bool truncated = R.max_returned == 0 && n_in >= R.capacity;
      P.stats[qid] = dk_search_stats{first.cmps, second ? first.hops + first.hops + range_hops : first.hops,
                                     written, (second ? 2u : 0u) | (truncated ? 4u : 0u)};
    }
  }
}

// Launches the kernel, or with `occupancy` set only reports its resident CTAs per SM.
template <int METRIC, int DIM>
cudaError_t launch_range(const SearchParams& P, const RangeParams& R, uint32_t grid,
                         cudaStream_t stream, int* occupancy) {
  auto k = k_range_rest<kCtaThreads, METRIC, DIM>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_bytes);
  if (e != cudaSuccess) return e;
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, k, kCtaThreads, P.smem_bytes);
  k<<<grid, kCtaThreads, P.smem_bytes, stream>>>(P, R);
  return cudaGetLastError();
}

template <int METRIC>
cudaError_t range_dims(const SearchParams& P, const RangeParams& R, uint32_t grid,
                       cudaStream_t stream, int* occupancy) {
  switch (P.dim) {
    case 96: return launch_range<METRIC, 96>(P, R, grid, stream, occupancy);
    case 128: return launch_range<METRIC, 128>(P, R, grid, stream, occupancy);
    case 384: return launch_range<METRIC, 384>(P, R, grid, stream, occupancy);
    case 768: return launch_range<METRIC, 768>(P, R, grid, stream, occupancy);
    default: return launch_range<METRIC, 0>(P, R, grid, stream, occupancy);
  }
}

cudaError_t range_dispatch(int32_t metric, const SearchParams& P, const RangeParams& R,
                           uint32_t grid, cudaStream_t stream, int* occupancy) {
  switch (metric) {
    case DK_METRIC_L2: return range_dims<DK_METRIC_L2>(P, R, grid, stream, occupancy);
    case DK_METRIC_INNER_PRODUCT: return range_dims<DK_METRIC_INNER_PRODUCT>(P, R, grid, stream, occupancy);
    case DK_METRIC_COSINE: return range_dims<DK_METRIC_COSINE>(P, R, grid, stream, occupancy);
    default: return range_dims<DK_METRIC_COSINE_NORMALIZED>(P, R, grid, stream, occupancy);
  }
}

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

// Range::with_options validation (range_search.rs:63-110) plus this API's own bounds.
int32_t check_range(const dk_index* ix, uint32_t starting_l, uint32_t beam_width, float radius,
                    float inner_radius, float initial_slack, float range_slack,
                    uint32_t max_returned, uint32_t capacity, uint64_t qstride) {
  if (!ix) return fail(DK_ERR_INVALID_ARGUMENT, "index is null");
  if (beam_width == 0) return fail(DK_ERR_BEAM_WIDTH_ZERO, "beam width cannot be zero");
  if (starting_l == 0) return fail(DK_ERR_L_ZERO, "l_value cannot be zero");
  if (max_returned && max_returned < starting_l)
    return fail(DK_ERR_INVALID_ARGUMENT, "max_returned must be greater than or equal to starting_l");
  if (!(initial_slack >= 0.0f && initial_slack <= 1.0f))
    return fail(DK_ERR_INVALID_ARGUMENT, "initial_search_slack must be between 0 and 1.0");
  if (!(range_slack >= 1.0f))
    return fail(DK_ERR_INVALID_ARGUMENT, "range_search_slack must be greater than or equal to 1.0");
  if (!std::isnan(inner_radius) && inner_radius > radius)
    return fail(DK_ERR_INVALID_ARGUMENT, "inner_radius must be less than or equal to radius");
  if (capacity < starting_l) return fail(DK_ERR_INVALID_ARGUMENT, "capacity below starting_l");
  if (max_returned && capacity < max_returned)
    return fail(DK_ERR_INVALID_ARGUMENT, "capacity below max_returned");
  if (beam_width > 64) return fail(DK_ERR_UNSUPPORTED, "beam_width above 64 is not supported");
  if ((uint64_t)starting_l + ix->f > 16384) return fail(DK_ERR_UNSUPPORTED, "starting_l above 16383 is not supported");
  if (qstride < ix->dim) return fail(DK_ERR_DIMENSION_MISMATCH, "query stride below dim");
  return DK_OK;
}

int32_t launch_range_search(dk_index* ix, const float* queries, uint64_t qstride, uint32_t nq,
                            const RangeParams& R0, uint32_t beam, uint32_t* ids, float* dists,
                            dk_search_stats* stats, cudaStream_t stream) {
  if (nq == 0) return DK_OK;
  RangeParams R = R0;
  const uint32_t sl = R.starting_l;
  SearchParams P{};
  dk::base_params(ix, DK_STRATEGY_FULL_PRECISION, 1, sl, beam, P);
  P.cap = 0;  // round two keeps no queue; its lists hold beam x max_degree candidates
  P.queries = queries;
  P.qstride = qstride;
  P.nq = nq;
  P.out_ids = ids;
  P.out_dists = dists;
  P.stats = stats;
  P.hash_limit = 0xFFFFFFFFu;  // the bitmap never fills
  P.smem_bytes = dk::plan_query_smem(P, false, false);
  int max_optin = 0, sms = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  if (P.smem_bytes > (uint32_t)max_optin)
    return fail(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory");
  // Round two: one exact bitmap over all ids per resident CTA (occupancy), within 512 MiB.
  const uint32_t words = (ix->n + ix->f + 31u) / 32u;
  const uint64_t per = (uint64_t)words * 4u;
  int occ = 0;
  const cudaError_t eo = range_dispatch(ix->metric, P, R, 0, nullptr, &occ);
  if (eo != cudaSuccess) return fail(DK_ERR_CUDA, std::string("range occupancy: ") + cudaGetErrorString(eo));
  uint32_t grid = std::min<uint32_t>(nq, (uint32_t)std::max(1, occ) * (uint32_t)std::max(1, sms));
  if (per * grid > (512ull << 20)) grid = (uint32_t)std::max<uint64_t>(1, (512ull << 20) / per);
  // Scratch: round one's ids | distances | stats | round two's bitmaps.
  auto up = [](uint64_t x) { return (x + 255) / 256 * 256; };
  const uint64_t o_d = up((uint64_t)nq * sl * 4), o_st = o_d + up((uint64_t)nq * sl * 4);
  const uint64_t o_bm = o_st + up((uint64_t)nq * sizeof(dk_search_stats));
  unsigned char* scratch = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&scratch), o_bm + per * grid,
                                          ix->pool, stream);
  if (e != cudaSuccess)
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("range scratch: ") + cudaGetErrorString(e));
  uint32_t* first_ids = reinterpret_cast<uint32_t*>(scratch);
  float* first_d = reinterpret_cast<float*>(scratch + o_d);
  dk_search_stats* first_st = reinterpret_cast<dk_search_stats*>(scratch + o_st);
  // Round one: the k-NN search with L = k = starting_l, start points kept in its output.
  const int32_t rc = dk_launch_search(ix, DK_STRATEGY_FULL_PRECISION, queries, qstride, nq, sl,
                                      sl, beam, first_ids, first_d, first_st, stream, nullptr,
                                      true);
  if (rc == DK_OK) {
    R.first_ids = first_ids;
    R.first_d = first_d;
    R.first_stats = first_st;
    P.bitmap = reinterpret_cast<uint32_t*>(scratch + o_bm);
    P.bitmap_words = words;
    e = range_dispatch(ix->metric, P, R, grid, stream, nullptr);
  }
  cudaFreeAsync(scratch, stream);
  if (rc != DK_OK) return rc;
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("range launch: ") + cudaGetErrorString(e));
  return DK_OK;
}

// Packs each query's filled result slots (row pitch `capacity`) into one contiguous run at
// offs[q] (the exclusive prefix sum of the result counts), so that the copy to host memory
// carries the results only, not every query's full capacity.  One warp per query.
__global__ void __launch_bounds__(256) k_pack_results(const uint32_t* ids, const float* d,
                                                      uint32_t capacity, const uint64_t* offs,
                                                      uint32_t nq, uint32_t* pid, float* pd) {
  const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
  for (uint32_t q = blockIdx.x * wpb + (threadIdx.x >> 5); q < nq; q += gridDim.x * wpb) {
    const uint64_t o = offs[q];
    const uint32_t c = (uint32_t)(offs[q + 1] - o);
    for (uint32_t j = lane; j < c; j += 32u) {
      pid[o + j] = ids[(size_t)q * capacity + j];
      pd[o + j] = d[(size_t)q * capacity + j];
    }
  }
}

// Spreads `total` packed values, stored at the tail of the caller's nq x capacity array, into
// the heads of their rows, in place.  Rows are visited in order and each moves to or before
// its packed position (the results of rows q.. number at most (nq - q) * capacity), and a
// row's moved values end where the next row's packed values begin, so nothing unread is
// overwritten.
template <typename T>
void spread_in_place(T* a, uint32_t nq, uint32_t capacity, const std::vector<uint64_t>& offs) {
  const uint64_t total = offs[nq];
  T* packed = a + (uint64_t)nq * capacity - total;
  for (uint32_t q = 0; q < nq; ++q) {
    const uint64_t c = offs[q + 1] - offs[q];
    if (c) memmove(a + (uint64_t)q * capacity, packed + offs[q], c * sizeof(T));
  }
}

}  // namespace

extern "C" int32_t dk_range_search_device(dk_index* ix, const float* queries,
                                          uint64_t query_stride, uint32_t nq, uint32_t starting_l,
                                          uint32_t beam_width, float radius, float inner_radius,
                                          float initial_slack, float range_slack,
                                          uint32_t max_returned, uint32_t capacity, uint32_t* ids,
                                          float* dists, dk_search_stats* stats, void* stream) {
  const int32_t v = check_range(ix, starting_l, beam_width, radius, inner_radius, initial_slack,
                                range_slack, max_returned, capacity, query_stride);
  if (v != DK_OK) return v;
  if (nq && (!queries || !ids || !dists || !stats))
    return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids, dists and stats are required");
  dk::DeviceGuard guard(ix->device);
  const RangeParams R{radius, inner_radius, initial_slack, range_slack, starting_l, max_returned,
                      capacity};
  return launch_range_search(ix, queries, query_stride, nq, R, beam_width, ids, dists, stats,
                             static_cast<cudaStream_t>(stream));
}

extern "C" int32_t dk_range_search(dk_index* ix, const float* queries, uint64_t query_stride,
                                   uint32_t nq, uint32_t starting_l, uint32_t beam_width,
                                   float radius, float inner_radius, float initial_slack,
                                   float range_slack, uint32_t max_returned, uint32_t capacity,
                                   uint32_t* ids, float* dists, dk_search_stats* stats) {
  const int32_t v = check_range(ix, starting_l, beam_width, radius, inner_radius, initial_slack,
                                range_slack, max_returned, capacity, query_stride);
  if (v != DK_OK) return v;
  if (nq == 0) return DK_OK;
  if (!queries || !ids || !dists) return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids and dists are required");
  dk::DeviceGuard guard(ix->device);
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  const size_t qbytes = (size_t)nq * ix->dim * 4, obytes = (size_t)nq * capacity * 4;
  const size_t off_ids = (qbytes + 255) / 256 * 256;
  const size_t off_d = off_ids + (obytes + 255) / 256 * 256;
  const size_t off_st = off_d + (obytes + 255) / 256 * 256;
  const size_t total = off_st + (size_t)nq * sizeof(dk_search_stats);
  unsigned char* buf = nullptr;
  e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&buf), total, ix->pool, s);
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("range buffers: ") + cudaGetErrorString(e));
  }
  if (query_stride == ix->dim)
    e = cudaMemcpyAsync(buf, queries, qbytes, cudaMemcpyHostToDevice, s);
  else
    e = cudaMemcpy2DAsync(buf, ix->dim * 4, queries, query_stride * 4, ix->dim * 4, nq,
                          cudaMemcpyHostToDevice, s);
  int32_t rc = DK_OK;
  if (e == cudaSuccess) {
    const RangeParams R{radius, inner_radius, initial_slack, range_slack, starting_l,
                        max_returned, capacity};
    rc = launch_range_search(ix, reinterpret_cast<const float*>(buf), ix->dim, nq, R, beam_width,
                             reinterpret_cast<uint32_t*>(buf + off_ids),
                             reinterpret_cast<float*>(buf + off_d),
                             reinterpret_cast<dk_search_stats*>(buf + off_st), s);
    // The counts first; then only the filled slots come back (packed on the device), unless
    // the rows are mostly full anyway.
    std::vector<dk_search_stats> st(nq);
    if (rc == DK_OK)
      e = cudaMemcpyAsync(st.data(), buf + off_st, (size_t)nq * sizeof(dk_search_stats),
                          cudaMemcpyDeviceToHost, s);
    if (rc == DK_OK && e == cudaSuccess) e = cudaStreamSynchronize(s);
    std::vector<uint64_t> offs(nq + 1, 0);
    if (rc == DK_OK && e == cudaSuccess) {
      for (uint32_t q = 0; q < nq; ++q) offs[q + 1] = offs[q] + std::min(st[q].result_count, capacity);
      const uint64_t total = offs[nq];
      if (2 * total >= (uint64_t)nq * capacity) {
        e = cudaMemcpyAsync(ids, buf + off_ids, obytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dists, buf + off_d, obytes, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      } else if (total) {
        const size_t p_offs = 0, p_ids = ((size_t)(nq + 1) * 8 + 255) / 256 * 256;
        const size_t p_d = p_ids + (total * 4 + 255) / 256 * 256, p_total = p_d + total * 4;
        unsigned char* pk = nullptr;
        e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&pk), p_total, ix->pool, s);
        if (e == cudaSuccess) {
          e = cudaMemcpyAsync(pk + p_offs, offs.data(), (size_t)(nq + 1) * 8, cudaMemcpyHostToDevice, s);
          if (e == cudaSuccess) {
            const uint32_t blocks = std::min<uint32_t>((nq + 7) / 8, 4096);
            k_pack_results<<<blocks, 256, 0, s>>>(
                reinterpret_cast<const uint32_t*>(buf + off_ids),
                reinterpret_cast<const float*>(buf + off_d), capacity,
                reinterpret_cast<const uint64_t*>(pk + p_offs), nq,
                reinterpret_cast<uint32_t*>(pk + p_ids), reinterpret_cast<float*>(pk + p_d));
            e = cudaGetLastError();
          }
          const uint64_t tail = (uint64_t)nq * capacity - total;
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(ids + tail, pk + p_ids, total * 4, cudaMemcpyDeviceToHost, s);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(dists + tail, pk + p_d, total * 4, cudaMemcpyDeviceToHost, s);
          cudaFreeAsync(pk, s);
          const cudaError_t ep = cudaStreamSynchronize(s);
          if (e == cudaSuccess) e = ep;
          if (e == cudaSuccess) {
            spread_in_place(ids, nq, capacity, offs);
            spread_in_place(dists, nq, capacity, offs);
          }
        }
      }
      if (e == cudaSuccess && stats) memcpy(stats, st.data(), (size_t)nq * sizeof(dk_search_stats));
    }
  }
  cudaFreeAsync(buf, s);
  const cudaError_t es = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (rc != DK_OK) return rc;
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("range copy: ") + cudaGetErrorString(e));
  if (es != cudaSuccess) return fail(DK_ERR_CUDA, std::string("range search: ") + cudaGetErrorString(es));
  return DK_OK;
}
