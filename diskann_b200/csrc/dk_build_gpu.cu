// Device side of graph construction; see dk_build_gpu.h.

#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dk_build_gpu.h"
#include "dk_kernels.cuh"

struct dk_build_gpu {
  dk_index* ix = nullptr;
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t l_build = 0, max_batch = 0, rec_cap = 0;
  // Device: outputs of one batch search (k = 1) and the records.
  uint32_t* d_ids = nullptr;
  float* d_dists = nullptr;
  dk_search_stats* d_stats = nullptr;
  uint32_t* d_rec_ids = nullptr;
  float* d_rec_d = nullptr;
  // Pinned host copies.
  dk_search_stats* h_stats = nullptr;
  uint32_t* h_hops = nullptr;
  uint32_t* h_rec_ids = nullptr;
  float* h_rec_d = nullptr;
  // Row updates: packed rows and their node ids, grown on demand.
  uint32_t* h_rows = nullptr;
  uint32_t* d_rows = nullptr;
  uint32_t* h_nodes = nullptr;
  uint32_t* d_nodes = nullptr;
  uint32_t rows_cap = 0;
  uint32_t last_start = 0, last_count = 0;  // the batch whose records are on the device
  // Forward prune outputs (max_batch x degree, and counts), device and pinned host.
  uint32_t* d_out = nullptr;
  uint32_t* d_out_cnt = nullptr;
  uint32_t* h_out = nullptr;
  uint32_t* h_out_cnt = nullptr;
  uint32_t out_degree = 0;
  // Back-edge groups (targets, offsets, sources, oversize flags), grown on demand.
  uint32_t* d_groups = nullptr;
  uint32_t* h_groups = nullptr;
  uint64_t groups_cap = 0;  // words
};

namespace {

using namespace dk;

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

int32_t cuda_fail(cudaError_t e, const char* what) {
  return fail(DK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Row r of `rows` (astride words: degree, ids, zero padding) goes to adjacency row nodes[r].
__global__ void k_scatter_rows(uint32_t* __restrict__ adj, uint32_t astride,
                               const uint32_t* __restrict__ rows, const uint32_t* __restrict__ nodes,
                               uint32_t count) {
  const uint64_t total = (uint64_t)count * astride;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / astride;
    const uint32_t c = (uint32_t)(i - r * astride);
    adj[(uint64_t)nodes[r] * astride + c] = rows[i];
  }
}

// ---- occlude_list on the device -------------------------------------------------------

struct PruneArgs {
  uint32_t ntasks;
  // Forward prune: task t is point start + t with its search record.
  uint32_t start;
  const uint32_t* rec_ids;
  const float* rec_d;
  const dk_search_stats* rec_stats;
  uint32_t rec_cap;
  uint32_t* out;      // ntasks x degree
  uint32_t* out_cnt;  // ntasks; UINT32_MAX: record overflowed
  // Back edges: group g appends src[off[g] .. off[g+1]) to row targets[g]; task t is group
  // groups_of[t] (or t when null).
  const uint32_t* groups_of;
  const uint32_t* targets;
  const uint32_t* off;
  const uint32_t* src;
  uint32_t* oversize;  // per group: 1 if its list would not fit `cap`
  uint32_t* adj;
  uint32_t astride, max_degree;
  // occlude_list parameters.
  float alpha;
  uint32_t degree, max_occlusion, occluding;
  // Per-warp shared memory: query row | sort keys | ids | dists | occlusion factors |
  // last-checked | selected | a chunk of 4 ids and distances.
  uint32_t cap;  // pool entries (power of two)
  uint32_t dpad, off_key, off_ids, off_d, off_of, off_lc, off_nb, off_ch, warp_bytes;
};

// Sort key of (distance, id), ascending like sort_pool's comparator: distance first (-0 taken
// as +0, which compares equal to it), then id.
__device__ __forceinline__ uint64_t pool_key(float d, uint32_t id) {
  uint32_t b = __float_as_uint(d == 0.0f ? 0.0f : d);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
  return ((uint64_t)b << 32) | id;
}
__device__ __forceinline__ float key_dist(uint64_t k) {
  uint32_t b = (uint32_t)(k >> 32);
  b = (b & 0x80000000u) ? (b & 0x7FFFFFFFu) : ~b;
  return __uint_as_float(b);
}

// Sort ids/dist[0..m) by (distance, id) and keep the first max_occlusion (sort_pool).
__device__ uint32_t warp_sort_pool(const PruneArgs& A, uint64_t* key, uint32_t* ids, float* dist,
                                   uint32_t m, uint32_t lane) {
  uint32_t S = 32;
  while (S < m) S <<= 1;
  for (uint32_t j = lane; j < S; j += 32) key[j] = j < m ? pool_key(dist[j], ids[j]) : ~0ull;
  __syncwarp();
  for (uint32_t k = 2; k <= S; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = lane; i < S; i += 32) {
        const uint32_t x = i ^ j;
        if (x > i) {
          const uint64_t a = key[i], b = key[x];
          if ((a > b) == ((i & k) == 0)) {
            key[i] = b;
            key[x] = a;
          }
        }
      }
      __syncwarp();
    }
  m = min(m, A.max_occlusion);
  for (uint32_t j = lane; j < m; j += 32) {
    ids[j] = (uint32_t)key[j];
    dist[j] = key_dist(key[j]);
  }
  __syncwarp();
  return m;
}

__device__ __forceinline__ void warp_load_row(const SearchParams& P, uint32_t id, float* q,
                                              uint32_t dpad, uint32_t lane) {
  const float* r = P.vectors + (size_t)id * P.vstride;
  for (uint32_t i = lane; i < dpad; i += 32) q[i] = i < P.dim ? r[i] : 0.0f;
  __syncwarp();
}

// occlude_list (index.rs:2570-2782) over the sorted pool, restating the host version
// (dk_build.cpp Builder::occlude) step for step: the alpha schedule, each candidate's running
// occlusion factor and last-checked position, and the early exit once it exceeds the current
// alpha.  The distances a candidate needs are computed four at a time by the warp's 8-lane
// subgroups (the bit-exact search scoring) and then applied in order, so the state after each
// step is the host's.  Every lane runs the same control flow; lane 0 writes.  Returns the
// number selected; st_nb[0..found) are their pool positions.
template <int METRIC, int DIM>
__device__ uint32_t warp_occlude(const SearchParams& P, const PruneArgs& A, uint32_t m,
                                 const uint32_t* ids, const float* dist, float* st_of,
                                 uint32_t* st_lc, uint32_t* st_nb, float* q, uint32_t* ch_ids,
                                 float* ch_d, uint32_t lane) {
  const uint32_t s = lane & 7u, sg = lane >> 3;
  const unsigned gmask = 0xFFu << (8u * sg);
  for (uint32_t j = lane; j < m; j += 32) {
    st_of[j] = 0.0f;
    st_lc[j] = 0u;
  }
  __syncwarp();
  uint32_t found = 0;
  float cur = 1.0f;
  const float inc = fminf(A.alpha, 1.2f);
  while (found < A.degree) {
    for (uint32_t i = 0; i < m && found < A.degree; ++i) {
      float of = st_of[i];
      uint32_t lc = st_lc[i];
      if (of > cur) continue;
      bool loaded = false, over = false;
      while (lc != found && !over) {
        uint32_t scan = lc, cnt = 0;
        while (scan != found && cnt < 4u) {
          if (st_nb[scan] < i) ++cnt;
          ++scan;
        }
        if (cnt) {
          if (!loaded) {
            warp_load_row(P, ids[i], q, A.dpad, lane);
            loaded = true;
          }
          if (lane == 0) {
            uint32_t c = 0;
            for (uint32_t e = lc; e < scan; ++e)
              if (st_nb[e] < i) ch_ids[c++] = ids[st_nb[e]];
          }
          __syncwarp();
          score_fp<METRIC, DIM, 1>(P, q, ch_ids, ch_d, cnt, sg, 4u, s, gmask);
          __syncwarp();
        }
        uint32_t c = 0;
        for (uint32_t e = lc; e < scan; ++e) {
          const uint32_t rp = st_nb[e];
          lc = e + 1;
          if (rp >= i) continue;
          const float djk = ch_d[c++];
          const float dik = dist[i];
          if (A.occluding) {
            if (djk < cur * dik) of = cur + 0.01f;
          } else {
            const float r = djk == 0.0f ? FLT_MAX : __fdiv_rn(dik, djk);
            of = (of < r) ? r : of;
          }
          if (of > cur) {
            over = true;
            break;
          }
        }
        __syncwarp();
      }
      if (lane == 0) st_lc[i] = lc;
      if (of > cur) {
        if (lane == 0) st_of[i] = of;
        __syncwarp();
        continue;
      }
      if (lane == 0) {
        st_of[i] = FLT_MAX;
        st_nb[found] = i;
      }
      __syncwarp();
      ++found;
    }
    if (cur == A.alpha) break;
    cur = fminf(cur * inc, A.alpha);
  }
  return found;
}

// One warp per task, persistent over the tasks.  BACK = false: forward prune of a searched
// point from its record; BACK = true: a back-edge group.
template <int METRIC, int DIM, bool BACK>
__global__ void __launch_bounds__(128) k_prune(const SearchParams P, const PruneArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned char* base = smem + (size_t)warp * A.warp_bytes;
  float* q = reinterpret_cast<float*>(base);
  uint64_t* key = reinterpret_cast<uint64_t*>(base + A.off_key);
  uint32_t* ids = reinterpret_cast<uint32_t*>(base + A.off_ids);
  float* dist = reinterpret_cast<float*>(base + A.off_d);
  float* st_of = reinterpret_cast<float*>(base + A.off_of);
  uint32_t* st_lc = reinterpret_cast<uint32_t*>(base + A.off_lc);
  uint32_t* st_nb = reinterpret_cast<uint32_t*>(base + A.off_nb);
  uint32_t* ch_ids = reinterpret_cast<uint32_t*>(base + A.off_ch);
  float* ch_d = reinterpret_cast<float*>(base + A.off_ch + 16);
  const uint32_t s = lane & 7u, sg = lane >> 3;
  const unsigned gmask = 0xFFu << (8u * sg);
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + warp; t < A.ntasks; t += nw) {
    uint32_t target, m = 0;
    uint32_t* row = nullptr;
    if (!BACK) {
      target = A.start + t;
      const uint32_t n = A.rec_stats[t].hops;
      if (n > A.rec_cap) {
        if (lane == 0) A.out_cnt[t] = 0xFFFFFFFFu;
        continue;
      }
      // The record without the point itself (insert, index.rs:226-341).
      const uint32_t* ri = A.rec_ids + (size_t)t * A.rec_cap;
      const float* rd = A.rec_d + (size_t)t * A.rec_cap;
      for (uint32_t j0 = 0; j0 < n; j0 += 32) {
        const uint32_t j = j0 + lane;
        const uint32_t id = j < n ? ri[j] : target;
        const bool keep = id != target;
        const unsigned b = __ballot_sync(kFull, keep);
        if (keep) {
          const uint32_t pos = m + __popc(b & ((1u << lane) - 1u));
          ids[pos] = id;
          dist[pos] = rd[j];
        }
        m += __popc(b);
      }
      __syncwarp();
    } else {
      const uint32_t gi = A.groups_of ? A.groups_of[t] : t;
      target = A.targets[gi];
      row = A.adj + (size_t)target * A.astride;
      uint32_t len = row[0];
      for (uint32_t j = lane; j < len; j += 32) ids[j] = row[1 + j];
      __syncwarp();
      bool added = false, too_big = false;
      for (uint32_t e = A.off[gi]; e < A.off[gi + 1]; ++e) {
        const uint32_t sid = A.src[e];
        bool present = false;
        for (uint32_t j0 = 0; j0 < len; j0 += 32) {
          const uint32_t j = j0 + lane;
          present |= __any_sync(kFull, j < len && ids[j] == sid);
        }
        if (present) continue;
        if (len == A.cap) {
          too_big = true;
          break;
        }
        if (lane == 0) ids[len] = sid;
        __syncwarp();
        ++len;
        added = true;
      }
      if (too_big) {
        if (lane == 0) A.oversize[gi] = 1u;
        continue;
      }
      if (!added) continue;
      if (len <= A.max_degree) {
        for (uint32_t j = lane; j < len; j += 32) row[1 + j] = ids[j];
        if (lane == 0) row[0] = len;
        continue;
      }
      // add_edge_and_prune: the list without the target, distances to the target.
      for (uint32_t j0 = 0; j0 < len; j0 += 32) {
        const uint32_t j = j0 + lane;
        const uint32_t id = j < len ? ids[j] : target;
        const bool keep = id != target;
        const unsigned b = __ballot_sync(kFull, keep);
        __syncwarp();
        if (keep) ids[m + __popc(b & ((1u << lane) - 1u))] = id;
        m += __popc(b);
        __syncwarp();
      }
      warp_load_row(P, target, q, A.dpad, lane);
      score_fp<METRIC, DIM, 1>(P, q, ids, dist, m, sg, 4u, s, gmask);
      __syncwarp();
    }
    m = warp_sort_pool(A, key, ids, dist, m, lane);
    const uint32_t found = warp_occlude<METRIC, DIM>(P, A, m, ids, dist, st_of, st_lc, st_nb, q,
                                                     ch_ids, ch_d, lane);
    if (!BACK) {
      for (uint32_t j = lane; j < found; j += 32) A.out[(size_t)t * A.degree + j] = ids[st_nb[j]];
      if (lane == 0) A.out_cnt[t] = found;
    } else {
      for (uint32_t j = lane; j < found; j += 32) row[1 + j] = ids[st_nb[j]];
      if (lane == 0) row[0] = found;
    }
    __syncwarp();
  }
}

template <int METRIC, bool BACK>
cudaError_t launch_prune(const SearchParams& P, const PruneArgs& A, cudaStream_t stream) {
  auto k = P.dim == 128 ? k_prune<METRIC, 128, BACK> : k_prune<METRIC, 0, BACK>;
  const uint32_t warps = std::max<uint32_t>(1u, std::min<uint32_t>(4u, (200u << 10) / A.warp_bytes));
  const uint32_t smem = warps * A.warp_bytes;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int occ = 0, sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, 32 * warps, smem);
  if (e != cudaSuccess) return e;
  const uint32_t need = (A.ntasks + warps - 1) / warps;
  const uint32_t grid = std::max<uint32_t>(1u, std::min<uint32_t>(need, (uint32_t)std::max(1, occ) * sms));
  k<<<grid, 32 * warps, smem, stream>>>(P, A);
  return cudaGetLastError();
}

template <bool BACK>
cudaError_t dispatch_prune(int32_t metric, const SearchParams& P, const PruneArgs& A,
                           cudaStream_t stream) {
  switch (metric) {
    case DK_METRIC_L2: return launch_prune<DK_METRIC_L2, BACK>(P, A, stream);
    case DK_METRIC_INNER_PRODUCT: return launch_prune<DK_METRIC_INNER_PRODUCT, BACK>(P, A, stream);
    case DK_METRIC_COSINE: return launch_prune<DK_METRIC_COSINE, BACK>(P, A, stream);
    default: return launch_prune<DK_METRIC_COSINE_NORMALIZED, BACK>(P, A, stream);
  }
}

// Shared-memory layout of a pool of `cap` entries (a power of two >= 32).
void prune_layout(PruneArgs& A, uint32_t dim, uint32_t cap) {
  auto up = [](uint32_t x) { return (x + 15u) & ~15u; };
  A.cap = cap;
  A.dpad = (dim + 15u) & ~15u;
  uint32_t o = up(A.dpad * 4u);
  A.off_key = o;
  o = up(o + cap * 8u);
  A.off_ids = o;
  o = up(o + cap * 4u);
  A.off_d = o;
  o = up(o + cap * 4u);
  A.off_of = o;
  o = up(o + cap * 4u);
  A.off_lc = o;
  o = up(o + cap * 4u);
  A.off_nb = o;
  o = up(o + cap * 4u);
  A.off_ch = o;
  A.warp_bytes = up(o + 32u);
}

uint32_t pow2_at_least(uint32_t x) {
  uint32_t p = 32;
  while (p < x) p <<= 1;
  return p;
}

}  // namespace

int32_t dk_build_gpu_create(const float* vectors, uint64_t stride, uint32_t num_points,
                            uint32_t num_frozen, uint32_t dim, int32_t metric,
                            uint32_t max_degree, uint32_t l_build, uint32_t max_batch,
                            int32_t device, dk_build_gpu** out) {
  *out = nullptr;
  const uint64_t total = (uint64_t)num_points + num_frozen;
  // An empty graph of the final slot width; rows are written as the build proceeds.
  std::vector<uint32_t> empty_adj((size_t)total * max_degree, 0u), degrees((size_t)total, 0u);
  dk_index_desc d{};
  d.num_points = num_points;
  d.num_frozen = num_frozen;
  d.dim = dim;
  d.metric = metric;
  d.vectors = vectors;
  d.vector_stride = stride;
  d.adjacency = empty_adj.data();
  d.adjacency_stride = max_degree;
  d.degrees = degrees.data();
  d.max_degree = max_degree;
  dk_build_gpu* g = new dk_build_gpu();
  int32_t rc = dk_index_create(&d, device, &g->ix);
  if (rc != DK_OK) {
    delete g;
    return rc;
  }
  dk::DeviceGuard guard(device);
  g->device = device;
  g->l_build = l_build;
  g->max_batch = max_batch;
  g->rec_cap = 4u * l_build + 64u;
  const size_t recs = (size_t)max_batch * g->rec_cap;
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_ids), 4ull * max_batch);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_dists), 4ull * max_batch);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_stats), sizeof(dk_search_stats) * max_batch);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_rec_ids), 4ull * recs);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_rec_d), 4ull * recs);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_stats), sizeof(dk_search_stats) * max_batch, 0);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_hops), 4ull * max_batch, 0);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_rec_ids), 4ull * recs, 0);
  if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_rec_d), 4ull * recs, 0);
  if (e != cudaSuccess) {
    dk_build_gpu_destroy(g);
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("build buffers: ") + cudaGetErrorString(e));
  }
  *out = g;
  return DK_OK;
}

int32_t dk_build_gpu_search(dk_build_gpu* g, uint32_t start, uint32_t count, bool copy_records,
                            const uint32_t** rec_ids, const float** rec_d,
                            const uint32_t** hops, uint32_t* rec_cap) {
  if (count > g->max_batch) return fail(DK_ERR_INVALID_ARGUMENT, "build batch above max_batch");
  dk::DeviceGuard guard(g->device);
  dk_index* ix = g->ix;
  const SearchRecord rec{g->d_rec_ids, g->d_rec_d, g->rec_cap};
  int32_t rc = dk_launch_search(ix, DK_STRATEGY_FULL_PRECISION,
                                ix->vectors + (size_t)start * ix->vstride, ix->vstride, count, 1,
                                g->l_build, 1, g->d_ids, g->d_dists, g->d_stats, g->stream, &rec);
  if (rc != DK_OK) return rc;
  const size_t n = (size_t)count * g->rec_cap;
  cudaError_t e = cudaMemcpyAsync(g->h_stats, g->d_stats, sizeof(dk_search_stats) * count,
                                  cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess && copy_records)
    e = cudaMemcpyAsync(g->h_rec_ids, g->d_rec_ids, 4ull * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess && copy_records)
    e = cudaMemcpyAsync(g->h_rec_d, g->d_rec_d, 4ull * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "build search");
  for (uint32_t i = 0; i < count; ++i) g->h_hops[i] = g->h_stats[i].hops;
  g->last_start = start;
  g->last_count = count;
  *rec_ids = copy_records ? g->h_rec_ids : nullptr;
  *rec_d = copy_records ? g->h_rec_d : nullptr;
  *hops = g->h_hops;
  *rec_cap = g->rec_cap;
  return DK_OK;
}

int32_t dk_build_gpu_set_rows(dk_build_gpu* g, const uint32_t* nodes, uint32_t count,
                              const std::vector<std::vector<uint32_t>>& adj) {
  if (count == 0) return DK_OK;
  dk::DeviceGuard guard(g->device);
  dk_index* ix = g->ix;
  const uint32_t astride = ix->astride;
  cudaError_t e = cudaSuccess;
  if (count > g->rows_cap) {
    // Let the previous copies finish before the staging buffers are replaced.
    e = cudaStreamSynchronize(g->stream);
    if (g->h_rows) cudaFreeHost(g->h_rows);
    if (g->h_nodes) cudaFreeHost(g->h_nodes);
    if (g->d_rows) cudaFree(g->d_rows);
    if (g->d_nodes) cudaFree(g->d_nodes);
    g->h_rows = g->h_nodes = g->d_rows = g->d_nodes = nullptr;
    g->rows_cap = std::max<uint32_t>(count, 2 * g->rows_cap);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_rows), 4ull * astride * g->rows_cap, 0);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_nodes), 4ull * g->rows_cap, 0);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_rows), 4ull * astride * g->rows_cap);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_nodes), 4ull * g->rows_cap);
    if (e != cudaSuccess) return fail(DK_ERR_OUT_OF_MEMORY, std::string("build rows: ") + cudaGetErrorString(e));
  } else {
    e = cudaStreamSynchronize(g->stream);  // the staging buffers are about to be rewritten
    if (e != cudaSuccess) return cuda_fail(e, "build rows");
  }
  for (uint32_t r = 0; r < count; ++r) {
    const auto& lst = adj[nodes[r]];
    if (lst.size() > ix->max_degree) return fail(DK_ERR_INVALID_GRAPH, "adjacency list above max_degree");
    uint32_t* row = g->h_rows + (size_t)r * astride;
    row[0] = (uint32_t)lst.size();
    std::copy(lst.begin(), lst.end(), row + 1);
    std::fill(row + 1 + lst.size(), row + astride, 0u);
    g->h_nodes[r] = nodes[r];
  }
  e = cudaMemcpyAsync(g->d_rows, g->h_rows, 4ull * astride * count, cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->d_nodes, g->h_nodes, 4ull * count, cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) {
    const uint32_t blocks = std::min<uint32_t>(1184, (uint32_t)(((uint64_t)count * astride + 255) / 256));
    k_scatter_rows<<<blocks, 256, 0, g->stream>>>(ix->adj, astride, g->d_rows, g->d_nodes, count);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return cuda_fail(e, "build rows");
  return DK_OK;
}

namespace {

SearchParams prune_params(const dk_index* ix) {
  SearchParams P{};
  dk::base_params(ix, DK_STRATEGY_FULL_PRECISION, 1, 1, 1, P);
  return P;
}

PruneArgs prune_args(const dk_build_prune_cfg& cfg) {
  PruneArgs A{};
  A.alpha = cfg.alpha;
  A.degree = cfg.degree;
  A.max_occlusion = cfg.max_occlusion;
  A.occluding = cfg.occluding;
  return A;
}

}  // namespace

int32_t dk_build_gpu_prune_forward(dk_build_gpu* g, uint32_t count, const dk_build_prune_cfg& cfg,
                                   const uint32_t** out, const uint32_t** counts) {
  if (count != g->last_count) return fail(DK_ERR_INVALID_ARGUMENT, "prune of a batch that was not searched");
  dk::DeviceGuard guard(g->device);
  cudaError_t e = cudaSuccess;
  if (g->out_degree != cfg.degree) {
    cudaFree(g->d_out);
    cudaFree(g->d_out_cnt);
    if (g->h_out) cudaFreeHost(g->h_out);
    if (g->h_out_cnt) cudaFreeHost(g->h_out_cnt);
    g->d_out = g->d_out_cnt = g->h_out = g->h_out_cnt = nullptr;
    const size_t words = (size_t)g->max_batch * cfg.degree;
    e = cudaMalloc(reinterpret_cast<void**>(&g->d_out), 4 * words);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&g->d_out_cnt), 4ull * g->max_batch);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_out), 4 * words, 0);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_out_cnt), 4ull * g->max_batch, 0);
    if (e != cudaSuccess) return fail(DK_ERR_OUT_OF_MEMORY, std::string("prune buffers: ") + cudaGetErrorString(e));
    g->out_degree = cfg.degree;
  }
  const SearchParams P = prune_params(g->ix);
  PruneArgs A = prune_args(cfg);
  A.ntasks = count;
  A.start = g->last_start;
  A.rec_ids = g->d_rec_ids;
  A.rec_d = g->d_rec_d;
  A.rec_stats = g->d_stats;
  A.rec_cap = g->rec_cap;
  A.out = g->d_out;
  A.out_cnt = g->d_out_cnt;
  prune_layout(A, g->ix->dim, pow2_at_least(g->rec_cap));
  e = dispatch_prune<false>(g->ix->metric, P, A, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->h_out, g->d_out, 4ull * count * cfg.degree, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->h_out_cnt, g->d_out_cnt, 4ull * count, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "build prune");
  *out = g->h_out;
  *counts = g->h_out_cnt;
  return DK_OK;
}

int32_t dk_build_gpu_backedges(dk_build_gpu* g, const uint32_t* targets, const uint32_t* off,
                               const uint32_t* src, uint32_t groups, uint32_t max_group,
                               const dk_build_prune_cfg& cfg, std::vector<uint32_t>& oversize) {
  oversize.clear();
  if (groups == 0) return DK_OK;
  dk::DeviceGuard guard(g->device);
  // Staging: targets | offsets | oversize flags | second-tier group list | sources.
  const uint64_t nsrc = off[groups];
  const uint64_t words = 4ull * groups + 1 + nsrc;
  cudaError_t e = cudaStreamSynchronize(g->stream);  // the staging buffers may be in use
  if (e == cudaSuccess && words > g->groups_cap) {
    cudaFree(g->d_groups);
    if (g->h_groups) cudaFreeHost(g->h_groups);
    g->d_groups = g->h_groups = nullptr;
    g->groups_cap = std::max<uint64_t>(words, 2 * g->groups_cap);
    e = cudaMalloc(reinterpret_cast<void**>(&g->d_groups), 4 * g->groups_cap);
    if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void**>(&g->h_groups), 4 * g->groups_cap, 0);
    if (e != cudaSuccess) {
      g->groups_cap = 0;
      return fail(DK_ERR_OUT_OF_MEMORY, std::string("back-edge buffers: ") + cudaGetErrorString(e));
    }
  }
  if (e != cudaSuccess) return cuda_fail(e, "back edges");
  uint32_t* h = g->h_groups;
  uint32_t* d = g->d_groups;
  const uint64_t o_off = groups, o_flag = 2ull * groups + 1, o_list = 3ull * groups + 1,
                 o_src = 4ull * groups + 1;
  std::memcpy(h, targets, 4ull * groups);
  std::memcpy(h + o_off, off, 4ull * (groups + 1));
  std::memset(h + o_flag, 0, 4ull * groups);
  std::memcpy(h + o_src, src, 4ull * nsrc);
  e = cudaMemcpyAsync(d, h, 4 * (o_list), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d + o_src, h + o_src, 4 * nsrc, cudaMemcpyHostToDevice, g->stream);
  const SearchParams P = prune_params(g->ix);
  PruneArgs A = prune_args(cfg);
  A.targets = d;
  A.off = d + o_off;
  A.oversize = d + o_flag;
  A.src = d + o_src;
  A.adj = g->ix->adj;
  A.astride = g->ix->astride;
  A.max_degree = g->ix->max_degree;
  // Two tiers: every group with a pool of the list plus a few sources (small shared memory,
  // many warps resident), then the groups that did not fit with a pool for the largest group.
  // Lists beyond 4096 entries go to the caller.  Tests shrink the pools to exercise the
  // second tier (DK_BUILD_POOL_CAP_FIRST) and the caller's path (DK_BUILD_POOL_CAP).
  auto env_cap = [](const char* name, uint32_t dflt) {
    const char* v = getenv(name);
    return v ? std::max<uint32_t>(32u, pow2_at_least((uint32_t)atoi(v))) : dflt;
  };
  const uint32_t cap_limit = env_cap("DK_BUILD_POOL_CAP", 4096u);
  const uint32_t cap1 = std::min<uint32_t>(env_cap("DK_BUILD_POOL_CAP_FIRST", cap_limit),
                                           std::min<uint32_t>(cap_limit, pow2_at_least(g->ix->max_degree + 8u)));
  const uint32_t cap2 = std::min<uint32_t>(cap_limit, pow2_at_least(g->ix->max_degree + max_group));
  A.ntasks = groups;
  A.groups_of = nullptr;
  prune_layout(A, g->ix->dim, cap1);
  if (e == cudaSuccess) e = dispatch_prune<true>(g->ix->metric, P, A, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h + o_flag, A.oversize, 4ull * groups, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "back edges");
  uint32_t n2 = 0;
  for (uint32_t i = 0; i < groups; ++i)
    if (h[o_flag + i]) h[o_list + n2++] = i;
  if (n2 && cap2 > cap1) {
    std::memset(h + o_flag, 0, 4ull * groups);
    e = cudaMemcpyAsync(d + o_flag, h + o_flag, 4ull * (groups + n2), cudaMemcpyHostToDevice, g->stream);
    A.ntasks = n2;
    A.groups_of = d + o_list;
    prune_layout(A, g->ix->dim, cap2);
    if (e == cudaSuccess) e = dispatch_prune<true>(g->ix->metric, P, A, g->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h + o_flag, A.oversize, 4ull * groups, cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) return cuda_fail(e, "back edges");
    for (uint32_t i = 0; i < groups; ++i)
      if (h[o_flag + i]) oversize.push_back(i);
  } else {
    for (uint32_t i = 0; i < n2; ++i) oversize.push_back(h[o_list + i]);
  }
  return DK_OK;
}

int32_t dk_build_gpu_get_rows(dk_build_gpu* g, std::vector<std::vector<uint32_t>>& adj) {
  dk::DeviceGuard guard(g->device);
  const dk_index* ix = g->ix;
  const uint64_t total = (uint64_t)ix->n + ix->f;
  std::vector<uint32_t> rows(total * ix->astride);
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess) e = cudaMemcpy(rows.data(), ix->adj, 4 * rows.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "build rows read-back");
  adj.resize(total);
  for (uint64_t r = 0; r < total; ++r) {
    const uint32_t* row = rows.data() + r * ix->astride;
    adj[r].assign(row + 1, row + 1 + row[0]);
  }
  return DK_OK;
}

int32_t dk_build_gpu_get_row(dk_build_gpu* g, uint32_t node, std::vector<uint32_t>& out) {
  dk::DeviceGuard guard(g->device);
  const dk_index* ix = g->ix;
  std::vector<uint32_t> row(ix->astride);
  cudaError_t e = cudaStreamSynchronize(g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpy(row.data(), ix->adj + (size_t)node * ix->astride, 4ull * ix->astride, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "build row read-back");
  out.assign(row.begin() + 1, row.begin() + 1 + row[0]);
  return DK_OK;
}

void dk_build_gpu_destroy(dk_build_gpu* g) {
  if (!g) return;
  {
    dk::DeviceGuard guard(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    cudaFree(g->d_ids);
    cudaFree(g->d_dists);
    cudaFree(g->d_stats);
    cudaFree(g->d_rec_ids);
    cudaFree(g->d_rec_d);
    cudaFree(g->d_rows);
    cudaFree(g->d_nodes);
    cudaFree(g->d_out);
    cudaFree(g->d_out_cnt);
    cudaFree(g->d_groups);
    if (g->h_out) cudaFreeHost(g->h_out);
    if (g->h_out_cnt) cudaFreeHost(g->h_out_cnt);
    if (g->h_groups) cudaFreeHost(g->h_groups);
    if (g->h_stats) cudaFreeHost(g->h_stats);
    if (g->h_hops) cudaFreeHost(g->h_hops);
    if (g->h_rec_ids) cudaFreeHost(g->h_rec_ids);
    if (g->h_rec_d) cudaFreeHost(g->h_rec_d);
    if (g->h_rows) cudaFreeHost(g->h_rows);
    if (g->h_nodes) cudaFreeHost(g->h_nodes);
    if (g->stream) cudaStreamDestroy(g->stream);
  }
  if (g->ix) dk_index_destroy(g->ix);
  delete g;
}
