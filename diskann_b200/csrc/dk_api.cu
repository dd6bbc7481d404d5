// C ABI: index lifetime, validation, and the search entry points.
//
// The index is built once from host arrays (the reference's `DefaultProvider` stores:
// vectors, PQ codes, adjacency, frozen start points — inmem/provider.rs:227-352) and is
// read-only afterwards, so concurrent searches need no locking.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dk_internal.cuh"

namespace {

thread_local int32_t g_last_status = DK_OK;
thread_local std::string g_last_error;

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

int32_t cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? DK_ERR_OUT_OF_MEMORY : DK_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

inline uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

void free_index(dk_index* ix) {
  if (!ix) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ix->device);
  cudaFree(ix->vectors);
  cudaFree(ix->adj);
  cudaFree(ix->codes);
  cudaFree(ix->pivots);
  cudaFree(ix->pivots_cm);
  cudaFree(ix->offsets);
  cudaFree(ix->vec_bf16);
  cudaFree(ix->vec_fp8);
  cudaFree(ix->bf16_meta);
  cudaFree(ix->fp8_meta);
  cudaFree(ix->raw);
  cudaFree(ix->readable);
  cudaFree(ix->ext);
  cudaFree(ix->hint_dev);
  if (ix->hint_stage) cudaFreeHost(ix->hint_stage);
  if (ix->pool) cudaMemPoolDestroy(ix->pool);
  cudaSetDevice(prev);
  delete ix;
}


}  // namespace

int32_t dk_check_search_args(const dk_index* ix, int32_t strategy, uint32_t k, uint32_t l,
                             uint32_t beam, uint64_t qstride) {
  if (!ix) return fail(DK_ERR_INVALID_ARGUMENT, "index is null");
  const int32_t v = dk_knn_validate(k, l, beam);
  if (v != DK_OK) return v;
  if (strategy < DK_STRATEGY_FULL_PRECISION || strategy > DK_STRATEGY_FP8)
    return fail(DK_ERR_INVALID_ARGUMENT, "unknown strategy");
  if (strategy == DK_STRATEGY_HYBRID || strategy == DK_STRATEGY_QUANTIZED) {
    if (ix->pq_chunks == 0) return fail(DK_ERR_NO_PQ, "index has no PQ data");
  }
  if (strategy == DK_STRATEGY_BF16 && !ix->vec_bf16)
    return fail(DK_ERR_NO_LOW_PRECISION, "index was created without DK_INDEX_BF16");
  if (strategy == DK_STRATEGY_FP8 && !ix->vec_fp8)
    return fail(DK_ERR_NO_LOW_PRECISION, "index was created without DK_INDEX_FP8");
  if (beam > 64) return fail(DK_ERR_UNSUPPORTED, "beam_width above 64 is not supported");
  if ((uint64_t)l + ix->f > 16384) return fail(DK_ERR_UNSUPPORTED, "L above 16383 is not supported");
  if (qstride < ix->dim) return fail(DK_ERR_DIMENSION_MISMATCH, "query stride below dim");
  return DK_OK;
}

void dk_set_error(int32_t status, const std::string& msg) {
  g_last_status = status;
  g_last_error = msg;
}

extern "C" int32_t dk_abi_version(void) { return DK_ABI_VERSION; }

extern "C" int32_t dk_last_error(char* buf, uint64_t len) {
  if (buf && len) {
    const size_t n = std::min<size_t>(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = '\0';
  }
  return g_last_status;
}

// diskann/src/graph/search/knn_search.rs:94-119.
extern "C" int32_t dk_knn_validate(uint32_t k, uint32_t l, uint32_t beam_width) {
  if (k == 0) return fail(DK_ERR_K_ZERO, "k_value must be nonzero");
  if (l == 0) return fail(DK_ERR_L_ZERO, "l_value must be nonzero");
  if (k > l)
    return fail(DK_ERR_L_LESS_THAN_K, "l_value (" + std::to_string(l) +
                                          ") cannot be less than k_value (" + std::to_string(k) + ")");
  if (beam_width == 0) return fail(DK_ERR_BEAM_WIDTH_ZERO, "beam width must be nonzero");
  return DK_OK;
}

extern "C" int32_t dk_index_create(const dk_index_desc* d, int32_t device, dk_index** out) {
  if (!d || !out) return fail(DK_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (d->dim == 0) return fail(DK_ERR_INVALID_ARGUMENT, "dim must be nonzero");
  if (d->num_frozen == 0) return fail(DK_ERR_INVALID_ARGUMENT, "at least one frozen start point is required");
  if (!d->vectors || !d->adjacency || !d->degrees)
    return fail(DK_ERR_INVALID_ARGUMENT, "vectors, adjacency and degrees are required");
  if (d->vector_stride < d->dim) return fail(DK_ERR_DIMENSION_MISMATCH, "vector_stride below dim");
  if (d->max_degree == 0 || d->adjacency_stride < d->max_degree)
    return fail(DK_ERR_INVALID_ARGUMENT, "adjacency_stride below max_degree");
  if (d->metric < DK_METRIC_COSINE || d->metric > DK_METRIC_COSINE_NORMALIZED)
    return fail(DK_ERR_INVALID_ARGUMENT, "unknown metric");
  const uint64_t total = (uint64_t)d->num_points + d->num_frozen;
  if (total >= 0x7FFFFFFFull) return fail(DK_ERR_UNSUPPORTED, "more than 2^31-1 points");
  if (d->max_degree > 1024) return fail(DK_ERR_UNSUPPORTED, "max_degree above 1024");
  if (d->pq_chunks) {
    if (!d->pq_offsets || !d->pq_pivots || !d->pq_codes)
      return fail(DK_ERR_INVALID_ARGUMENT, "PQ offsets, pivots and codes are required");
    if (d->pq_offsets[0] != 0 || d->pq_offsets[d->pq_chunks] != d->dim)
      return fail(DK_ERR_INVALID_ARGUMENT, "PQ offsets must run from 0 to dim");
    for (uint32_t m = 0; m < d->pq_chunks; ++m)
      if (d->pq_offsets[m + 1] <= d->pq_offsets[m])
        return fail(DK_ERR_INVALID_ARGUMENT, "PQ offsets must be strictly increasing");
    if (d->pq_code_stride < d->pq_chunks) return fail(DK_ERR_INVALID_ARGUMENT, "pq_code_stride below pq_chunks");
    if ((uint64_t)d->pq_chunks * 256 * 4 > 160 * 1024)
      return fail(DK_ERR_UNSUPPORTED, "PQ table above 160 KB of shared memory");
  }

  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  if (device < 0 || device >= ndev) return fail(DK_ERR_INVALID_ARGUMENT, "no such CUDA device");
  dk::DeviceGuard guard(device);

  auto* ix = new dk_index();
  ix->device = device;
  ix->n = d->num_points;
  ix->f = d->num_frozen;
  ix->dim = d->dim;
  ix->metric = d->metric;
  ix->max_degree = d->max_degree;
  ix->pq_chunks = d->pq_chunks;
  ix->vstride = (uint32_t)round_up(d->dim, 4);
  ix->astride = (uint32_t)round_up(1 + d->max_degree, 4);
  ix->cstride = (uint32_t)round_up(std::max<uint32_t>(d->pq_chunks, 1), 16);

  // Adjacency rows [degree, ids...]: validate ids and degrees; drop repeated ids within a
  // list (keeping the first), which leaves search results unchanged because the visited
  // set already rejects a repeat (glue.rs:524-561).
  std::vector<uint32_t> adj((size_t)total * ix->astride, 0u);
  for (uint64_t r = 0; r < total; ++r) {
    const uint32_t deg = d->degrees[r];
    if (deg > d->max_degree) {
      free_index(ix);
      return fail(DK_ERR_INVALID_GRAPH, "node " + std::to_string(r) + " has degree " +
                                            std::to_string(deg) + " above max_degree");
    }
    uint32_t* dst = adj.data() + r * ix->astride;
    const uint32_t* src = d->adjacency + r * d->adjacency_stride;
    uint32_t w = 0;
    for (uint32_t t = 0; t < deg; ++t) {
      const uint32_t id = src[t];
      if (id >= total) {
        free_index(ix);
        return fail(DK_ERR_INVALID_GRAPH, "node " + std::to_string(r) + " lists neighbour id " +
                                              std::to_string(id) + " out of range");
      }
      bool dup = false;
      for (uint32_t u = 0; u < w; ++u) dup |= dst[1 + u] == id;
      if (!dup) dst[1 + w++] = id;
    }
    dst[0] = w;
  }

  // Vectors, padded rows.
  std::vector<float> vec((size_t)total * ix->vstride, 0.0f);
  for (uint64_t r = 0; r < total; ++r)
    std::memcpy(vec.data() + r * ix->vstride, d->vectors + r * d->vector_stride, d->dim * sizeof(float));

  auto upload = [&](void** dst, const void* src, size_t bytes) -> cudaError_t {
    cudaError_t err = cudaMalloc(dst, bytes);
    if (err != cudaSuccess) return err;
    ix->bytes += bytes;
    return cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
  };
  e = upload(reinterpret_cast<void**>(&ix->vectors), vec.data(), vec.size() * sizeof(float));
  if (e == cudaSuccess)
    e = upload(reinterpret_cast<void**>(&ix->adj), adj.data(), adj.size() * sizeof(uint32_t));
  if (e == cudaSuccess && d->pq_chunks) {
    std::vector<uint8_t> codes((size_t)total * ix->cstride, 0u);
    for (uint64_t r = 0; r < total; ++r)
      std::memcpy(codes.data() + r * ix->cstride, d->pq_codes + r * d->pq_code_stride, d->pq_chunks);
    e = upload(reinterpret_cast<void**>(&ix->codes), codes.data(), codes.size());
    if (e == cudaSuccess)
      e = upload(reinterpret_cast<void**>(&ix->pivots), d->pq_pivots, (size_t)256 * d->dim * sizeof(float));
    if (e == cudaSuccess) {
      // Chunk-major pivots: chunk m's 256 centres are contiguous runs of len_m floats.
      std::vector<float> cm((size_t)256 * d->dim);
      for (uint32_t m = 0; m < d->pq_chunks; ++m) {
        const uint32_t s = d->pq_offsets[m], len = d->pq_offsets[m + 1] - s;
        for (uint32_t c = 0; c < 256; ++c)
          std::memcpy(&cm[(size_t)s * 256 + (size_t)c * len], d->pq_pivots + (size_t)c * d->dim + s,
                      len * sizeof(float));
      }
      e = upload(reinterpret_cast<void**>(&ix->pivots_cm), cm.data(), cm.size() * sizeof(float));
    }
    if (e == cudaSuccess)
      e = upload(reinterpret_cast<void**>(&ix->offsets), d->pq_offsets, (d->pq_chunks + 1) * sizeof(uint32_t));
  }
  if (e == cudaSuccess && (d->flags & (DK_INDEX_BF16 | DK_INDEX_FP8)))
    e = dk_build_low_precision(ix, d->flags);
  if (e == cudaSuccess) {
    e = cudaMalloc(reinterpret_cast<void**>(&ix->hint_dev), 4 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemset(ix->hint_dev, 0, 4 * sizeof(uint32_t));
    if (e == cudaSuccess)
      e = cudaHostAlloc(reinterpret_cast<void**>(&ix->hint_stage), 4 * sizeof(uint32_t), cudaHostAllocDefault);
    if (e == cudaSuccess) std::memset(ix->hint_stage, 0, 4 * sizeof(uint32_t));
  }
  if (e == cudaSuccess) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    e = cudaMemPoolCreate(&ix->pool, &props);
    uint64_t keep = UINT64_MAX;
    if (e == cudaSuccess) e = cudaMemPoolSetAttribute(ix->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e != cudaSuccess) {
    free_index(ix);
    return cuda_fail(e, "index upload");
  }
  *out = ix;
  return DK_OK;
}

extern "C" int32_t dk_index_destroy(dk_index* index) {
  if (!index) return fail(DK_ERR_INVALID_ARGUMENT, "index is null");
  free_index(index);
  return DK_OK;
}

extern "C" int32_t dk_index_get_info(const dk_index* ix, dk_index_info* info) {
  if (!ix || !info) return fail(DK_ERR_INVALID_ARGUMENT, "null argument");
  info->num_points = ix->n;
  info->num_frozen = ix->f;
  info->dim = ix->dim;
  info->max_degree = ix->max_degree;
  info->pq_chunks = ix->pq_chunks;
  info->metric = ix->metric;
  info->device = ix->device;
  info->device_bytes = ix->bytes;
  return DK_OK;
}

extern "C" int32_t dk_search_device(dk_index* ix, int32_t strategy, const float* queries,
                                    uint64_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                                    uint32_t beam_width, uint32_t* ids, float* dists,
                                    dk_search_stats* stats, void* stream) {
  const int32_t v = dk_check_search_args(ix, strategy, k, l, beam_width, query_stride);
  if (v != DK_OK) return v;
  if (nq && (!queries || !ids || !dists || !stats))
    return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids, dists and stats are required");
  dk::DeviceGuard guard(ix->device);
  return dk_launch_search(ix, strategy, queries, query_stride, nq, k, l, beam_width, ids, dists,
                          stats, static_cast<cudaStream_t>(stream));
}

extern "C" int32_t dk_search(dk_index* ix, int32_t strategy, const float* queries,
                             uint64_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                             uint32_t beam_width, uint32_t* ids, float* dists,
                             dk_search_stats* stats) {
  const int32_t v = dk_check_search_args(ix, strategy, k, l, beam_width, query_stride);
  if (v != DK_OK) return v;
  if (nq == 0) return DK_OK;
  if (!queries || !ids || !dists) return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids and dists are required");
  dk::DeviceGuard guard(ix->device);
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate");
  const size_t qbytes = (size_t)nq * ix->dim * sizeof(float);
  const size_t obytes = (size_t)nq * k;
  unsigned char* buf = nullptr;
  const size_t off_ids = round_up(qbytes, 256);
  const size_t off_d = off_ids + round_up(obytes * 4, 256);
  const size_t off_st = off_d + round_up(obytes * 4, 256);
  const size_t total = off_st + (size_t)nq * sizeof(dk_search_stats);
  int32_t rc = DK_OK;
  e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&buf), total, ix->pool, s);
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return cuda_fail(e, "cudaMallocFromPoolAsync");
  }
  float* dq = reinterpret_cast<float*>(buf);
  uint32_t* dids = reinterpret_cast<uint32_t*>(buf + off_ids);
  float* dd = reinterpret_cast<float*>(buf + off_d);
  dk_search_stats* dst = reinterpret_cast<dk_search_stats*>(buf + off_st);
  if (query_stride == ix->dim) {
    e = cudaMemcpyAsync(dq, queries, qbytes, cudaMemcpyHostToDevice, s);
  } else {
    e = cudaMemcpy2DAsync(dq, ix->dim * sizeof(float), queries, query_stride * sizeof(float),
                          ix->dim * sizeof(float), nq, cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) {
    rc = dk_launch_search(ix, strategy, dq, ix->dim, nq, k, l, beam_width, dids, dd, dst, s);
    if (rc == DK_OK) {
      e = cudaMemcpyAsync(ids, dids, obytes * 4, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaMemcpyAsync(dists, dd, obytes * 4, cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess && stats)
        e = cudaMemcpyAsync(stats, dst, (size_t)nq * sizeof(dk_search_stats), cudaMemcpyDeviceToHost, s);
    }
  }
  cudaFreeAsync(buf, s);
  const cudaError_t es = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (rc != DK_OK) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "search copy");
  if (es != cudaSuccess) return cuda_fail(es, "search");
  return DK_OK;
}
