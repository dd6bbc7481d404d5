// Device side of graph construction; see dk_build_gpu.h.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "dk_build_gpu.h"
#include "dk_internal.cuh"

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
};

namespace {

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

int32_t dk_build_gpu_search(dk_build_gpu* g, uint32_t start, uint32_t count,
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
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->h_rec_ids, g->d_rec_ids, 4ull * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->h_rec_d, g->d_rec_d, 4ull * n, cudaMemcpyDeviceToHost, g->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  if (e != cudaSuccess) return cuda_fail(e, "build search");
  for (uint32_t i = 0; i < count; ++i) g->h_hops[i] = g->h_stats[i].hops;
  *rec_ids = g->h_rec_ids;
  *rec_d = g->h_rec_d;
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
