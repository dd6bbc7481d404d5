// dk_score_candidates: the distance each strategy scores a candidate with during traversal,
// for a batch of (query, candidate list) pairs.  This is the accessor's per-candidate distance
// of the reference batched on the device: the preprocessed query distance of the FullPrecision
// accessor (diskann/src/utils/vector_repr.rs:48-93, diskann-vector/src/distance/
// implementations.rs:215-405), the PQ QueryComputer of the quantised accessors
// (diskann-providers/src/model/pq/distance/dynamic.rs:64-84), and, for the BF16 / FP8
// strategies (no counterpart in the reference), the low-precision distance that steers their
// traversal.  Every strategy runs the same device scorer as the search kernels, so
// FullPrecision distances are bit-exact and the others equal what the search uses.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "dk_kernels.cuh"

namespace {

constexpr uint32_t kChunk = 1024;  // candidates scored per round (shared-memory lists)

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

// One warp per query: the query's state (FP32 copy, or the PQ table) is built once, then its
// candidates are scored kChunk at a time.  An id outside the index scores NaN and reads nothing.
template <int METRIC, int MODE>
__global__ void __launch_bounds__(32) k_score(const SearchParams P, const uint32_t* ids,
                                              uint32_t per, float* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const dk::State S = dk::carve(smem, P);
  const uint32_t q = blockIdx.x, lane = threadIdx.x;
  const float* qsrc = P.queries + (size_t)q * P.qstride;
  const uint32_t dpad = (P.dim + 15u) & ~15u;  // zero padded: FP8 pieces hold 16 elements
  for (uint32_t i = lane; i < dpad; i += 32u) S.q[i] = i < P.dim ? qsrc[i] : 0.0f;
  __syncwarp();
  if constexpr (MODE == kModePQ && METRIC != DK_METRIC_COSINE) {
    dk::build_table<METRIC>(P, S.q, S.table, lane, 32u);
    __syncwarp();
  }
  const uint32_t total = P.n + P.f;
  const uint32_t* qids = ids + (size_t)q * per;
  float* qout = out + (size_t)q * per;
  for (uint32_t c0 = 0; c0 < per; c0 += kChunk) {
    const uint32_t n = min(kChunk, per - c0);
    for (uint32_t i = lane; i < n; i += 32u) {
      const uint32_t id = qids[c0 + i];
      S.cand_id[i] = id < total ? id : 0u;
    }
    __syncwarp();
    dk::warp_score<METRIC, MODE, 0, 1>(P, S, S.cand_id, S.cand_d, n, lane);
    for (uint32_t i = lane; i < n; i += 32u)
      qout[c0 + i] = qids[c0 + i] < total ? S.cand_d[i] : __int_as_float(0x7FC00000);
    __syncwarp();
  }
}

template <int METRIC>
cudaError_t launch_metric(int mode, const SearchParams& P, const uint32_t* ids, uint32_t per,
                          float* out, cudaStream_t stream) {
  auto go = [&](auto kernel) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)P.smem_bytes);
    if (e != cudaSuccess) return e;
    kernel<<<P.nq, 32, P.smem_bytes, stream>>>(P, ids, per, out);
    return cudaGetLastError();
  };
  switch (mode) {
    case kModePQ: return go(k_score<METRIC, kModePQ>);
    case kModeBF16: return go(k_score<METRIC, kModeBF16>);
    case kModeFP8: return go(k_score<METRIC, kModeFP8>);
    default: return go(k_score<METRIC, kModeFP32>);
  }
}

}  // namespace

extern "C" int32_t dk_score_candidates(dk_index* ix, int32_t strategy, const float* queries,
                                       uint64_t query_stride, uint32_t nq, const uint32_t* ids,
                                       uint32_t per_query, float* dists, void* stream_) {
  const int32_t v = dk_check_search_args(ix, strategy, 1, 1, 1, query_stride);
  if (v != DK_OK) return v;
  if (nq == 0 || per_query == 0) return DK_OK;
  if (!queries || !ids || !dists)
    return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids and dists are required");
  if (nq > 0x7FFFFFFFu) return fail(DK_ERR_INVALID_ARGUMENT, "nq above 2^31 - 1");
  dk::DeviceGuard guard(ix->device);
  const int mode = mode_of_strategy(strategy);
  SearchParams P{};
  dk::base_params(ix, strategy, 1, 1, 1, P);
  P.queries = queries;
  P.qstride = query_stride;
  P.nq = nq;
  P.list_cap = std::max<uint32_t>(P.list_cap, kChunk);
  P.smem_bytes = dk::plan_query_smem(P, mode == kModePQ, false);
  int max_optin = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device);
  if (P.smem_bytes > (uint32_t)max_optin)
    return fail(DK_ERR_UNSUPPORTED, "query state does not fit in shared memory");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);
  cudaError_t e;
  switch (ix->metric) {
    case DK_METRIC_L2: e = launch_metric<DK_METRIC_L2>(mode, P, ids, per_query, dists, stream); break;
    case DK_METRIC_INNER_PRODUCT:
      e = launch_metric<DK_METRIC_INNER_PRODUCT>(mode, P, ids, per_query, dists, stream);
      break;
    case DK_METRIC_COSINE: e = launch_metric<DK_METRIC_COSINE>(mode, P, ids, per_query, dists, stream); break;
    default:
      e = launch_metric<DK_METRIC_COSINE_NORMALIZED>(mode, P, ids, per_query, dists, stream);
      break;
  }
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("score launch: ") + cudaGetErrorString(e));
  return DK_OK;
}
