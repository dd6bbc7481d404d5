// Low-precision copies of the vector store for the BF16 / FP8 traversal strategies.
//
//  * BF16: each element rounded to nearest even (__float2bfloat16_rn).
//  * FP8-E4M3 with one FP32 scale per vector: scale = max|x| / 448 (448 is the largest
//    finite E4M3 value; an all-zero row gets scale 1), element = saturating E4M3 of x / scale.
// Rows are `lp_stride` elements (a multiple of 16) so every row starts 16-byte aligned and
// the padding is zero.

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dk_internal.cuh"

namespace {

__global__ void k_to_bf16(const float* __restrict__ src, uint32_t vstride, uint32_t dim,
                          uint16_t* __restrict__ dst, uint32_t lps, uint64_t rows) {
  const uint64_t total = rows * lps;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / lps;
    const uint32_t c = (uint32_t)(i - r * lps);
    const float x = c < dim ? src[r * vstride + c] : 0.0f;
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    dst[i] = *reinterpret_cast<const uint16_t*>(&b);
  }
}

// One warp per row.
__global__ void k_to_fp8(const float* __restrict__ src, uint32_t vstride, uint32_t dim,
                         uint8_t* __restrict__ dst, float* __restrict__ scale, uint32_t lps,
                         uint64_t rows) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
       r += warps) {
    const float* row = src + r * vstride;
    float m = 0.0f;
    for (uint32_t c = lane; c < dim; c += 32u) m = fmaxf(m, fabsf(row[c]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xFFFFFFFFu, m, o));
    const float s = m > 0.0f ? m / 448.0f : 1.0f;
    if (lane == 0) scale[r] = s;
    for (uint32_t c = lane; c < lps; c += 32u) {
      const float x = c < dim ? row[c] / s : 0.0f;
      dst[r * lps + c] = (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
    }
  }
}

}  // namespace

cudaError_t dk_build_low_precision(dk_index* ix, uint32_t flags) {
  const uint64_t rows = (uint64_t)ix->n + ix->f;
  ix->lp_stride = (ix->dim + 15u) & ~15u;
  cudaError_t e = cudaSuccess;
  if (flags & DK_INDEX_BF16) {
    const size_t bytes = rows * ix->lp_stride * sizeof(uint16_t);
    e = cudaMalloc(reinterpret_cast<void**>(&ix->vec_bf16), bytes);
    if (e != cudaSuccess) return e;
    ix->bytes += bytes;
    k_to_bf16<<<1184, 256>>>(ix->vectors, ix->vstride, ix->dim, ix->vec_bf16, ix->lp_stride, rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (flags & DK_INDEX_FP8) {
    const size_t bytes = rows * ix->lp_stride;
    e = cudaMalloc(reinterpret_cast<void**>(&ix->vec_fp8), bytes);
    if (e != cudaSuccess) return e;
    ix->bytes += bytes;
    e = cudaMalloc(reinterpret_cast<void**>(&ix->fp8_scale), rows * sizeof(float));
    if (e != cudaSuccess) return e;
    ix->bytes += rows * sizeof(float);
    k_to_fp8<<<1184, 256>>>(ix->vectors, ix->vstride, ix->dim, ix->vec_fp8, ix->fp8_scale,
                            ix->lp_stride, rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaDeviceSynchronize();
}
