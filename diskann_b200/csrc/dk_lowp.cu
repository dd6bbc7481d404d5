// Low-precision copies of the vector store for the BF16 / FP8 traversal strategies.
//
//  * BF16: each element rounded to nearest even (__float2bfloat16_rn); scale 1.
//  * FP8-E4M3 with one FP32 scale per vector: scale = max|x| / 448 (448 is the largest
//    finite E4M3 value; an all-zero row gets scale 1), element = saturating E4M3 of x / scale.
// Rows are `lp_stride` elements (a multiple of 16) so every row starts 16-byte aligned and
// the padding is zero.  Beside each row: (scale, squared norm of the de-quantised row), so
// the traversal kernels score with one multiply-add per element: |q - s x|^2 =
// |q|^2 + norm - 2 s (q . x).

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dk_internal.cuh"

namespace {

// One warp per row.
__global__ void k_to_bf16(const float* __restrict__ src, uint32_t vstride, uint32_t dim,
                          uint16_t* __restrict__ dst, float2* __restrict__ meta, uint32_t lps,
                          uint64_t rows) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t r = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); r < rows;
       r += warps) {
    const float* row = src + r * vstride;
    float nn = 0.0f;
    for (uint32_t c = lane; c < lps; c += 32u) {
      const float x = c < dim ? row[c] : 0.0f;
      const __nv_bfloat16 b = __float2bfloat16_rn(x);
      dst[r * lps + c] = *reinterpret_cast<const uint16_t*>(&b);
      const float y = __bfloat162float(b);
      nn = __fmaf_rn(y, y, nn);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xFFFFFFFFu, nn, o);
    if (lane == 0) meta[r] = make_float2(1.0f, nn);
  }
}

// One warp per row.
__global__ void k_to_fp8(const float* __restrict__ src, uint32_t vstride, uint32_t dim,
                         uint8_t* __restrict__ dst, float2* __restrict__ meta, uint32_t lps,
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
    float nn = 0.0f;
    for (uint32_t c = lane; c < lps; c += 32u) {
      const float x = c < dim ? row[c] / s : 0.0f;
      const __nv_fp8_storage_t f = __nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3);
      dst[r * lps + c] = (uint8_t)f;
      const __half_raw h = __nv_cvt_fp8_to_halfraw(f, __NV_E4M3);
      const float y = s * __half2float(*reinterpret_cast<const __half*>(&h));
      nn = __fmaf_rn(y, y, nn);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nn += __shfl_xor_sync(0xFFFFFFFFu, nn, o);
    if (lane == 0) meta[r] = make_float2(s, nn);
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
    e = cudaMalloc(reinterpret_cast<void**>(&ix->bf16_meta), rows * sizeof(float2));
    if (e != cudaSuccess) return e;
    ix->bytes += bytes + rows * sizeof(float2);
    k_to_bf16<<<1184, 256>>>(ix->vectors, ix->vstride, ix->dim, ix->vec_bf16, ix->bf16_meta,
                             ix->lp_stride, rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (flags & DK_INDEX_FP8) {
    const size_t bytes = rows * ix->lp_stride;
    e = cudaMalloc(reinterpret_cast<void**>(&ix->vec_fp8), bytes);
    if (e != cudaSuccess) return e;
    e = cudaMalloc(reinterpret_cast<void**>(&ix->fp8_meta), rows * sizeof(float2));
    if (e != cudaSuccess) return e;
    ix->bytes += bytes + rows * sizeof(float2);
    k_to_fp8<<<1184, 256>>>(ix->vectors, ix->vstride, ix->dim, ix->vec_fp8, ix->fp8_meta,
                            ix->lp_stride, rows);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaDeviceSynchronize();
}
