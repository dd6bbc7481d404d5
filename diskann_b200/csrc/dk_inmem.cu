// The diskann-inmem provider on the GPU: its store (typed rows with an in-row concurrency tag,
// external ids per slot) and its search (diskann-inmem/src/provider.rs:380-960).
//
// The index is an ordinary dk_index (adjacency, an FP32 copy of the rows, the pool) plus the
// rows in their element type, one readable bit per slot taken from the tags, and the
// external-id table.  Search runs the CTA search loop (cta_search) with an exact per-CTA
// bitmap as the visited set, one 128-thread CTA per query, persistent over the batch; the
// readable bits make unreadable neighbours visited-but-unscored, and the post-processor
// translates ids (Translate, provider.rs:906-945).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "dk_kernels.cuh"

namespace {

using namespace dk;

constexpr uint8_t kTagPublished = 254;  // tag.rs: PUBLISHED = u8::MAX - 1, FROZEN = u8::MAX

struct TranslateOut {
  const uint64_t* ext;
  uint64_t* ids;  // nq x k external ids
};

// Translate (provider.rs:906-945): the queue's entries in order, those with an external id,
// up to k, written as external ids.
template <int NT>
__device__ void cta_translate(const SearchParams& P, const State& S, const TranslateOut& T,
                              uint32_t qid) {
  const uint32_t tid = threadIdx.x;
  Misc* M = S.misc;
  const uint32_t size = M->size;
  const float* qd = S.qd[M->cur];
  const uint32_t* qi = S.qi[M->cur];
  uint64_t* out_ids = T.ids + (size_t)qid * P.k;
  float* out_d = P.out_dists + (size_t)qid * P.k;
  uint32_t base = 0;
  for (uint32_t t0 = 0; t0 < size && base < P.k; t0 += NT) {
    const uint32_t i = t0 + tid;
    uint64_t ext = DK_NO_EXTERNAL_ID;
    if (i < size) ext = __ldg(reinterpret_cast<const unsigned long long*>(T.ext) + (qi[i] & kIdMask));
    const bool keep = ext != DK_NO_EXTERNAL_ID;
    uint32_t total;
    const uint32_t pos = base + block_scan<NT>(keep, M->warp_sums, total);
    if (keep && pos < P.k) {
      out_ids[pos] = ext;
      out_d[pos] = qd[i];
    }
    base += total;
  }
  const uint32_t written = min(base, P.k);
  for (uint32_t j = written + tid; j < P.k; j += NT) {
    out_ids[j] = DK_NO_EXTERNAL_ID;
    out_d[j] = INFINITY;
  }
  if (tid == 0) M->result_count = written;
}

template <int NT, int METRIC, int MODE, int DIM>
__global__ void __launch_bounds__(NT) k_inmem(const SearchParams P, const TranslateOut T) {
  extern __shared__ __align__(16) unsigned char smem[];
  const State S = carve(smem, P);
  const BitmapSet vset{P.bitmap + (size_t)blockIdx.x * P.bitmap_words, P.bitmap_words};
  for (uint32_t qid = blockIdx.x; qid < P.nq; qid += gridDim.x) {
    __syncthreads();
    uint32_t cmps = 0, hops = 0;
    cta_search<NT, METRIC, MODE, DIM>(P, S, vset, qid, cmps, hops);
    __syncthreads();
    cta_translate<NT>(P, S, T, qid);
    __syncthreads();
    if (threadIdx.x == 0) P.stats[qid] = dk_search_stats{cmps, hops, S.misc->result_count, 0u};
  }
}

// Launches the kernel, or with `occupancy` set only reports its resident CTAs per SM.
template <int METRIC, int MODE, int DIM>
cudaError_t launch_inmem(const SearchParams& P, const TranslateOut& T, uint32_t grid,
                         cudaStream_t stream, int* occupancy) {
  auto k = k_inmem<kCtaThreads, METRIC, MODE, DIM>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)P.smem_bytes);
  if (e != cudaSuccess) return e;
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, k, kCtaThreads, P.smem_bytes);
  k<<<grid, kCtaThreads, P.smem_bytes, stream>>>(P, T);
  return cudaGetLastError();
}

template <int METRIC>
cudaError_t inmem_modes(int32_t elem, const SearchParams& P, const TranslateOut& T,
                        uint32_t grid, cudaStream_t stream, int* occupancy) {
  const bool d128 = P.dim == 128;
  switch (elem) {
    case DK_ELEM_F32:
      return d128 ? launch_inmem<METRIC, kModeFP32, 128>(P, T, grid, stream, occupancy)
                  : launch_inmem<METRIC, kModeFP32, 0>(P, T, grid, stream, occupancy);
    case DK_ELEM_F16:
      return d128 ? launch_inmem<METRIC, kModeF16, 128>(P, T, grid, stream, occupancy)
                  : launch_inmem<METRIC, kModeF16, 0>(P, T, grid, stream, occupancy);
    case DK_ELEM_U8: return launch_inmem<METRIC, kModeU8, 0>(P, T, grid, stream, occupancy);
    default: return launch_inmem<METRIC, kModeI8, 0>(P, T, grid, stream, occupancy);
  }
}

// u8 / i8 with CosineNormalized score as cosine (layers/full.rs:458-470, 487-492).
cudaError_t inmem_dispatch(const dk_index* ix, const SearchParams& P, const TranslateOut& T,
                           uint32_t grid, cudaStream_t stream, int* occupancy) {
  const int32_t elem = ix->elem;
  const bool int_elem = elem == DK_ELEM_U8 || elem == DK_ELEM_I8;
  switch (ix->metric) {
    case DK_METRIC_L2: return inmem_modes<DK_METRIC_L2>(elem, P, T, grid, stream, occupancy);
    case DK_METRIC_INNER_PRODUCT:
      return inmem_modes<DK_METRIC_INNER_PRODUCT>(elem, P, T, grid, stream, occupancy);
    case DK_METRIC_COSINE: return inmem_modes<DK_METRIC_COSINE>(elem, P, T, grid, stream, occupancy);
    default:
      return int_elem ? inmem_modes<DK_METRIC_COSINE>(elem, P, T, grid, stream, occupancy)
                      : inmem_modes<DK_METRIC_COSINE_NORMALIZED>(elem, P, T, grid, stream, occupancy);
  }
}

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

uint32_t elem_bytes(int32_t elem) {
  return elem == DK_ELEM_F32 ? 4u : (elem == DK_ELEM_F16 ? 2u : 1u);
}

// Element i of a typed row as a float (exact for every element type).
float elem_value(int32_t elem, const uint8_t* row, uint32_t i) {
  switch (elem) {
    case DK_ELEM_F32: {
      float v;
      std::memcpy(&v, row + 4u * i, 4);
      return v;
    }
    case DK_ELEM_F16: {
      uint16_t h;
      std::memcpy(&h, row + 2u * i, 2);
      // IEEE binary16 -> binary32, exact.
      const uint32_t sign = (uint32_t)(h >> 15) << 31, ex = (h >> 10) & 0x1Fu, man = h & 0x3FFu;
      uint32_t bits;
      if (ex == 0x1F) {
        bits = sign | 0x7F800000u | (man << 13);
      } else if (ex != 0) {
        bits = sign | ((ex + 112u) << 23) | (man << 13);
      } else if (man == 0) {
        bits = sign;
      } else {  // subnormal: normalise
        uint32_t m = man, e = 113u;
        while (!(m & 0x400u)) {
          m <<= 1;
          --e;
        }
        bits = sign | (e << 23) | ((m & 0x3FFu) << 13);
      }
      float v;
      std::memcpy(&v, &bits, 4);
      return v;
    }
    case DK_ELEM_U8: return (float)row[i];
    default: return (float)(int8_t)row[i];
  }
}

}  // namespace

extern "C" int32_t dk_inmem_index_create(const dk_inmem_desc* d, int32_t device, dk_index** out) {
  if (!d || !out) return fail(DK_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (d->elem < DK_ELEM_F32 || d->elem > DK_ELEM_I8) return fail(DK_ERR_INVALID_ARGUMENT, "unknown element type");
  if (!d->rows || !d->external_ids) return fail(DK_ERR_INVALID_ARGUMENT, "rows and external_ids are required");
  const uint32_t eb = elem_bytes(d->elem);
  if (d->dim == 0) return fail(DK_ERR_INVALID_ARGUMENT, "dim must be nonzero");
  if (d->row_stride < (uint64_t)d->dim * eb + 1)
    return fail(DK_ERR_INVALID_ARGUMENT, "row_stride leaves no room for the tag");
  if (d->elem != DK_ELEM_F32 && d->elem != DK_ELEM_F16 && d->dim > 33000)
    return fail(DK_ERR_UNSUPPORTED, "integer rows above 33000 elements");
  const uint64_t total = (uint64_t)d->capacity + d->num_frozen;
  if (total >= 0x7FFFFFFFull) return fail(DK_ERR_UNSUPPORTED, "more than 2^31-1 slots");
  for (uint64_t r = d->capacity; r < total; ++r)
    if (d->rows[r * d->row_stride + (uint64_t)d->dim * eb] < kTagPublished)
      return fail(DK_ERR_INVALID_ARGUMENT, "start point " + std::to_string(r) + " is not readable");

  // The shared parts (validated adjacency, an FP32 copy of the rows, pool) come from the
  // ordinary index.
  std::vector<float> vec((size_t)total * d->dim);
  for (uint64_t r = 0; r < total; ++r)
    for (uint32_t i = 0; i < d->dim; ++i)
      vec[r * d->dim + i] = elem_value(d->elem, d->rows + r * d->row_stride, i);
  dk_index_desc base{};
  base.num_points = d->capacity;
  base.num_frozen = d->num_frozen;
  base.dim = d->dim;
  base.metric = d->metric;
  base.vectors = vec.data();
  base.vector_stride = d->dim;
  base.adjacency = d->adjacency;
  base.adjacency_stride = d->adjacency_stride;
  base.degrees = d->degrees;
  base.max_degree = d->max_degree;
  dk_index* ix = nullptr;
  int32_t rc = dk_index_create(&base, device, &ix);
  if (rc != DK_OK) return rc;
  vec.clear();
  vec.shrink_to_fit();
  dk::DeviceGuard guard(device);
  ix->elem = d->elem;
  // Typed rows, zero padded to a multiple of 32 bytes (integer scoring reads whole words of
  // 8 lanes; FP16 scoring reads 8-byte pieces).
  cudaError_t e = cudaSuccess;
  if (d->elem != DK_ELEM_F32) {
    const uint32_t stride = (uint32_t)((d->dim * eb + 31u) / 32u * 32u);
    std::vector<uint8_t> raw((size_t)total * stride, 0u);
    for (uint64_t r = 0; r < total; ++r)
      std::memcpy(raw.data() + r * stride, d->rows + r * d->row_stride, (size_t)d->dim * eb);
    ix->raw_stride = stride;
    e = cudaMalloc(reinterpret_cast<void**>(&ix->raw), raw.size());
    if (e == cudaSuccess) e = cudaMemcpy(ix->raw, raw.data(), raw.size(), cudaMemcpyHostToDevice);
    ix->bytes += raw.size();
  }
  const size_t words = (size_t)(total + 31u) / 32u;
  std::vector<uint32_t> bits(words, 0u);
  for (uint64_t r = 0; r < total; ++r)
    if (d->rows[r * d->row_stride + (uint64_t)d->dim * eb] >= kTagPublished) bits[r >> 5] |= 1u << (r & 31u);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&ix->readable), words * 4);
  if (e == cudaSuccess) e = cudaMemcpy(ix->readable, bits.data(), words * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&ix->ext), total * 8);
  if (e == cudaSuccess) e = cudaMemcpy(ix->ext, d->external_ids, total * 8, cudaMemcpyHostToDevice);
  ix->bytes += words * 4 + total * 8;
  if (e != cudaSuccess) {
    dk_index_destroy(ix);
    return fail(DK_ERR_CUDA, std::string("inmem store upload: ") + cudaGetErrorString(e));
  }
  *out = ix;
  return DK_OK;
}

extern "C" int32_t dk_inmem_set_tags(dk_index* ix, uint32_t first, uint32_t count, const uint8_t* tags) {
  if (!ix || ix->elem < 0) return fail(DK_ERR_INVALID_ARGUMENT, "not a diskann-inmem index");
  if (count == 0) return DK_OK;
  if (!tags) return fail(DK_ERR_INVALID_ARGUMENT, "tags is null");
  const uint64_t total = (uint64_t)ix->n + ix->f;
  if ((uint64_t)first + count > total) return fail(DK_ERR_INVALID_ARGUMENT, "slots out of range");
  for (uint32_t i = 0; i < count; ++i)
    if ((uint64_t)first + i >= ix->n && tags[i] < kTagPublished)
      return fail(DK_ERR_INVALID_ARGUMENT, "start points must stay readable");
  dk::DeviceGuard guard(ix->device);
  // Read-modify-write of the covering words.
  const uint32_t w0 = first >> 5, w1 = (uint32_t)(((uint64_t)first + count + 31u) >> 5);
  std::vector<uint32_t> bits(w1 - w0);
  cudaError_t e = cudaMemcpy(bits.data(), ix->readable + w0, bits.size() * 4, cudaMemcpyDeviceToHost);
  for (uint32_t i = 0; i < count; ++i) {
    const uint32_t id = first + i, w = (id >> 5) - w0, b = 1u << (id & 31u);
    if (tags[i] >= kTagPublished) bits[w] |= b;
    else bits[w] &= ~b;
  }
  if (e == cudaSuccess) e = cudaMemcpy(ix->readable + w0, bits.data(), bits.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("set tags: ") + cudaGetErrorString(e));
  return DK_OK;
}

extern "C" int32_t dk_inmem_search(dk_index* ix, const void* queries, uint64_t query_stride,
                                   uint32_t nq, uint32_t k, uint32_t l, uint32_t beam,
                                   uint64_t* ids, float* dists, dk_search_stats* stats) {
  if (!ix || ix->elem < 0) return fail(DK_ERR_INVALID_ARGUMENT, "not a diskann-inmem index");
  const int32_t v = dk_check_search_args(ix, DK_STRATEGY_FULL_PRECISION, k, l, beam, query_stride);
  if (v != DK_OK) return v;
  if (nq == 0) return DK_OK;
  if (!queries || !ids || !dists) return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids and dists are required");
  const int32_t elem = ix->elem;
  const uint32_t eb = elem_bytes(elem), dim = ix->dim;
  // Device query rows of `dim` floats: f32 values (f16 queries converted, as the f16 layer
  // does), or for u8 / i8 the packed bytes in the first words, zero padded.
  std::vector<float> qh((size_t)nq * dim, 0.0f);
  for (uint32_t q = 0; q < nq; ++q) {
    const uint8_t* src = static_cast<const uint8_t*>(queries) + (size_t)q * query_stride * eb;
    float* dst = qh.data() + (size_t)q * dim;
    if (elem == DK_ELEM_U8 || elem == DK_ELEM_I8) std::memcpy(dst, src, dim);
    else
      for (uint32_t i = 0; i < dim; ++i) dst[i] = elem_value(elem, src, i);
  }
  dk::DeviceGuard guard(ix->device);
  SearchParams P{};
  dk::base_params(ix, DK_STRATEGY_FULL_PRECISION, k, l, beam, P);
  P.nq = nq;
  P.qstride = dim;
  P.hash_limit = 0xFFFFFFFFu;  // the bitmap never fills
  P.raw = ix->raw;
  P.raw_stride = ix->raw_stride;
  P.readable = ix->readable;
  P.smem_bytes = dk::plan_query_smem(P, false, false);
  int max_optin = 0, sms = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);
  if (P.smem_bytes > (uint32_t)max_optin) return fail(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory (L too large)");
  // Persistent grid: every resident CTA (occupancy) owns a bitmap, within 512 MiB of bitmaps.
  const uint32_t words = (ix->n + ix->f + 31u) / 32u;
  const uint64_t per = (uint64_t)words * 4u;
  int occ = 0;
  cudaError_t eo = inmem_dispatch(ix, P, TranslateOut{}, 0, nullptr, &occ);
  if (eo != cudaSuccess) return fail(DK_ERR_CUDA, std::string("inmem occupancy: ") + cudaGetErrorString(eo));
  uint32_t grid = std::min<uint32_t>(nq, (uint32_t)std::max(1, occ) * (uint32_t)std::max(1, sms));
  if (per * grid > (512ull << 20)) grid = (uint32_t)std::max<uint64_t>(1, (512ull << 20) / per);
  const size_t qbytes = qh.size() * 4, obytes = (size_t)nq * k;
  const size_t o_ids = (qbytes + 255) / 256 * 256;
  const size_t o_d = o_ids + (obytes * 8 + 255) / 256 * 256;
  const size_t o_st = o_d + (obytes * 4 + 255) / 256 * 256;
  const size_t o_bm = o_st + ((size_t)nq * sizeof(dk_search_stats) + 255) / 256 * 256;
  const size_t total = o_bm + per * grid;
  cudaStream_t s = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  unsigned char* buf = nullptr;
  e = cudaMallocFromPoolAsync(reinterpret_cast<void**>(&buf), total, ix->pool, s);
  if (e != cudaSuccess) {
    cudaStreamDestroy(s);
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("inmem search buffers: ") + cudaGetErrorString(e));
  }
  e = cudaMemcpyAsync(buf, qh.data(), qbytes, cudaMemcpyHostToDevice, s);
  P.queries = reinterpret_cast<const float*>(buf);
  P.out_dists = reinterpret_cast<float*>(buf + o_d);
  P.stats = reinterpret_cast<dk_search_stats*>(buf + o_st);
  P.bitmap = reinterpret_cast<uint32_t*>(buf + o_bm);
  P.bitmap_words = words;
  const TranslateOut T{ix->ext, reinterpret_cast<uint64_t*>(buf + o_ids)};
  if (e == cudaSuccess) e = inmem_dispatch(ix, P, T, grid, s, nullptr);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ids, buf + o_ids, obytes * 8, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dists, buf + o_d, obytes * 4, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && stats)
    e = cudaMemcpyAsync(stats, buf + o_st, (size_t)nq * sizeof(dk_search_stats), cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  const cudaError_t es = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess) return fail(DK_ERR_CUDA, std::string("inmem search: ") + cudaGetErrorString(e));
  if (es != cudaSuccess) return fail(DK_ERR_CUDA, std::string("inmem search: ") + cudaGetErrorString(es));
  return DK_OK;
}
