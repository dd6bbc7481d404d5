// Internal definitions shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "diskann_b200.h"

// Device-resident in-memory index.  HBM layout:
//  * vectors  : (N+F) rows x vstride floats, vstride = round_up(D, 4), rows 16-B aligned and
//               zero padded, so a row is read with 16-byte loads;
//  * adjacency: (N+F) rows x astride u32, row = [degree, id_0 .. id_{max_degree-1}, pad],
//               astride = round_up(1 + max_degree, 4): one hop reads one contiguous row;
//  * pq codes : (N+F) rows x cstride bytes, cstride = round_up(M, 16);
//  * pq pivots: 256 x D floats (row-major, the FixedChunkPQTable layout); offsets: M+1 u32.
struct dk_index {
  int device = 0;
  uint32_t n = 0, f = 0, dim = 0, max_degree = 0, pq_chunks = 0;
  int32_t metric = 0;
  uint32_t vstride = 0, astride = 0, cstride = 0;
  float* vectors = nullptr;
  uint32_t* adj = nullptr;
  uint8_t* codes = nullptr;
  float* pivots = nullptr;
  float* pivots_cm = nullptr;  // chunk-major copy: chunk m, centre c -> len_m floats
  uint32_t* offsets = nullptr;
  // Low-precision copies: rows of lp_stride elements (a multiple of 16, zero padded), each
  // with (scale, squared norm of the de-quantised row) in the matching *_meta array.
  uint16_t* vec_bf16 = nullptr;   // BF16 bit patterns (scale 1)
  uint8_t* vec_fp8 = nullptr;     // FP8-E4M3, value = fp8 * scale
  float2* bf16_meta = nullptr;
  float2* fp8_meta = nullptr;
  uint32_t lp_stride = 0;
  uint64_t bytes = 0;
  // Visited-set sizing hint, in units of cmps * 256 / (L + F).  Kernels update three device
  // words (largest value, sum, count) with L2 atomics; each launch sequence ends with an
  // asynchronous copy of them to pinned host memory (`hint_stage`) and a reset, and the next
  // launch plans from the staged values.  Only performance depends on the hint: an
  // undersized visited table spills, exactly.
  uint32_t* hint_dev = nullptr;
  uint32_t* hint_stage = nullptr;
  uint32_t hint_max = 0;   // last staged largest value
  uint32_t hint_mean = 0;  // last staged mean
  // Stream-ordered scratch of every search on this index comes from this pool, which keeps
  // freed memory reserved (release threshold: unlimited), so a repeated search reuses it
  // instead of mapping new memory each call.
  cudaMemPool_t pool = nullptr;
  // diskann-inmem store (dk_inmem.cu): element type, rows of that type (raw_stride bytes,
  // zero padded; FP32 indexes use `vectors`), readable-slot bits from the rows' tags, and the
  // external id of each slot (DK_NO_EXTERNAL_ID: none).  Unset for other indexes.
  int32_t elem = -1;
  unsigned char* raw = nullptr;
  uint32_t raw_stride = 0;
  uint32_t* readable = nullptr;
  uint64_t* ext = nullptr;
};

// Per-launch parameters of the beam-search kernels.
struct SearchParams {
  const float* vectors;
  const uint32_t* adj;
  const uint8_t* codes;
  const float* pivots;
  const float* pivots_cm;
  const uint32_t* offsets;
  const uint16_t* vec_bf16;
  const uint8_t* vec_fp8;
  const float2* bf16_meta;
  const float2* fp8_meta;
  uint32_t lp_stride;
  uint32_t n, f, dim, vstride, astride, max_degree, cstride, pq_chunks;
  const float* queries;
  uint64_t qstride;
  uint32_t nq;
  uint32_t k, l, cap, beam;
  int32_t strategy;
  uint32_t* out_ids;
  float* out_dists;
  dk_search_stats* stats;
  // Visited set: shared-memory hash (first pass) or global bitmap slice per CTA (spill pass).
  uint32_t hash_log2;
  uint32_t hash_slots;  // warp kernel: shared-level slots (any multiple of 32)
  uint32_t hash_limit;  // inserts allowed before the hash counts as full
  uint32_t* bitmap;
  uint32_t bitmap_words;
  // Warp kernel: persistent work counter and each warp's global overflow hash (second level
  // of the visited set, used once the shared hash holds `hash_limit` ids).
  uint32_t* work_counter;
  uint32_t* spill_count;  // queries the first pass abandoned (the spill pass exits at 0); may be null
  uint32_t* gtable;
  uint32_t gtable_log2;
  uint32_t gtable_limit;
  // Warp kernel: issue a whole adjacency row's global-level probes together (one round trip
  // per row; the default) instead of one round trip per 32-id round.
  uint32_t row_probes;
  // Shared-memory carve-up: byte offsets from the CTA's dynamic shared memory (CTA kernel)
  // or from the warp's slice of it (warp kernel, slices of `warp_smem` bytes).
  uint32_t off_query, off_table, off_qd0, off_qi0, off_qd1, off_qi1;
  uint32_t off_cand_id, off_cand_d, off_new_d, off_new_id, off_hash, off_misc;
  // Warp kernel, strategies without a rerank: the queue is merged in place and its second
  // buffer (the rerank's scratch) is not needed, so both queue buffers alias one region.
  uint32_t single_queue;
  uint32_t smem_bytes;
  uint32_t warp_smem;
  uint32_t list_cap;  // capacity of the candidate / rerank lists
  uint32_t* hint;     // device words of the visited-size hint (may be null)
  // Graph construction: the expanded nodes of each query in order, with their distances
  // (the reference's visited search record), up to rec_cap per query; null when unused.
  uint32_t* rec_ids;
  float* rec_d;
  uint32_t rec_cap;
  // Serving launches: per-request (k, L) pairs; outputs keep a stride of `k` (= max_k).
  // Null for batch launches, where every query uses `k` and `l`.
  const uint32_t* req_kl;
  // diskann-inmem indexes: element rows of raw_stride bytes (FP16 / u8 / i8 modes), and the
  // slots whose tag is readable (one bit per id); null elsewhere.
  const unsigned char* raw;
  uint32_t raw_stride;
  const uint32_t* readable;
  // FullPrecision output without FilterStartPoints (range search's first round).
  uint32_t keep_start;
  // Serving: after a query's results are written, done_flags[qid] = done_value (mapped host
  // memory, written after a system-scope fence), so the host can collect each request on its
  // own; null elsewhere.
  uint32_t* done_flags;
  uint32_t done_value;
};

constexpr uint32_t kFlagSpilled = 1u;

// How candidates are scored during traversal.
constexpr int kModeFP32 = 0;
constexpr int kModePQ = 1;
constexpr int kModeBF16 = 2;
constexpr int kModeFP8 = 3;
// diskann-inmem element types (dk_inmem.cu): FP16 rows, and u8 / i8 rows scored in integers.
constexpr int kModeF16 = 4;
constexpr int kModeU8 = 5;
constexpr int kModeI8 = 6;

inline int mode_of_strategy(int32_t strategy) {
  switch (strategy) {
    case DK_STRATEGY_HYBRID:
    case DK_STRATEGY_QUANTIZED: return kModePQ;
    case DK_STRATEGY_BF16: return kModeBF16;
    case DK_STRATEGY_FP8: return kModeFP8;
    default: return kModeFP32;
  }
}

// Strategies whose post-processing re-ranks the queue with exact FP32 distances.
__host__ __device__ inline bool strategy_reranks(int32_t strategy) {
  return strategy == DK_STRATEGY_HYBRID || strategy == DK_STRATEGY_BF16 ||
         strategy == DK_STRATEGY_FP8;
}

// Thread-local error reporting for the C ABI.
void dk_set_error(int32_t status, const std::string& msg);

namespace dk {
// Makes `dev` current for the scope and restores the caller's current device on exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int now = -1;
    cudaGetDevice(&now);
    if (prev >= 0 && now != prev) cudaSetDevice(prev);
  }
};
}  // namespace dk

// Argument checks shared by every search entry point (sets the thread's error).
int32_t dk_check_search_args(const dk_index* ix, int32_t strategy, uint32_t k, uint32_t l,
                             uint32_t beam, uint64_t qstride);

// Derive the low-precision copies requested by `flags` from the index's FP32 rows.
cudaError_t dk_build_low_precision(dk_index* ix, uint32_t flags);

// Optional output of dk_launch_search: each query's expanded nodes in order with their queue
// distances (rec_cap per query; a query that expanded more than rec_cap nodes records the
// first rec_cap, and its stats.hops tells).
struct SearchRecord {
  uint32_t* ids;
  float* dists;
  uint32_t cap;
};

// Launch the search (first pass + spill pass) on `stream`.  Parameters are validated by
// the caller.  `keep_start`: the FullPrecision output keeps start points (range search's
// first round reads the queue as it stands).
int32_t dk_launch_search(dk_index* ix, int32_t strategy, const float* queries,
                         uint64_t qstride, uint32_t nq, uint32_t k, uint32_t l, uint32_t beam,
                         uint32_t* ids, float* dists, dk_search_stats* stats,
                         cudaStream_t stream, const SearchRecord* record = nullptr,
                         bool keep_start = false);
