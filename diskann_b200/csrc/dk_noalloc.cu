// dk_search_device_noalloc: the batched search of dk_search_device for callers that cannot
// allocate device memory while they search.  Every piece of scratch the search needs (the
// warp kernel's work counter and per-warp visited tables, the spill pass's bitmaps) is carved
// from one fixed array of DK_NOALLOC_SCRATCH_BYTES declared in this file, which the library
// holds on every GPU that loads it until the process exits.  No counterpart in the reference.
//
// Set-up: the first call on a device, made with that device current, looks the array's device
// address up with cudaGetSymbolAddress and keeps it for later calls.  With CUDA's lazy module
// loading the array's memory is committed when that look-up loads the module, so the set-up
// call (nq = 0 is enough) belongs before the caller's allocator reserves the GPU's memory; a
// set-up that finds no room fails with DK_ERR_CUDA.  The array is shared by every call on a
// device and keeps the last call's contents; each call clears the one word that must start at
// zero (the work counter), and the kernels clear their own visited tables and bitmaps.  Calls
// whose work overlaps on the GPU race on the array.  The visited tables are sized from the
// index's visited-size estimate, which only dk_search_device updates; this entry point reads it.
// The spill pass runs at most one CTA per SM here, with at most half of the room one CTA's
// tables leave (dk_search_device allows up to eight per SM), so batches in which many queries
// spill finish more slowly through this entry point.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "dk_kernels.cuh"

static __device__ __align__(256) unsigned char g_noalloc_scratch[DK_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

inline uint64_t align_up64(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

uint32_t env_u32(const char* name, uint32_t dflt) {
  const char* v = getenv(name);
  if (!v || !*v) return dflt;
  return (uint32_t)strtoul(v, nullptr, 10);
}

uint32_t log2_at_least(double x, uint32_t lo, uint32_t hi) {
  uint32_t l = lo;
  while (l < hi && (double)(1u << l) < x) ++l;
  return l;
}

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

// Device address of the scratch array on the current device `dev` (looked up once).
int32_t scratch_of(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(DK_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(DK_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_ptr[dev];
  return DK_OK;
}

int32_t too_big_smem() {
  return fail(DK_ERR_UNSUPPORTED, "search state does not fit in shared memory (L or PQ too large)");
}

int32_t too_big_scratch(uint64_t need) {
  return fail(DK_ERR_UNSUPPORTED,
              "dk_search_device_noalloc needs at least " + std::to_string(need) +
                  " bytes of scratch for this index and L; its fixed array holds " +
                  std::to_string((uint64_t)DK_NOALLOC_SCRATCH_BYTES) +
                  " (dk_search_device allocates what it needs)");
}

}  // namespace

extern "C" int32_t dk_search_device_noalloc(dk_index* ix, int32_t strategy, const float* queries,
                                            uint64_t query_stride, uint32_t nq, uint32_t k,
                                            uint32_t l, uint32_t beam_width, uint32_t* ids,
                                            float* dists, dk_search_stats* stats, void* stream_) {
  const int32_t v = dk_check_search_args(ix, strategy, k, l, beam_width, query_stride);
  if (v != DK_OK) return v;
  if (nq && (!queries || !ids || !dists || !stats))
    return fail(DK_ERR_INVALID_ARGUMENT, "queries, ids, dists and stats are required");
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != ix->device) cudaSetDevice(ix->device);
  struct Restore {
    int prev, dev;
    ~Restore() {
      if (prev >= 0 && prev != dev) cudaSetDevice(prev);
    }
  } restore{prev, ix->device};
  unsigned char* scratch = nullptr;
  int32_t rc = scratch_of(ix->device, &scratch);
  if (rc != DK_OK || nq == 0) return rc;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_);

  const int mode = mode_of_strategy(strategy);
  const bool pq = mode == kModePQ;
  SearchParams P{};
  dk::base_params(ix, strategy, k, l, beam_width, P);
  P.queries = queries;
  P.qstride = query_stride;
  P.nq = nq;
  P.out_ids = ids;
  P.out_dists = dists;
  P.stats = stats;
  // The visited tables are sized from the estimate that dk_search_device keeps on this index;
  // this entry point only reads it (it records nothing into, and resets nothing of, the
  // index's estimate words, which a dk_search_device on another stream may be using).
  P.hint = nullptr;
  double est = 0, est_mean = 0;
  dk::visited_estimates(ix, P, est, est_mean, /*absorb=*/false);
  int max_optin = 0, sms = 0;
  cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ix->device);

  const char* kenv = getenv("DK_KERNEL");
  bool warp = beam_width <= 4;
  if (kenv && !strcmp(kenv, "warp")) warp = true;
  if (kenv && !strcmp(kenv, "cta")) warp = false;

  // Scratch layout: work counter (256 B) | per-warp visited tables | spill bitmaps.  The spill
  // pass needs one bitmap of N+F bits per CTA; it keeps up to one CTA per SM, fewer when the
  // array is short, and the warp kernel runs as many warps as the tables left room for.
  const uint64_t cap_bytes = DK_NOALLOC_SCRATCH_BYTES;
  const uint32_t words = (ix->n + ix->f + 31u) / 32u;
  const uint64_t per_bitmap = align_up64((uint64_t)words * 4u, 256);
  if (256 + per_bitmap > cap_bytes) return too_big_scratch(256 + per_bitmap);
  uint32_t spill_ctas = std::min<uint32_t>(nq, (uint32_t)std::max(1, sms));
  dk::LaunchPlan L{};
  L.score_u = env_u32("DK_SCORE_U", mode == kModeFP32 ? 4u : 2u);
  uint64_t off_bitmap = 256;
  if (warp) {
    L.kind = dk::KernelKind::kWarp;
    rc = dk::plan_warp(ix, P, L, mode, est, est_mean, nq, stream);
    if (rc != DK_OK) return rc;
    const uint64_t per_cta = (uint64_t)L.warps_per_cta * (4ull << P.gtable_log2);
    const uint64_t min_need = 256 + per_cta + per_bitmap;
    if (min_need > cap_bytes) return too_big_scratch(min_need);
    // Up to half of what one CTA's tables leave goes to spill bitmaps, the rest to tables.
    const uint64_t room = cap_bytes - 256 - per_cta;
    spill_ctas = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(spill_ctas, room / 2 / per_bitmap));
    const uint64_t tables = cap_bytes - 256 - (uint64_t)spill_ctas * per_bitmap;
    L.grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(L.grid, tables / per_cta));
    off_bitmap = align_up64(256 + (uint64_t)L.grid * per_cta, 256);
  } else {
    L.kind = dk::KernelKind::kCta;
    uint32_t log2h = log2_at_least(est / 0.75, 9, 16);
    log2h = env_u32("DK_HASH_LOG2", log2h);
    P.hash_log2 = std::min<uint32_t>(std::max<uint32_t>(log2h, 6), 20);
    while (true) {
      P.hash_limit = (uint32_t)((1u << P.hash_log2) * 0.75);
      P.smem_bytes = dk::plan_query_smem(P, pq, true);
      if (P.smem_bytes <= (uint32_t)max_optin) break;
      if (P.hash_log2 <= 6) return too_big_smem();
      --P.hash_log2;
    }
    spill_ctas = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(spill_ctas, (cap_bytes - 256) / per_bitmap));
  }
  SearchParams P2 = P;
  P2.single_queue = 0;  // the spill pass (CTA kernel) merges into its second queue buffer
  P2.hash_limit = 0xFFFFFFFFu;  // the bitmap never fills
  P2.smem_bytes = dk::plan_query_smem(P2, pq, false);
  if (P2.smem_bytes > (uint32_t)max_optin) return too_big_smem();

  cudaError_t e = cudaMemsetAsync(scratch, 0, 256, stream);  // the work counter starts at 0
  P.work_counter = reinterpret_cast<uint32_t*>(scratch);
  P.spill_count = reinterpret_cast<uint32_t*>(scratch) + 1;  // zeroed with the counter
  P.gtable = reinterpret_cast<uint32_t*>(scratch + 256);
  P2.bitmap = reinterpret_cast<uint32_t*>(scratch + off_bitmap);
  P2.spill_count = P.spill_count;
  P2.bitmap_words = words;
  L.p1 = P;
  L.p2 = P2;
  L.spill_ctas = spill_ctas;
  if (e == cudaSuccess) e = dk::dispatch(ix->metric, L, mode, stream);
  if (e != cudaSuccess)
    return fail(DK_ERR_CUDA, std::string("search launch: ") + cudaGetErrorString(e));
  return DK_OK;
}
