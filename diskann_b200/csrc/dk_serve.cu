// Serving: continuous admission of single requests with per-request k and L.
//
// The host keeps a table of outstanding requests (one entry per ticket modulo queue_depth)
// and a few launch contexts, each with its own stream, device buffers (queries, per-request
// k/L, results, a work counter and one global visited table per warp) and pinned staging.
// Requests queue on submit and go out as soon as a context is free: one launch carries every
// request queued at that moment, and launches on different contexts overlap on the device.
// Each request completes on its own: the kernel writes its results straight into the
// context's mapped pinned memory and then, after a system-scope fence, the request's done
// flag, which the host polls; a short request does not wait for a long one in its launch.
// The kernel is the batch path's warp-per-query kernel reading each request's own k and L,
// so a request's results do not depend on what else is in flight.  No device code waits on
// the host: a launch is an ordinary finite kernel, and the host learns of its end through
// the context's event.
//
// The reference has no counterpart: a search there is one async call per query
// (diskann/src/graph/index.rs:2034-2070) scheduled by the caller's runtime.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include "dk_kernels.cuh"

namespace {

inline uint64_t round_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

enum : uint8_t { kFree = 0, kPending = 1, kInFlight = 2, kDone = 3, kCancelled = 4 };

// One launch context.  Device buffer layout (each part 256-B aligned):
// counter | kl[cap][2] | queries[cap][dim] | ids[cap][max_k] | dists[cap][max_k] |
// stats[cap] | visited tables[slots][table].  Mapped pinned memory mirrors kl .. stats (the
// kernel writes results there) and holds the per-request done flags after them.
struct Context {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  unsigned char* dev = nullptr;
  unsigned char* host = nullptr;
  unsigned char* host_dev = nullptr;  // the device's pointer to `host`
  std::vector<uint64_t> tickets;
  uint32_t seq = 0;  // this context's launch count: the done-flag value of its current launch
  bool busy = false;
};

}  // namespace

struct dk_server {
  dk_index* ix = nullptr;
  dk_server_config cfg{};
  int mode = 0;
  std::mutex mu;
  dk::LaunchPlan plan{};  // grid = the most warps one launch uses
  std::vector<Context> ctx;
  // Offsets inside a context's buffers.
  uint64_t off_kl = 0, off_q = 0, off_ids = 0, off_d = 0, off_st = 0, off_gt = 0, dev_bytes = 0;
  uint64_t off_flag = 0;  // host buffers: done flags
  uint64_t host_bytes = 0;
  // Outstanding requests, indexed by ticket % queue_depth.
  std::vector<uint8_t> state;
  std::vector<uint8_t> cancel;       // cancelled while in flight: its results are dropped
  std::vector<uint32_t> req_k, req_l;
  std::vector<uint64_t> req_bytes;   // device memory reserved for the request's beam state
  // Admission by device memory: every outstanding request reserves the bytes its beam state
  // needs at its own L (beam_bytes); a request is admitted while the reservations fit
  // `memory_bytes` (the device memory held for beam state).
  uint64_t memory_bytes = 0, reserved_bytes = 0;
  double visited_per_entry = 0;  // visited ids per queue entry (the index's learned ratio)
  std::vector<float> queries;       // queue_depth x dim
  std::vector<uint32_t> res_ids;    // queue_depth x max_k
  std::vector<float> res_dists;     // queue_depth x max_k
  std::vector<dk_search_stats> res_stats;
  std::deque<uint64_t> pending;
  uint64_t next_ticket = 0;  // tickets issued
  uint64_t head = 0;         // lowest ticket not yet collected
  // Exact re-run of a request whose visited set outgrew its warp's tables.
  cudaStream_t side = nullptr;
  unsigned char* rerun = nullptr;
  uint64_t device_bytes = 0;
  uint64_t launches = 0;
};

namespace {

int32_t fail(int32_t status, const std::string& msg) {
  dk_set_error(status, msg);
  return status;
}

int32_t cuda_fail(cudaError_t e, const char* what) {
  return fail(DK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void release(dk_server* s) {
  for (Context& c : s->ctx) {
    if (c.stream) cudaStreamSynchronize(c.stream);
    if (c.done) cudaEventDestroy(c.done);
    if (c.stream) cudaStreamDestroy(c.stream);
    if (c.dev) cudaFree(c.dev);
    if (c.host) cudaFreeHost(c.host);
  }
  if (s->side) {
    cudaStreamSynchronize(s->side);
    cudaStreamDestroy(s->side);
  }
  if (s->rerun) cudaFree(s->rerun);
  delete s;
}

constexpr uint64_t kRetired = ~0ull;  // a context's ticket entry already collected

// Collect finished requests into the request table: each request as soon as its done flag
// is up, and a context's remaining ones when its launch has ended.  A collected request's
// entry in its context is retired at once: its table slot may be freed and handed to a newer
// request (ticket + queue_depth) on another context while this launch still runs, and that
// slot must not be matched against this launch's flags again.
int32_t reap(dk_server* s) {
  const uint32_t max_k = s->cfg.max_k, depth = s->cfg.queue_depth;
  for (Context& c : s->ctx) {
    if (!c.busy) continue;
    const cudaError_t q = cudaEventQuery(c.done);
    if (q != cudaErrorNotReady && q != cudaSuccess) return cuda_fail(q, "serving launch");
    const bool ended = q == cudaSuccess;
    const volatile uint32_t* flag = reinterpret_cast<const volatile uint32_t*>(c.host + s->off_flag);
    const uint32_t* ids = reinterpret_cast<const uint32_t*>(c.host + s->off_ids);
    const float* d = reinterpret_cast<const float*>(c.host + s->off_d);
    const dk_search_stats* st = reinterpret_cast<const dk_search_stats*>(c.host + s->off_st);
    for (size_t i = 0; i < c.tickets.size(); ++i) {
      if (c.tickets[i] == kRetired) continue;
      const uint32_t r = (uint32_t)(c.tickets[i] % depth);
      if (!ended && flag[i] != c.seq) continue;
      std::atomic_thread_fence(std::memory_order_acquire);
      c.tickets[i] = kRetired;
      if (s->cancel[r]) {  // cancelled while in flight: its results are not kept
        s->state[r] = kCancelled;
        continue;
      }
      const uint32_t k = s->req_k[r];
      memcpy(&s->res_ids[(size_t)r * max_k], ids + i * max_k, 4ull * k);
      memcpy(&s->res_dists[(size_t)r * max_k], d + i * max_k, 4ull * k);
      s->res_stats[r] = st[i];
      s->state[r] = kDone;
    }
    if (ended) {
      c.tickets.clear();
      c.busy = false;
    }
  }
  return DK_OK;
}

// Launch every queued request on a free context (one launch per free context while requests
// remain queued; a launch takes up to queue_depth requests).
int32_t launch_pending(dk_server* s) {
  const uint32_t dim = s->ix->dim, max_k = s->cfg.max_k, depth = s->cfg.queue_depth;
  for (Context& c : s->ctx) {
    if (s->pending.empty()) break;
    if (c.busy) continue;
    uint32_t* kl = reinterpret_cast<uint32_t*>(c.host + s->off_kl);
    float* q = reinterpret_cast<float*>(c.host + s->off_q);
    uint32_t b = 0;
    while (!s->pending.empty() && b < depth) {
      const uint64_t t = s->pending.front();
      s->pending.pop_front();
      const uint32_t r = (uint32_t)(t % depth);
      kl[2 * b] = s->req_k[r];
      kl[2 * b + 1] = s->req_l[r];
      memcpy(q + (size_t)b * dim, &s->queries[(size_t)r * dim], 4ull * dim);
      s->state[r] = kInFlight;
      c.tickets.push_back(t);
      ++b;
    }
    dk::LaunchPlan L = s->plan;
    L.p1.nq = b;
    L.p1.req_kl = reinterpret_cast<const uint32_t*>(c.dev + s->off_kl);
    L.p1.queries = reinterpret_cast<const float*>(c.dev + s->off_q);
    L.p1.qstride = dim;
    ++c.seq;
    if (c.seq == 0) c.seq = 1;  // flags start at 0: never a launch's value
    L.p1.out_ids = reinterpret_cast<uint32_t*>(c.host_dev + s->off_ids);
    L.p1.out_dists = reinterpret_cast<float*>(c.host_dev + s->off_d);
    L.p1.stats = reinterpret_cast<dk_search_stats*>(c.host_dev + s->off_st);
    L.p1.done_flags = reinterpret_cast<uint32_t*>(c.host_dev + s->off_flag);
    L.p1.done_value = c.seq;
    L.p1.work_counter = reinterpret_cast<uint32_t*>(c.dev);
    L.p1.gtable = reinterpret_cast<uint32_t*>(c.dev + s->off_gt);
    L.grid = std::min<uint32_t>(L.grid, (b + L.warps_per_cta - 1) / L.warps_per_cta);
    cudaError_t e = cudaMemcpyAsync(c.dev + s->off_kl, kl, 8ull * b, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(c.dev + s->off_q, q, 4ull * dim * b, cudaMemcpyHostToDevice, c.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c.dev, 0, 4, c.stream);
    if (e == cudaSuccess) e = dk::dispatch(s->ix->metric, L, s->mode, c.stream);
    if (e == cudaSuccess) e = cudaEventRecord(c.done, c.stream);
    if (e != cudaSuccess) return cuda_fail(e, "serving launch");
    c.busy = true;
    ++s->launches;
  }
  return DK_OK;
}

int32_t progress(dk_server* s) {
  const int32_t rc = reap(s);
  if (rc != DK_OK) return rc;
  return launch_pending(s);
}

// Device memory a request's beam state needs at its L: its double-buffered queue of L + F
// (distance, id) entries and its share of a visited table holding the expected visited set
// (the index's learned visited-per-entry ratio times L + F, plus one hop's candidates) at
// load 3/4.
uint64_t beam_bytes(const dk_server* s, uint32_t l) {
  const uint64_t cap = (uint64_t)l + s->ix->f;
  const double visited = s->visited_per_entry * (double)cap +
                         (double)s->cfg.beam_width * s->ix->max_degree + s->ix->f;
  return 16ull * cap + 4ull * (uint64_t)(visited / 0.75 + 1.0);
}

// Admission of one more request needing `need` bytes: queue depth, then device memory.
int32_t admit(const dk_server* s, uint64_t need) {
  if (s->next_ticket - s->head >= s->cfg.queue_depth)
    return fail(DK_ERR_ADMISSION, "queue_depth requests are outstanding");
  if (s->reserved_bytes + need > s->memory_bytes)
    return fail(DK_ERR_ADMISSION,
                "the request's beam state (" + std::to_string(need) + " bytes) does not fit the " +
                    "server's device memory for beam state (" + std::to_string(s->reserved_bytes) +
                    " of " + std::to_string(s->memory_bytes) + " bytes reserved)");
  return DK_OK;
}

// Free a collected (or cancelled) request's table slot and its memory reservation.
void retire(dk_server* s, uint32_t r) {
  s->state[r] = kFree;
  s->cancel[r] = 0;
  s->reserved_bytes -= s->req_bytes[r];
  s->req_bytes[r] = 0;
  const uint32_t depth = s->cfg.queue_depth;
  while (s->head < s->next_ticket && s->state[s->head % depth] == kFree) ++s->head;
}

}  // namespace

extern "C" int32_t dk_server_create(dk_index* ix, const dk_server_config* cfg, dk_server** out) {
  if (!ix || !cfg || !out) return fail(DK_ERR_INVALID_ARGUMENT, "index, config and out are required");
  *out = nullptr;
  int32_t v = dk_check_search_args(ix, cfg->strategy, cfg->max_k, cfg->max_l, cfg->beam_width,
                                   ix->dim);
  if (v != DK_OK) return v;
  if (cfg->queue_depth == 0) return fail(DK_ERR_INVALID_ARGUMENT, "queue_depth must be positive");
  if (cfg->queue_depth > (1u << 20)) return fail(DK_ERR_INVALID_ARGUMENT, "queue_depth above 2^20");
  if (cfg->beam_width > 4)
    return fail(DK_ERR_UNSUPPORTED, "serving runs beam_width <= 4 (one warp per request)");
  if (cfg->streams > 64) return fail(DK_ERR_INVALID_ARGUMENT, "streams above 64");
  dk::DeviceGuard guard(ix->device);
  dk_server* s = new dk_server();
  s->ix = ix;
  s->cfg = *cfg;
  if (s->cfg.streams == 0) s->cfg.streams = 16;
  s->mode = mode_of_strategy(cfg->strategy);
  const uint32_t dim = ix->dim, max_k = cfg->max_k, depth = cfg->queue_depth;

  SearchParams P{};
  dk::base_params(ix, cfg->strategy, max_k, cfg->max_l, cfg->beam_width, P);
  P.hint = nullptr;
  double est = 0, est_mean = 0;
  dk::visited_estimates(ix, P, est, est_mean);
  s->plan.kind = dk::KernelKind::kWarp;
  s->plan.score_u = s->mode == kModeFP32 ? 4u : 2u;
  s->plan.skip_spill = true;
  const uint64_t max_warps = cfg->max_slots ? cfg->max_slots : (1ull << 32);
  v = dk::plan_warp(ix, P, s->plan, s->mode, est, est_mean, max_warps, nullptr);
  if (v != DK_OK) {
    delete s;
    return v;
  }
  s->plan.p1 = P;

  // Buffers per context; the visited tables take what is left of half the free memory.
  s->off_kl = 256;
  s->off_q = round_up(s->off_kl + 8ull * depth, 256);
  s->off_ids = round_up(s->off_q + 4ull * dim * depth, 256);
  s->off_d = round_up(s->off_ids + 4ull * max_k * depth, 256);
  s->off_st = round_up(s->off_d + 4ull * max_k * depth, 256);
  s->off_gt = round_up(s->off_st + sizeof(dk_search_stats) * depth, 256);
  s->off_flag = s->off_gt;
  s->host_bytes = round_up(s->off_flag + 4ull * depth, 256);
  const uint64_t table_bytes = 4ull << P.gtable_log2;
  const uint64_t per_cta_tables = table_bytes * s->plan.warps_per_cta;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  const uint64_t budget = free_b / 2;
  uint64_t grid = s->plan.grid;
  while (grid > 0 && s->cfg.streams * (s->off_gt + grid * per_cta_tables) > budget) {
    if (s->cfg.streams > 1) --s->cfg.streams;
    else grid /= 2;
  }
  if (grid == 0) {
    delete s;
    return fail(DK_ERR_ADMISSION, "not enough free device memory for one serving context");
  }
  s->plan.grid = (uint32_t)grid;
  s->dev_bytes = s->off_gt + grid * per_cta_tables;

  s->ctx.resize(s->cfg.streams);
  cudaError_t e = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking);
  for (Context& c : s->ctx) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&c.dev), s->dev_bytes);
    if (e == cudaSuccess)
      e = cudaHostAlloc(reinterpret_cast<void**>(&c.host), s->host_bytes, cudaHostAllocMapped);
    if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&c.host_dev), c.host, 0);
    if (e == cudaSuccess) memset(c.host, 0, s->host_bytes);
  }
  const uint64_t rerun_bytes = round_up(4ull * dim, 256) + 2 * round_up(4ull * max_k, 256) +
                               sizeof(dk_search_stats);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s->rerun), rerun_bytes);
  if (e != cudaSuccess) {
    release(s);
    return fail(DK_ERR_OUT_OF_MEMORY, std::string("serving buffers: ") + cudaGetErrorString(e));
  }
  s->device_bytes = s->cfg.streams * s->dev_bytes + rerun_bytes;
  // Beam-state memory: the visited tables of every context's warps (the queues live in
  // shared memory beside them), unless the caller sets a smaller or larger budget.
  s->visited_per_entry = std::max(0.0, (est_mean - (double)cfg->beam_width * ix->max_degree - ix->f) /
                                           (double)P.cap);
  s->memory_bytes = cfg->memory_bytes ? cfg->memory_bytes
                                      : (uint64_t)s->cfg.streams * grid * per_cta_tables;
  s->state.assign(depth, kFree);
  s->cancel.assign(depth, 0);
  s->req_bytes.assign(depth, 0);
  s->req_k.assign(depth, 0);
  s->req_l.assign(depth, 0);
  s->queries.assign((size_t)depth * dim, 0.0f);
  s->res_ids.assign((size_t)depth * max_k, 0u);
  s->res_dists.assign((size_t)depth * max_k, 0.0f);
  s->res_stats.assign(depth, dk_search_stats{});
  *out = s;
  return DK_OK;
}

extern "C" int32_t dk_server_submit(dk_server* s, const float* query, uint32_t k, uint32_t l,
                                    uint64_t* ticket) {
  if (!s || !query || !ticket) return fail(DK_ERR_INVALID_ARGUMENT, "server, query and ticket are required");
  const int32_t v = dk_knn_validate(k, l, s->cfg.beam_width);
  if (v != DK_OK) return v;
  if (k > s->cfg.max_k || l > s->cfg.max_l)
    return fail(DK_ERR_INVALID_ARGUMENT, "k or L above the server's max_k / max_l");
  std::lock_guard<std::mutex> lock(s->mu);
  const uint64_t need = beam_bytes(s, l);
  const int32_t a = admit(s, need);
  if (a != DK_OK) return a;
  const uint64_t t = s->next_ticket++;
  const uint32_t r = (uint32_t)(t % s->cfg.queue_depth);
  s->req_k[r] = k;
  s->req_l[r] = l;
  s->req_bytes[r] = need;
  s->reserved_bytes += need;
  memcpy(&s->queries[(size_t)r * s->ix->dim], query, 4ull * s->ix->dim);
  s->state[r] = kPending;
  s->pending.push_back(t);
  *ticket = t;
  dk::DeviceGuard guard(s->ix->device);
  return progress(s);
}

extern "C" int32_t dk_server_poll(dk_server* s, uint64_t ticket, uint32_t* ids, float* dists,
                                  dk_search_stats* stats) {
  if (!s || !ids || !dists) return fail(DK_ERR_INVALID_ARGUMENT, "server, ids and dists are required");
  std::lock_guard<std::mutex> lock(s->mu);
  const uint32_t depth = s->cfg.queue_depth, max_k = s->cfg.max_k;
  const uint32_t r = (uint32_t)(ticket % depth);
  if (ticket >= s->next_ticket || ticket < s->head || s->state[r] == kFree)
    return fail(DK_ERR_NOT_FOUND, "unknown or already collected ticket");
  dk::DeviceGuard guard(s->ix->device);
  if (s->state[r] != kDone && s->state[r] != kCancelled) {
    const int32_t rc = progress(s);
    if (rc != DK_OK) return rc;
    if (s->state[r] != kDone && s->state[r] != kCancelled) return DK_ERR_NOT_READY;
  }
  if (s->state[r] == kCancelled) {
    retire(s, r);
    return fail(DK_ERR_CANCELLED, "the request was cancelled");
  }
  const uint32_t k = s->req_k[r];
  dk_search_stats st = s->res_stats[r];
  if (st.flags & kFlagSpilled) {
    // The warp's visited tables were too small for this request: run it again through the
    // batch path, whose bitmap pass is exact for any visited-set size.
    const uint32_t dim = s->ix->dim;
    float* q = reinterpret_cast<float*>(s->rerun);
    uint32_t* rid = reinterpret_cast<uint32_t*>(s->rerun + round_up(4ull * dim, 256));
    float* rd = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(rid) + round_up(4ull * max_k, 256));
    dk_search_stats* rst = reinterpret_cast<dk_search_stats*>(reinterpret_cast<unsigned char*>(rd) + round_up(4ull * max_k, 256));
    cudaError_t e = cudaMemcpyAsync(q, &s->queries[(size_t)r * dim], 4ull * dim,
                                    cudaMemcpyHostToDevice, s->side);
    if (e != cudaSuccess) return cuda_fail(e, "re-run copy");
    const int32_t rc = dk_launch_search(s->ix, s->cfg.strategy, q, dim, 1, k, s->req_l[r],
                                        s->cfg.beam_width, rid, rd, rst, s->side);
    if (rc != DK_OK) return rc;
    e = cudaMemcpyAsync(ids, rid, 4ull * k, cudaMemcpyDeviceToHost, s->side);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dists, rd, 4ull * k, cudaMemcpyDeviceToHost, s->side);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&st, rst, sizeof(st), cudaMemcpyDeviceToHost, s->side);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->side);
    if (e != cudaSuccess) return cuda_fail(e, "re-run");
    st.flags |= kFlagSpilled;
  } else {
    memcpy(ids, &s->res_ids[(size_t)r * max_k], 4ull * k);
    memcpy(dists, &s->res_dists[(size_t)r * max_k], 4ull * k);
  }
  if (stats) *stats = st;
  retire(s, r);
  return DK_OK;
}

extern "C" int32_t dk_server_cancel(dk_server* s, uint64_t ticket) {
  if (!s) return fail(DK_ERR_INVALID_ARGUMENT, "server is required");
  std::lock_guard<std::mutex> lock(s->mu);
  const uint32_t r = (uint32_t)(ticket % s->cfg.queue_depth);
  if (ticket >= s->next_ticket || ticket < s->head || s->state[r] == kFree)
    return fail(DK_ERR_NOT_FOUND, "unknown or already collected ticket");
  switch (s->state[r]) {
    case kPending:  // not launched yet: it never reaches the device
      s->pending.erase(std::find(s->pending.begin(), s->pending.end(), ticket));
      s->state[r] = kCancelled;
      break;
    case kInFlight:  // its launch finishes; the results are dropped when it is reaped
      s->cancel[r] = 1;
      break;
    case kDone:
      s->state[r] = kCancelled;
      break;
    default:
      break;
  }
  return DK_OK;
}

extern "C" int32_t dk_server_replay(dk_server* s, const float* queries, uint64_t query_stride,
                                    uint32_t nq, const uint32_t* ks, const uint32_t* ls,
                                    const uint64_t* arrival_ns, uint32_t n, uint64_t* latency_ns,
                                    uint32_t* ids, float* dists) {
  if (!s || !queries || !ks || !ls || !arrival_ns || !latency_ns || (n && nq == 0))
    return fail(DK_ERR_INVALID_ARGUMENT, "server, queries, k, L, arrivals and latencies are required");
  if (query_stride < s->ix->dim) return fail(DK_ERR_DIMENSION_MISMATCH, "query stride below dim");
  for (uint32_t i = 0; i < n; ++i) {
    const int32_t v = dk_knn_validate(ks[i], ls[i], s->cfg.beam_width);
    if (v != DK_OK) return v;
    if (ks[i] > s->cfg.max_k || ls[i] > s->cfg.max_l)
      return fail(DK_ERR_INVALID_ARGUMENT, "k or L above the server's max_k / max_l");
    if (i && arrival_ns[i] < arrival_ns[i - 1])
      return fail(DK_ERR_INVALID_ARGUMENT, "arrival times must not decrease");
    if (beam_bytes(s, ls[i]) > s->memory_bytes)
      return fail(DK_ERR_ADMISSION, "a request's beam state exceeds the server's device memory for beam state");
  }
  const uint32_t max_k = s->cfg.max_k, depth = s->cfg.queue_depth, dim = s->ix->dim;
  std::vector<std::pair<uint64_t, uint32_t>> out;  // (ticket, request) in flight
  out.reserve(std::min<uint32_t>(n, depth));
  std::vector<uint64_t> keep;
  const auto t0 = std::chrono::steady_clock::now();
  auto now_ns = [&]() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now() - t0).count();
  };
  uint32_t next = 0, done = 0;
  dk::DeviceGuard guard(s->ix->device);
  while (done < n) {
    std::lock_guard<std::mutex> lock(s->mu);
    // Submit every request whose arrival time has come, while admission allows.
    const uint64_t now = now_ns();
    while (next < n && arrival_ns[next] <= now && s->next_ticket - s->head < depth &&
           s->reserved_bytes + beam_bytes(s, ls[next]) <= s->memory_bytes) {
      const uint64_t t = s->next_ticket++;
      const uint32_t r = (uint32_t)(t % depth);
      s->req_k[r] = ks[next];
      s->req_l[r] = ls[next];
      s->req_bytes[r] = beam_bytes(s, ls[next]);
      s->reserved_bytes += s->req_bytes[r];
      memcpy(&s->queries[(size_t)r * dim], queries + (size_t)(next % nq) * query_stride, 4ull * dim);
      s->state[r] = kPending;
      s->pending.push_back(t);
      out.emplace_back(t, next);
      ++next;
    }
    const int32_t rc = progress(s);
    if (rc != DK_OK) return rc;
    // Collect what is done, in any order.
    size_t w = 0;
    for (size_t j = 0; j < out.size(); ++j) {
      const uint64_t t = out[j].first;
      const uint32_t i = out[j].second, r = (uint32_t)(t % depth);
      if (s->state[r] == kCancelled) {  // cancelled by another thread: no results
        const uint64_t fin = now_ns();
        latency_ns[i] = fin > arrival_ns[i] ? fin - arrival_ns[i] : 0;
        retire(s, r);
        ++done;
        continue;
      }
      if (s->state[r] != kDone || (s->res_stats[r].flags & kFlagSpilled)) {
        if (s->state[r] == kDone) {
          // Spilled: collect through the exact re-run of dk_server_poll (lock released there).
          keep.push_back(t);
        }
        out[w++] = out[j];
        continue;
      }
      const uint64_t fin = now_ns();
      latency_ns[i] = fin > arrival_ns[i] ? fin - arrival_ns[i] : 0;
      if (ids) memcpy(ids + (size_t)i * max_k, &s->res_ids[(size_t)r * max_k], 4ull * ks[i]);
      if (dists) memcpy(dists + (size_t)i * max_k, &s->res_dists[(size_t)r * max_k], 4ull * ks[i]);
      retire(s, r);
      ++done;
    }
    out.resize(w);
    if (!keep.empty()) {
      // Rare: a request whose visited tables overflowed is re-run exactly by the batch path.
      std::vector<uint32_t> tid(max_k);
      std::vector<float> td(max_k);
      for (uint64_t t : keep) {
        size_t j = 0;
        while (out[j].first != t) ++j;
        const uint32_t i = out[j].second;
        s->mu.unlock();
        const int32_t prc = dk_server_poll(s, t, tid.data(), td.data(), nullptr);
        s->mu.lock();
        if (prc != DK_OK) return prc;
        const uint64_t fin = now_ns();
        latency_ns[i] = fin > arrival_ns[i] ? fin - arrival_ns[i] : 0;
        if (ids) memcpy(ids + (size_t)i * max_k, tid.data(), 4ull * ks[i]);
        if (dists) memcpy(dists + (size_t)i * max_k, td.data(), 4ull * ks[i]);
        out.erase(out.begin() + (long)j);
        ++done;
      }
      keep.clear();
    }
  }
  return DK_OK;
}

extern "C" int32_t dk_server_get_info(const dk_server* s, dk_server_info* info) {
  if (!s || !info) return fail(DK_ERR_INVALID_ARGUMENT, "server and info are required");
  info->slots = s->plan.grid * s->plan.warps_per_cta;
  info->queue_depth = s->cfg.queue_depth;
  info->streams = s->cfg.streams;
  info->pad = 0;
  info->device_bytes = s->device_bytes;
  info->launches = s->launches;
  info->memory_bytes = s->memory_bytes;
  info->reserved_bytes = s->reserved_bytes;
  return DK_OK;
}

extern "C" int32_t dk_server_destroy(dk_server* s) {
  if (!s) return DK_OK;
  dk::DeviceGuard guard(s->ix->device);
  release(s);  // waits for launches in flight; uncollected results are dropped
  return DK_OK;
}
