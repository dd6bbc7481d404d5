// Host-side data tooling on either side of the search path: Vamana graph construction,
// the medoid start point, and product-quantisation training / encoding.
//
// Graph construction restates the reference's insert path
//   insert                 diskann/src/graph/index.rs:226-341
//   occlude_list           diskann/src/graph/index.rs:2570-2782 (alpha schedule, PruneKind)
//   add_edge_and_prune     diskann/src/graph/index.rs:2269-2346 (back edges, prune on overflow)
//   PruneKind              diskann/src/graph/config/mod.rs:69-103
// with deterministic batches instead of concurrent tasks: a batch of points is searched
// against the graph as it stood before the batch (in parallel), each point's out-list is
// pruned from its visited record, and back edges are then applied per target in point order.
// Batches grow 1, 2, 4, ... up to `max_batch`, so early points see a sequentially built graph.
// The result depends only on the inputs and the batch schedule, never on thread timing.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "diskann_b200.h"
#include "dk_build_gpu.h"
#include "dk_internal.cuh"

namespace {

// Distance with the reference's float rounding sequence (see dk_search.cu): four
// 8-lane accumulators over 32-float blocks, (s0+s1)+(s2+s3), masked remainder, sum_tree.
template <bool IP>
inline float simd_order(const float* x, const float* y, size_t len) {
  float s[4][8] = {};
  const size_t trip = len / 32, epi = (len - 32 * trip) / 8;
  for (size_t b = 0; b < trip; ++b)
    for (int j = 0; j < 4; ++j)
      for (int l = 0; l < 8; ++l) {
        const size_t e = 32 * b + 8 * j + l;
        if (IP) s[j][l] = std::fma(x[e], y[e], s[j][l]);
        else { const float c = x[e] - y[e]; s[j][l] = std::fma(c, c, s[j][l]); }
      }
  for (size_t j = 0; j < epi; ++j)
    for (int l = 0; l < 8; ++l) {
      const size_t e = 32 * trip + 8 * j + l;
      if (IP) s[j][l] = std::fma(x[e], y[e], s[j][l]);
      else { const float c = x[e] - y[e]; s[j][l] = std::fma(c, c, s[j][l]); }
    }
  float t[8];
  for (int l = 0; l < 8; ++l) t[l] = (s[0][l] + s[1][l]) + (s[2][l] + s[3][l]);
  const size_t rem = len % 8, base = len - rem;
  for (size_t l = 0; l < rem; ++l) {
    if (IP) t[l] = std::fma(x[base + l], y[base + l], t[l]);
    else { const float c = x[base + l] - y[base + l]; t[l] = std::fma(c, c, t[l]); }
  }
  const float q0 = t[0] + t[4], q1 = t[1] + t[5], q2 = t[2] + t[6], q3 = t[3] + t[7];
  return (q0 + q2) + (q1 + q3);
}

// CosineStateless on x86-64-v3: Strategy2x4 (simd.rs:422-482) — full 8-wide vectors
// alternate between two accumulator sets, combined as set0 + set1, then the masked remainder.
float cosine_sim(const float* x, const float* y, size_t len) {
  float sx[2][8] = {}, sy[2][8] = {}, sxy[2][8] = {};
  const size_t nvec = len / 8;
  for (size_t k = 0; k < nvec; ++k)
    for (int l = 0; l < 8; ++l) {
      const size_t e = 8 * k + l;
      const int j = (int)(k & 1);
      sx[j][l] = std::fma(x[e], x[e], sx[j][l]);
      sy[j][l] = std::fma(y[e], y[e], sy[j][l]);
      sxy[j][l] = std::fma(x[e], y[e], sxy[j][l]);
    }
  float tx[8], ty[8], txy[8];
  for (int l = 0; l < 8; ++l) {
    tx[l] = sx[0][l] + sx[1][l];
    ty[l] = sy[0][l] + sy[1][l];
    txy[l] = sxy[0][l] + sxy[1][l];
  }
  const size_t rem = len % 8, base = len - rem;
  for (size_t l = 0; l < rem; ++l) {
    const float a = x[base + l], b = y[base + l];
    tx[l] = std::fma(a, a, tx[l]);
    ty[l] = std::fma(b, b, ty[l]);
    txy[l] = std::fma(a, b, txy[l]);
  }
  auto tree = [](const float* t) {
    const float q0 = t[0] + t[4], q1 = t[1] + t[5], q2 = t[2] + t[6], q3 = t[3] + t[7];
    return (q0 + q2) + (q1 + q3);
  };
  const float nx = tree(tx), ny = tree(ty);
  const float denom = std::sqrt(nx) * std::sqrt(ny);
  const float prod = tree(txy);
  if (nx < std::numeric_limits<float>::min() || ny < std::numeric_limits<float>::min()) return 0.0f;
  return std::max(-1.0f, std::min(1.0f, prod / denom));
}

inline float metric_distance(int32_t metric, const float* x, const float* y, size_t len) {
  switch (metric) {
    case DK_METRIC_L2: return simd_order<false>(x, y, len);
    case DK_METRIC_INNER_PRODUCT: return -simd_order<true>(x, y, len);
    case DK_METRIC_COSINE: return 1.0f - cosine_sim(x, y, len);
    default: return 1.0f - simd_order<true>(x, y, len);
  }
}

void parallel_for(uint32_t threads, uint64_t n, const std::function<void(uint64_t, uint32_t)>& fn) {
  if (threads <= 1 || n <= 1) {
    for (uint64_t i = 0; i < n; ++i) fn(i, 0);
    return;
  }
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> pool;
  const uint32_t t = (uint32_t)std::min<uint64_t>(threads, n);
  pool.reserve(t);
  for (uint32_t w = 0; w < t; ++w)
    pool.emplace_back([&, w] {
      while (true) {
        const uint64_t i = next.fetch_add(1);
        if (i >= n) break;
        fn(i, w);
      }
    });
  for (auto& th : pool) th.join();
}

struct Candidate {
  uint32_t id;
  float dist;
};

// Per-thread search state for construction-time greedy search.
struct BuildScratch {
  std::vector<uint32_t> stamp;  // visited stamps, one per id
  uint32_t epoch = 0;
  std::vector<uint32_t> q_ids;
  std::vector<float> q_d;
  std::vector<uint8_t> q_vis;
  std::vector<Candidate> visited_record;
  std::vector<float> pool_vecs_dist;
};

struct Builder {
  const float* vec;
  uint64_t stride;
  uint32_t n, f, dim;
  int32_t metric;
  dk_build_params p;
  std::vector<std::vector<uint32_t>> adj;
  bool occluding;  // PruneKind::Occluding for inner product, TriangleInequality otherwise

  const float* row(uint32_t id) const { return vec + (uint64_t)id * stride; }
  float dist(uint32_t a, uint32_t b) const { return metric_distance(metric, row(a), row(b), dim); }

  // Greedy search (index.rs:1938-2005 with beam 1) from the frozen points; records every
  // expanded node with its distance (VisitedSearchRecord, search/record.rs:58-90).
  void search(uint32_t target, BuildScratch& S) const {
    const uint32_t cap = p.l_build + f;
    if (++S.epoch == 0) {
      std::fill(S.stamp.begin(), S.stamp.end(), 0u);
      S.epoch = 1;
    }
    S.q_ids.clear();
    S.q_d.clear();
    S.q_vis.clear();
    S.visited_record.clear();
    size_t cursor = 0;
    auto insert = [&](uint32_t id, float d) {
      if (std::isnan(d)) return;
      size_t size = S.q_ids.size();
      if (size == cap && S.q_d[size - 1] < d) return;
      size_t idx = 0;
      while (idx < size && S.q_d[idx] < d) ++idx;
      if (size == cap) {
        S.q_ids.pop_back();
        S.q_d.pop_back();
        S.q_vis.pop_back();
      }
      S.q_ids.insert(S.q_ids.begin() + idx, id);
      S.q_d.insert(S.q_d.begin() + idx, d);
      S.q_vis.insert(S.q_vis.begin() + idx, 0);
      if (idx < cursor) cursor = idx;
    };
    const float* q = row(target);
    for (uint32_t s = 0; s < f; ++s) {
      const uint32_t id = n + s;
      S.stamp[id] = S.epoch;
      insert(id, metric_distance(metric, q, row(id), dim));
    }
    std::vector<Candidate> batch;
    while (cursor < S.q_ids.size()) {
      const size_t c = cursor;
      S.q_vis[c] = 1;
      const uint32_t node = S.q_ids[c];
      S.visited_record.push_back({node, S.q_d[c]});
      ++cursor;
      while (cursor < S.q_ids.size() && S.q_vis[cursor]) ++cursor;
      batch.clear();
      for (uint32_t nb : adj[node]) {
        if (S.stamp[nb] == S.epoch) continue;
        S.stamp[nb] = S.epoch;
        batch.push_back({nb, metric_distance(metric, q, row(nb), dim)});
      }
      for (const auto& cd : batch) insert(cd.id, cd.dist);
    }
  }

  // occlude_list (index.rs:2570-2782) over a pool sorted by distance to `location`.
  void occlude(uint32_t location, const std::vector<Candidate>& pool,
               std::vector<uint32_t>& out) const {
    out.clear();
    if (pool.empty()) return;
    const uint32_t degree = p.pruned_degree;
    struct St { float of; uint32_t last_checked; uint32_t neighbor; };
    std::vector<St> st(pool.size(), St{0.0f, 0u, 0u});
    float current_alpha = 1.0f;
    const float inc = std::min(p.alpha, 1.2f);
    uint32_t found = 0;
    while (found < degree) {
      for (size_t i = 0; i < pool.size(); ++i) {
        if (found >= degree) break;
        float of = st[i].of;
        uint32_t lc = st[i].last_checked;
        if (of > current_alpha) continue;
        if (pool[i].id == location) {
          st[i].of = std::numeric_limits<float>::max();
          continue;
        }
        while (lc != found) {
          const uint32_t rp = st[lc].neighbor;
          ++lc;
          if (rp >= i) {
            st[i].last_checked = lc;
            continue;
          }
          const float djk = dist(pool[i].id, pool[rp].id);
          const float dik = pool[i].dist;
          if (occluding) {
            if (djk < current_alpha * dik) of = current_alpha + 0.01f;
          } else {
            of = djk == 0.0f ? std::numeric_limits<float>::max() : std::max(of, dik / djk);
          }
          if (of > current_alpha) break;
        }
        st[i].last_checked = lc;
        if (of > current_alpha) {
          st[i].of = of;
          continue;
        }
        st[i].of = std::numeric_limits<float>::max();
        st[found].neighbor = (uint32_t)i;
        ++found;
      }
      if (current_alpha == p.alpha) break;
      current_alpha = std::min(current_alpha * inc, p.alpha);
    }
    for (uint32_t j = 0; j < found; ++j) out.push_back(pool[st[j].neighbor].id);
  }

  static void sort_pool(std::vector<Candidate>& pool, size_t max_size) {
    std::sort(pool.begin(), pool.end(), [](const Candidate& a, const Candidate& b) {
      return a.dist < b.dist || (a.dist == b.dist && a.id < b.id);
    });
    if (pool.size() > max_size) pool.resize(max_size);
  }
};

}  // namespace

extern "C" int32_t dk_distance(int32_t metric, const float* x, const float* y, uint32_t len,
                               float* out) {
  if (!x || !y || !out) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "null argument");
    return DK_ERR_INVALID_ARGUMENT;
  }
  if (metric < DK_METRIC_COSINE || metric > DK_METRIC_COSINE_NORMALIZED) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "unknown metric");
    return DK_ERR_INVALID_ARGUMENT;
  }
  *out = metric_distance(metric, x, y, len);
  return DK_OK;
}

// ComputeMedoid for f32 (diskann-utils/src/sampling/medoid.rs:15-45): mean in f64 cast to
// f32, then the first row with the strictly smallest squared L2 distance to it.
extern "C" int32_t dk_compute_medoid(const float* vectors, uint64_t stride, uint32_t n,
                                     uint32_t dim, uint32_t* medoid) {
  if (!vectors || !medoid || n == 0 || dim == 0 || stride < dim) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "invalid medoid arguments");
    return DK_ERR_INVALID_ARGUMENT;
  }
  std::vector<double> sum(dim, 0.0);
  for (uint32_t i = 0; i < n; ++i) {
    const float* r = vectors + (uint64_t)i * stride;
    for (uint32_t d = 0; d < dim; ++d) sum[d] += (double)r[d];
  }
  std::vector<float> mean(dim);
  for (uint32_t d = 0; d < dim; ++d) mean[d] = (float)(sum[d] / (double)n);
  float best = std::numeric_limits<float>::max();
  uint32_t arg = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const float dd = simd_order<false>(mean.data(), vectors + (uint64_t)i * stride, dim);
    if (dd < best) {
      best = dd;
      arg = i;
    }
  }
  *medoid = arg;
  return DK_OK;
}

namespace {

// Batches at least this large search on the GPU when a device builder is given; smaller ones
// (the first few, which grow 1, 2, 4, ...) search on the host threads.
constexpr uint32_t kGpuMinBatch = 256;

int32_t build_impl(const float* vectors, uint64_t stride, uint32_t num_points, uint32_t num_frozen,
                   uint32_t dim, int32_t metric, const dk_build_params* params, uint32_t* adjacency,
                   uint64_t adjacency_stride, uint32_t* degrees, int32_t device) {
  if (!vectors || !params || !adjacency || !degrees || dim == 0 || stride < dim ||
      num_frozen == 0) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "invalid build arguments");
    return DK_ERR_INVALID_ARGUMENT;
  }
  const dk_build_params& p = *params;
  if (p.pruned_degree == 0 || p.max_degree < p.pruned_degree || p.l_build == 0 ||
      adjacency_stride < p.max_degree || !(p.alpha >= 1.0f) || p.max_backedges == 0 ||
      p.max_backedges > p.pruned_degree) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "invalid build parameters");
    return DK_ERR_INVALID_ARGUMENT;
  }
  Builder B;
  B.vec = vectors;
  B.stride = stride;
  B.n = num_points;
  B.f = num_frozen;
  B.dim = dim;
  B.metric = metric;
  B.p = p;
  if (B.p.max_occlusion == 0) B.p.max_occlusion = 750;
  if (B.p.max_batch == 0) B.p.max_batch = std::max<uint32_t>(64, num_points / 64);
  B.occluding = metric == DK_METRIC_INNER_PRODUCT;
  const uint32_t total = num_points + num_frozen;
  B.adj.assign(total, {});
  const uint32_t threads = std::max<uint32_t>(1, p.num_threads ? p.num_threads
                                                               : std::thread::hardware_concurrency());
  std::vector<BuildScratch> scratch(threads);
  for (auto& s : scratch) s.stamp.assign(total, 0u);

  dk_build_gpu* gpu = nullptr;
  if (device >= 0) {
    const int32_t rc = dk_build_gpu_create(vectors, stride, num_points, num_frozen, dim, metric,
                                           B.p.max_degree, B.p.l_build, B.p.max_batch, device, &gpu);
    if (rc != DK_OK) return rc;
  }
  struct GpuGuard {
    dk_build_gpu* g;
    ~GpuGuard() { dk_build_gpu_destroy(g); }
  } gpu_guard{gpu};

  std::vector<std::vector<uint32_t>> out;
  std::vector<uint32_t> changed;
  const dk_build_prune_cfg cfg{B.p.alpha, B.p.pruned_degree, B.p.max_occlusion,
                               B.occluding ? 1u : 0u};
  // While batches run on the GPU, the device adjacency is the graph and B.adj is stale until
  // it is read back; host batches keep B.adj current and push their changed rows.
  bool device_graph = false;
  auto pull_graph = [&]() -> int32_t {
    if (!device_graph) return DK_OK;
    device_graph = false;
    return dk_build_gpu_get_rows(gpu, B.adj);
  };
  // Back-edge grouping by target (sources in point order), reused across batches.
  std::vector<uint32_t> group_of(total, 0xFFFFFFFFu), g_targets, g_off, g_src, g_fill;
  uint32_t start = 0, bsize = 1;
  while (start < num_points) {
    const uint32_t end = std::min<uint32_t>(num_points, start + bsize);
    const uint32_t cnt = end - start;
    out.assign(cnt, {});
    if (gpu && cnt >= kGpuMinBatch) {
      // GPU batch: search, prune each point from its record, append and re-prune the back
      // edges, all on the device graph; the host only groups the back edges.
      device_graph = true;
      const uint32_t *rec_ids = nullptr, *hops = nullptr, *fo = nullptr, *fc = nullptr;
      const float* rec_d = nullptr;
      uint32_t rec_cap = 0;
      int32_t rc = dk_build_gpu_search(gpu, start, cnt, false, &rec_ids, &rec_d, &hops, &rec_cap);
      if (rc == DK_OK) rc = dk_build_gpu_prune_forward(gpu, cnt, cfg, &fo, &fc);
      if (rc != DK_OK) return rc;
      std::vector<uint32_t> host_points;
      for (uint32_t i = 0; i < cnt; ++i) {
        if (fc[i] == 0xFFFFFFFFu) host_points.push_back(i);
        else out[i].assign(fo + (size_t)i * B.p.pruned_degree, fo + (size_t)i * B.p.pruned_degree + fc[i]);
      }
      if (!host_points.empty()) {
        // Records that overflowed: search and prune on the host against the graph before the
        // batch (the device graph is unchanged so far in this batch).
        rc = dk_build_gpu_get_rows(gpu, B.adj);
        if (rc != DK_OK) return rc;
        parallel_for(threads, host_points.size(), [&](uint64_t h, uint32_t w) {
          const uint32_t i = host_points[h];
          BuildScratch& S = scratch[w];
          B.search(start + i, S);
          std::vector<Candidate> pool = S.visited_record;
          pool.erase(std::remove_if(pool.begin(), pool.end(),
                                    [&](const Candidate& c) { return c.id == start + i; }),
                     pool.end());
          Builder::sort_pool(pool, B.p.max_occlusion);
          B.occlude(start + i, pool, out[i]);
        });
      }
      changed.clear();
      for (uint32_t i = 0; i < cnt; ++i) {
        B.adj[start + i] = out[i];
        changed.push_back(start + i);
      }
      rc = dk_build_gpu_set_rows(gpu, changed.data(), (uint32_t)changed.size(), B.adj);
      if (rc != DK_OK) return rc;
      // Group the back edges by target with a counting pass; sources stay in point order.
      g_targets.clear();
      for (uint32_t i = 0; i < cnt; ++i)
        for (uint32_t j = 0; j < out[i].size() && j < p.max_backedges; ++j) {
          const uint32_t t = out[i][j];
          if (group_of[t] == 0xFFFFFFFFu) {
            group_of[t] = (uint32_t)g_targets.size();
            g_targets.push_back(t);
            g_off.push_back(0);
          }
          ++g_off[group_of[t]];
        }
      const uint32_t groups = (uint32_t)g_targets.size();
      g_off.resize(groups + 1);
      uint32_t max_group = 0, acc = 0;
      for (uint32_t gi = 0; gi < groups; ++gi) {
        const uint32_t c = g_off[gi];
        max_group = std::max(max_group, c);
        g_off[gi] = acc;
        acc += c;
      }
      g_off[groups] = acc;
      g_src.resize(acc);
      g_fill.assign(g_off.begin(), g_off.end() - 1);
      for (uint32_t i = 0; i < cnt; ++i)
        for (uint32_t j = 0; j < out[i].size() && j < p.max_backedges; ++j)
          g_src[g_fill[group_of[out[i][j]]]++] = start + i;
      std::vector<uint32_t> oversize;
      rc = dk_build_gpu_backedges(gpu, g_targets.data(), g_off.data(), g_src.data(), groups,
                                  max_group, cfg, oversize);
      if (rc != DK_OK) return rc;
      // Lists too long for the device pool: append and prune on the host, write back.
      for (uint32_t gi : oversize) {
        const uint32_t target = g_targets[gi];
        std::vector<uint32_t> lst;
        rc = dk_build_gpu_get_row(gpu, target, lst);
        if (rc != DK_OK) return rc;
        bool added = false;
        for (uint32_t e = g_off[gi]; e < g_off[gi + 1]; ++e)
          if (std::find(lst.begin(), lst.end(), g_src[e]) == lst.end()) {
            lst.push_back(g_src[e]);
            added = true;
          }
        if (!added) continue;
        if (lst.size() > p.max_degree) {
          std::vector<Candidate> pool;
          for (uint32_t id : lst)
            if (id != target) pool.push_back({id, B.dist(target, id)});
          Builder::sort_pool(pool, B.p.max_occlusion);
          std::vector<uint32_t> pruned;
          B.occlude(target, pool, pruned);
          lst = pruned;
        }
        B.adj[target] = lst;
        rc = dk_build_gpu_set_rows(gpu, &target, 1, B.adj);
        if (rc != DK_OK) return rc;
      }
      for (uint32_t t : g_targets) group_of[t] = 0xFFFFFFFFu;
      g_off.clear();
      start = end;
      bsize = std::min<uint32_t>(bsize * 2, B.p.max_batch);
      continue;
    }
    if (gpu) {
      const int32_t rc = pull_graph();
      if (rc != DK_OK) return rc;
    }
    parallel_for(threads, cnt, [&](uint64_t i, uint32_t w) {
      const uint32_t id = start + (uint32_t)i;
      BuildScratch& S = scratch[w];
      B.search(id, S);
      std::vector<Candidate> pool = S.visited_record;
      pool.erase(std::remove_if(pool.begin(), pool.end(),
                                [&](const Candidate& c) { return c.id == id; }),
                 pool.end());
      Builder::sort_pool(pool, B.p.max_occlusion);
      B.occlude(id, pool, out[i]);
    });
    changed.clear();
    for (uint32_t i = 0; i < cnt; ++i) {
      B.adj[start + i] = out[i];
      changed.push_back(start + i);
    }
    // Back edges (add_edge_and_prune), grouped by target, sources in point order.
    std::vector<std::pair<uint32_t, uint32_t>> edges;  // (target, source)
    for (uint32_t i = 0; i < cnt; ++i) {
      const auto& lst = out[i];
      for (uint32_t j = 0; j < lst.size() && j < p.max_backedges; ++j)
        edges.emplace_back(lst[j], start + i);
    }
    std::sort(edges.begin(), edges.end());
    std::vector<std::pair<size_t, size_t>> groups;
    for (size_t a = 0; a < edges.size();) {
      size_t b = a;
      while (b < edges.size() && edges[b].first == edges[a].first) ++b;
      groups.emplace_back(a, b);
      a = b;
    }
    std::vector<uint8_t> touched(groups.size(), 0);
    parallel_for(threads, groups.size(), [&](uint64_t g, uint32_t) {
      const uint32_t target = edges[groups[g].first].first;
      std::vector<uint32_t> lst = B.adj[target];
      bool added = false;
      for (size_t e = groups[g].first; e < groups[g].second; ++e) {
        const uint32_t src = edges[e].second;
        if (std::find(lst.begin(), lst.end(), src) == lst.end()) {
          lst.push_back(src);
          added = true;
        }
      }
      if (!added) return;
      touched[g] = 1;
      if (lst.size() <= p.max_degree) {
        B.adj[target] = lst;
        return;
      }
      std::vector<Candidate> pool;
      pool.reserve(lst.size());
      for (uint32_t id : lst)
        if (id != target) pool.push_back({id, B.dist(target, id)});
      Builder::sort_pool(pool, B.p.max_occlusion);
      std::vector<uint32_t> pruned;
      B.occlude(target, pool, pruned);
      B.adj[target] = pruned;
    });
    if (gpu) {
      for (size_t g = 0; g < groups.size(); ++g)
        if (touched[g]) {
          const uint32_t target = edges[groups[g].first].first;
          if (target < start || target >= end) changed.push_back(target);
        }
      const int32_t rc = dk_build_gpu_set_rows(gpu, changed.data(), (uint32_t)changed.size(), B.adj);
      if (rc != DK_OK) return rc;
    }
    start = end;
    bsize = std::min<uint32_t>(bsize * 2, B.p.max_batch);
  }
  if (gpu) {
    const int32_t rc = pull_graph();
    if (rc != DK_OK) return rc;
  }
  for (uint32_t i = 0; i < total; ++i) {
    const auto& lst = B.adj[i];
    degrees[i] = (uint32_t)lst.size();
    uint32_t* dst = adjacency + (uint64_t)i * adjacency_stride;
    std::fill(dst, dst + adjacency_stride, 0u);
    std::copy(lst.begin(), lst.end(), dst);
  }
  return DK_OK;
}

}  // namespace

extern "C" int32_t dk_build_vamana(const float* vectors, uint64_t stride, uint32_t num_points,
                                   uint32_t num_frozen, uint32_t dim, int32_t metric,
                                   const dk_build_params* params, uint32_t* adjacency,
                                   uint64_t adjacency_stride, uint32_t* degrees) {
  return build_impl(vectors, stride, num_points, num_frozen, dim, metric, params, adjacency,
                    adjacency_stride, degrees, -1);
}

extern "C" int32_t dk_build_vamana_device(const float* vectors, uint64_t stride,
                                          uint32_t num_points, uint32_t num_frozen, uint32_t dim,
                                          int32_t metric, const dk_build_params* params,
                                          uint32_t* adjacency, uint64_t adjacency_stride,
                                          uint32_t* degrees, int32_t device) {
  if (device < 0) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "device must be a CUDA device ordinal");
    return DK_ERR_INVALID_ARGUMENT;
  }
  return build_impl(vectors, stride, num_points, num_frozen, dim, metric, params, adjacency,
                    adjacency_stride, degrees, device);
}

// Chunk offsets: the first dim % chunks chunks are one longer (diskann-quantization
// views.rs `partition_into`).
static void chunk_offsets(uint32_t dim, uint32_t chunks, uint32_t* off) {
  const uint32_t base = dim / chunks, extra = dim % chunks;
  off[0] = 0;
  for (uint32_t m = 0; m < chunks; ++m) off[m + 1] = off[m] + base + (m < extra ? 1u : 0u);
}

// PQ training: per chunk, k-means++ seeding then Lloyd iterations (256 centres) on the
// given training rows.  Deterministic for a seed.
extern "C" int32_t dk_pq_train(const float* data, uint64_t stride, uint32_t n, uint32_t dim,
                               uint32_t chunks, uint32_t iters, uint64_t seed,
                               uint32_t num_threads, uint32_t* offsets, float* pivots) {
  if (!data || !offsets || !pivots || n == 0 || chunks == 0 || chunks > dim || stride < dim) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "invalid PQ training arguments");
    return DK_ERR_INVALID_ARGUMENT;
  }
  chunk_offsets(dim, chunks, offsets);
  const uint32_t K = 256;
  const uint32_t threads = std::max<uint32_t>(1, num_threads ? num_threads : std::thread::hardware_concurrency());
  parallel_for(threads, chunks, [&](uint64_t m, uint32_t) {
    const uint32_t s = offsets[m], len = offsets[m + 1] - s;
    std::mt19937_64 rng(seed * 1000003ull + m);
    std::vector<float> x((size_t)n * len);
    for (uint32_t i = 0; i < n; ++i)
      std::memcpy(&x[(size_t)i * len], data + (uint64_t)i * stride + s, len * sizeof(float));
    auto d2 = [&](const float* a, const float* b) {
      double acc = 0.0;
      for (uint32_t t = 0; t < len; ++t) {
        const double c = (double)a[t] - (double)b[t];
        acc += c * c;
      }
      return acc;
    };
    std::vector<float> cent((size_t)K * len, 0.0f);
    // k-means++ seeding.
    std::vector<double> best(n, std::numeric_limits<double>::max());
    uint32_t first = (uint32_t)(rng() % n);
    std::memcpy(&cent[0], &x[(size_t)first * len], len * sizeof(float));
    for (uint32_t c = 1; c < K; ++c) {
      double total = 0.0;
      const float* prev = &cent[(size_t)(c - 1) * len];
      for (uint32_t i = 0; i < n; ++i) {
        best[i] = std::min(best[i], d2(&x[(size_t)i * len], prev));
        total += best[i];
      }
      uint32_t pick = (uint32_t)(rng() % n);
      if (total > 0.0) {
        const double r = std::uniform_real_distribution<double>(0.0, total)(rng);
        double acc = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
          acc += best[i];
          if (acc >= r) { pick = i; break; }
        }
      }
      std::memcpy(&cent[(size_t)c * len], &x[(size_t)pick * len], len * sizeof(float));
    }
    // Lloyd iterations.
    std::vector<uint32_t> assign(n, 0);
    std::vector<double> acc((size_t)K * len);
    std::vector<uint32_t> cnt(K);
    for (uint32_t it = 0; it < iters; ++it) {
      for (uint32_t i = 0; i < n; ++i) {
        double bd = std::numeric_limits<double>::max();
        uint32_t bc = 0;
        for (uint32_t c = 0; c < K; ++c) {
          const double dd = d2(&x[(size_t)i * len], &cent[(size_t)c * len]);
          if (dd < bd) { bd = dd; bc = c; }
        }
        assign[i] = bc;
      }
      std::fill(acc.begin(), acc.end(), 0.0);
      std::fill(cnt.begin(), cnt.end(), 0u);
      for (uint32_t i = 0; i < n; ++i) {
        ++cnt[assign[i]];
        for (uint32_t t = 0; t < len; ++t) acc[(size_t)assign[i] * len + t] += x[(size_t)i * len + t];
      }
      for (uint32_t c = 0; c < K; ++c) {
        if (cnt[c] == 0) {  // re-seed an empty centre from a random row
          const uint32_t r = (uint32_t)(rng() % n);
          std::memcpy(&cent[(size_t)c * len], &x[(size_t)r * len], len * sizeof(float));
          continue;
        }
        for (uint32_t t = 0; t < len; ++t)
          cent[(size_t)c * len + t] = (float)(acc[(size_t)c * len + t] / cnt[c]);
      }
    }
    for (uint32_t c = 0; c < K; ++c)
      std::memcpy(pivots + (size_t)c * dim + s, &cent[(size_t)c * len], len * sizeof(float));
  });
  return DK_OK;
}

// PQ encoding: nearest pivot (squared L2) per chunk.
extern "C" int32_t dk_pq_encode(const float* data, uint64_t stride, uint32_t n, uint32_t dim,
                                uint32_t chunks, const uint32_t* offsets, const float* pivots,
                                uint32_t num_threads, uint8_t* codes, uint64_t code_stride) {
  if (!data || !offsets || !pivots || !codes || chunks == 0 || code_stride < chunks || stride < dim) {
    dk_set_error(DK_ERR_INVALID_ARGUMENT, "invalid PQ encode arguments");
    return DK_ERR_INVALID_ARGUMENT;
  }
  const uint32_t threads = std::max<uint32_t>(1, num_threads ? num_threads : std::thread::hardware_concurrency());
  const uint64_t block = 4096;
  parallel_for(threads, (n + block - 1) / block, [&](uint64_t b, uint32_t) {
    const uint64_t lo = b * block, hi = std::min<uint64_t>(n, lo + block);
    for (uint64_t i = lo; i < hi; ++i) {
      const float* r = data + i * stride;
      for (uint32_t m = 0; m < chunks; ++m) {
        const uint32_t s = offsets[m], e = offsets[m + 1];
        float bd = std::numeric_limits<float>::max();
        uint32_t bc = 0;
        for (uint32_t c = 0; c < 256; ++c) {
          const float* pv = pivots + (size_t)c * dim;
          float acc = 0.0f;
          for (uint32_t t = s; t < e; ++t) {
            const float d = r[t] - pv[t];
            acc += d * d;
          }
          if (acc < bd) { bd = acc; bc = c; }
        }
        codes[i * code_stride + m] = (uint8_t)bc;
      }
    }
  });
  return DK_OK;
}
