// ORACLE — TEST INFRASTRUCTURE ONLY.  CPU restatement of Vamana graph construction: the
// reference's insert path with a deterministic batch schedule, used as the checker of the
// library's host and device builders and to build the benchmark's graph in processes that
// must not load the library (the timed CPU reference arm).
//
// Per inserted point (diskann/src/graph/index.rs:226-341, `insert`):
//   * greedy search from the frozen start points with the build window L_build (beam 1,
//     index.rs:1938-2005), recording every expanded node with its distance (the visited
//     search record, diskann/src/graph/search/record.rs);
//   * the record, sorted by distance and cut to max_occlusion_size (SortedNeighbors,
//     diskann/src/graph/internal/sorted_neighbors.rs:26-40; ties here by id, one of the orders
//     the reference's unstable sort may give), pruned by occlude_list (index.rs:2570-2782:
//     alpha schedule 1, min(alpha,1.2)x, ... up to alpha; TriangleInequality for L2 / cosine,
//     Occluding for inner product, diskann/src/graph/config/mod.rs:60-103) to pruned_degree;
//   * back edges to the point from its first max_backedges out-neighbours
//     (add_edge_and_prune, index.rs:2269-2346): append when new; when the list then exceeds
//     max_degree, prune it with the distances from its owner (robust_prune_list,
//     index.rs:2402-2459).
// Schedule (the library's builder uses the same one): batches of 1, 2, 4, ... up to max_batch
// points; every point of a batch searches the graph as it stood before the batch; then the
// batch's out-lists are set, and the back edges are applied per target with their sources in
// point order.  The graph depends only on the inputs, never on the thread count.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <functional>
#include <limits>
#include <thread>
#include <vector>

#include "oracle.h"

namespace {

struct Cand {
  uint32_t id;
  float d;
};

struct Graph {
  const float* vec;
  uint32_t stride, n, f, dim;
  int32_t metric;
  uint32_t pruned_degree, max_degree, l_build, max_backedges, max_occlusion;
  float alpha;
  std::vector<std::vector<uint32_t>> adj;

  const float* row(uint32_t id) const { return vec + (uint64_t)id * stride; }
  float dist(uint32_t a, uint32_t b) const { return orc_distance(metric, row(a), row(b), dim); }
};

// Search state of one worker: the queue of neighbor/queue.rs (sorted by distance, a new item
// before equal distances, capacity L_build + F) and visited stamps.
struct Worker {
  std::vector<uint32_t> stamp;
  uint32_t epoch = 0;
  std::vector<Cand> queue;
  std::vector<uint8_t> expanded;
  std::vector<Cand> record;
  std::vector<Cand> fresh;
};

void greedy_search(const Graph& G, uint32_t target, Worker& W) {
  const size_t cap = (size_t)G.l_build + G.f;
  if (++W.epoch == 0) {
    std::fill(W.stamp.begin(), W.stamp.end(), 0u);
    W.epoch = 1;
  }
  W.queue.clear();
  W.expanded.clear();
  W.record.clear();
  size_t cursor = 0;
  // NeighborPriorityQueue::insert (queue.rs:130-171).
  auto insert = [&](Cand c) {
    if (std::isnan(c.d)) return;
    const size_t size = W.queue.size();
    if (size == cap && W.queue[size - 1].d < c.d) return;
    size_t at = 0;
    while (at < size && W.queue[at].d < c.d) ++at;
    if (size == cap) {
      W.queue.pop_back();
      W.expanded.pop_back();
    }
    W.queue.insert(W.queue.begin() + at, c);
    W.expanded.insert(W.expanded.begin() + at, 0);
    cursor = std::min(cursor, at);
  };
  const float* q = G.row(target);
  for (uint32_t s = 0; s < G.f; ++s) {
    const uint32_t id = G.n + s;
    W.stamp[id] = W.epoch;
    insert({id, orc_distance(G.metric, q, G.row(id), G.dim)});
  }
  while (cursor < W.queue.size()) {
    // closest_notvisited (queue.rs:297-313).
    const size_t c = cursor;
    W.expanded[c] = 1;
    const Cand node = W.queue[c];
    W.record.push_back(node);
    ++cursor;
    while (cursor < W.queue.size() && W.expanded[cursor]) ++cursor;
    // Score the unvisited neighbours in adjacency order, then insert them in that order.
    W.fresh.clear();
    for (uint32_t nb : G.adj[node.id]) {
      if (W.stamp[nb] == W.epoch) continue;
      W.stamp[nb] = W.epoch;
      W.fresh.push_back({nb, orc_distance(G.metric, q, G.row(nb), G.dim)});
    }
    for (const Cand& x : W.fresh) insert(x);
  }
}

void sort_and_cut(std::vector<Cand>& pool, size_t max_size) {
  std::sort(pool.begin(), pool.end(),
            [](const Cand& a, const Cand& b) { return a.d < b.d || (a.d == b.d && a.id < b.id); });
  if (pool.size() > max_size) pool.resize(max_size);
}

// occlude_list (index.rs:2570-2782) over `pool` sorted by distance to `location`.
std::vector<uint32_t> occlude_list(const Graph& G, uint32_t location, const std::vector<Cand>& pool) {
  std::vector<uint32_t> out;
  if (pool.empty()) return out;
  const bool occluding = G.metric == ORC_METRIC_INNER_PRODUCT;
  std::vector<float> factor(pool.size(), 0.0f);
  std::vector<uint32_t> checked(pool.size(), 0u), chosen;
  float current_alpha = 1.0f;
  const float step = std::min(G.alpha, 1.2f);
  while (chosen.size() < G.pruned_degree) {
    for (size_t i = 0; i < pool.size() && chosen.size() < G.pruned_degree; ++i) {
      float of = factor[i];
      uint32_t lc = checked[i];
      if (of > current_alpha) continue;
      if (pool[i].id == location) {  // the excluded id (a self loop)
        factor[i] = std::numeric_limits<float>::max();
        continue;
      }
      while (lc != chosen.size()) {
        const uint32_t j = chosen[lc];
        ++lc;
        if (j >= i) {
          checked[i] = lc;
          continue;
        }
        const float djk = G.dist(pool[i].id, pool[j].id);
        const float dik = pool[i].d;
        if (occluding) {
          if (djk < current_alpha * dik) of = current_alpha + 0.01f;
        } else {
          of = djk == 0.0f ? std::numeric_limits<float>::max() : std::max(of, dik / djk);
        }
        if (of > current_alpha) break;
      }
      checked[i] = lc;
      if (of > current_alpha) {
        factor[i] = of;
        continue;
      }
      factor[i] = std::numeric_limits<float>::max();
      chosen.push_back((uint32_t)i);
    }
    if (current_alpha == G.alpha) break;
    current_alpha = std::min(current_alpha * step, G.alpha);
  }
  for (uint32_t j : chosen) out.push_back(pool[j].id);
  return out;
}

void for_each_index(uint32_t threads, size_t n, const std::function<void(size_t, uint32_t)>& fn) {
  if (threads <= 1 || n <= 1) {
    for (size_t i = 0; i < n; ++i) fn(i, 0);
    return;
  }
  std::atomic<size_t> next{0};
  std::vector<std::thread> pool;
  const uint32_t t = (uint32_t)std::min<size_t>(threads, n);
  for (uint32_t w = 0; w < t; ++w)
    pool.emplace_back([&, w] {
      for (size_t i; (i = next.fetch_add(1)) < n;) fn(i, w);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" int32_t orc_build_vamana(const float* vectors, uint32_t vector_stride,
                                    uint32_t num_points, uint32_t num_frozen, uint32_t dim,
                                    int32_t metric, const orc_build_params* p,
                                    uint32_t* adjacency, uint32_t adjacency_stride,
                                    uint32_t* degrees) {
  if (!vectors || !p || !adjacency || !degrees || num_frozen == 0 || dim == 0 ||
      vector_stride < dim || p->pruned_degree == 0 || p->max_degree < p->pruned_degree ||
      adjacency_stride < p->max_degree || p->l_build == 0 || !(p->alpha >= 1.0f) ||
      p->max_backedges == 0 || p->max_backedges > p->pruned_degree)
    return ORC_ERR_INVALID_ARGUMENT;
  Graph G;
  G.vec = vectors;
  G.stride = vector_stride;
  G.n = num_points;
  G.f = num_frozen;
  G.dim = dim;
  G.metric = metric;
  G.pruned_degree = p->pruned_degree;
  G.max_degree = p->max_degree;
  G.l_build = p->l_build;
  G.alpha = p->alpha;
  G.max_backedges = p->max_backedges;
  G.max_occlusion = p->max_occlusion ? p->max_occlusion : 750u;
  const uint32_t max_batch = p->max_batch ? p->max_batch : std::max<uint32_t>(64, num_points / 64);
  const uint32_t threads = std::max<uint32_t>(
      1, p->num_threads ? p->num_threads : std::thread::hardware_concurrency());
  const uint32_t total = num_points + num_frozen;
  G.adj.assign(total, {});
  std::vector<Worker> workers(threads);
  for (auto& w : workers) w.stamp.assign(total, 0u);

  std::vector<std::vector<uint32_t>> out;
  uint32_t start = 0, bsize = 1;
  while (start < num_points) {
    const uint32_t end = std::min<uint32_t>(num_points, start + bsize);
    const uint32_t cnt = end - start;
    out.assign(cnt, {});
    for_each_index(threads, cnt, [&](size_t i, uint32_t w) {
      const uint32_t id = start + (uint32_t)i;
      Worker& W = workers[w];
      greedy_search(G, id, W);
      std::vector<Cand> pool;
      for (const Cand& c : W.record)
        if (c.id != id) pool.push_back(c);
      sort_and_cut(pool, G.max_occlusion);
      out[i] = occlude_list(G, id, pool);
    });
    for (uint32_t i = 0; i < cnt; ++i) G.adj[start + i] = out[i];
    // Back edges grouped by target; within a target, sources in point order.
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    for (uint32_t i = 0; i < cnt; ++i)
      for (uint32_t j = 0; j < out[i].size() && j < G.max_backedges; ++j)
        edges.emplace_back(out[i][j], start + i);
    std::sort(edges.begin(), edges.end());
    std::vector<std::pair<size_t, size_t>> groups;
    for (size_t a = 0; a < edges.size();) {
      size_t b = a;
      while (b < edges.size() && edges[b].first == edges[a].first) ++b;
      groups.emplace_back(a, b);
      a = b;
    }
    for_each_index(threads, groups.size(), [&](size_t gi, uint32_t) {
      const uint32_t target = edges[groups[gi].first].first;
      std::vector<uint32_t> lst = G.adj[target];
      bool added = false;
      for (size_t e = groups[gi].first; e < groups[gi].second; ++e) {
        const uint32_t src = edges[e].second;
        if (std::find(lst.begin(), lst.end(), src) == lst.end()) {
          lst.push_back(src);
          added = true;
        }
      }
      if (!added) return;
      if (lst.size() > G.max_degree) {
        std::vector<Cand> pool;
        for (uint32_t id : lst)
          if (id != target) pool.push_back({id, G.dist(target, id)});
        sort_and_cut(pool, G.max_occlusion);
        lst = occlude_list(G, target, pool);
      }
      G.adj[target] = lst;
    });
    start = end;
    bsize = std::min<uint32_t>(bsize * 2, max_batch);
  }
  for (uint32_t i = 0; i < total; ++i) {
    degrees[i] = (uint32_t)G.adj[i].size();
    uint32_t* dst = adjacency + (uint64_t)i * adjacency_stride;
    std::fill(dst, dst + adjacency_stride, 0u);
    std::copy(G.adj[i].begin(), G.adj[i].end(), dst);
  }
  return ORC_OK;
}

// ComputeMedoid for f32 (diskann-utils/src/sampling/medoid.rs:15-45): column sums in f64, the
// mean cast to f32, then the first row whose f32 SquaredL2 to it is strictly smallest.  (The
// reference returns a zero vector when no distance is below f32::MAX; this returns row 0.)
extern "C" uint32_t orc_medoid(const float* vectors, uint32_t stride, uint32_t n, uint32_t dim) {
  std::vector<double> sum(dim, 0.0);
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t d = 0; d < dim; ++d) sum[d] += (double)vectors[(uint64_t)i * stride + d];
  std::vector<float> mean(dim);
  for (uint32_t d = 0; d < dim; ++d) mean[d] = (float)(sum[d] / (double)n);
  float best = std::numeric_limits<float>::max();
  uint32_t arg = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const float d = orc_distance(ORC_METRIC_L2, mean.data(), vectors + (uint64_t)i * stride, dim);
    if (d < best) {
      best = d;
      arg = i;
    }
  }
  return arg;
}
