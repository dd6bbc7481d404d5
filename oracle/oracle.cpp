// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of the reference's in-memory greedy beam search, used as the
// correctness checker for the CUDA path and as the timed CPU baseline.  Nothing in the
// product (the `diskann_b200` package and its shared library) links or calls this file;
// only the tests, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline leg do.
//
// The reference is a Rust workspace that cannot be compiled in this environment (no
// cargo/rustc, crates not vendored), so this restatement is pinned against the
// reference's own golden vectors (diskann/test/generated/graph/test/cases/grid_search/
// *.json, extracted into tests/golden/) which fix exact ids, distances, comparison and
// hop counts, tie order included.
//
// Every function cites the reference file:line it restates.  Paths are relative to the
// reference repository root.
//
// Build: see oracle/Makefile (g++ -O3 -mavx2 -mfma -ffp-contract=off; no fast-math, so every float
// operation rounds exactly as written and every fused multiply-add is an explicit fmaf).

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <thread>
#include <unordered_set>
#include <vector>

#include "oracle.h"

namespace {

// ---------------------------------------------------------------------------------------
// Distances.
//
// diskann-vector/src/distance/simd.rs:686-745 (`simd_op`): with SIMD width 8 and the
// `Strategy4x1` main loop (simd.rs:321-363, BLOCK_SIZE 4), elements are consumed in
// blocks of 32.  Accumulator s_j (j = 0..3), lane l, receives element 32*b + 8*j + l of
// every full block b.  Left-over full 8-wide vectors after the last full block go to
// s0, s1, s2 in turn.  The accumulators are combined as (s0+s1)+(s2+s3) (lane-wise
// vector adds), then a remainder shorter than 8 is masked-loaded (zeros elsewhere) and
// accumulated into the combined accumulator (simd.rs:548-575 default `epilogue`).
// The final reduction is `sum_tree` (diskann-wide/src/arch/x86_64/v3/f32x8_.rs:187-212):
//   q_i = x_i + x_{i+4} (i<4);  d0 = q0 + q2;  d1 = q1 + q3;  result = d0 + d1.
// `mul_add_simd` is `_mm256_fmadd_ps` (f32x8_.rs:53-55): one rounding per lane.
// x86-64-v4 (AVX-512) uses the same f32x8 schema for L2 and IP (simd.rs:786-815,
// 1555-1583), so this order holds on both.
// ---------------------------------------------------------------------------------------

inline float sum_tree8(const float t[8]) {
  const float q0 = t[0] + t[4], q1 = t[1] + t[5], q2 = t[2] + t[6], q3 = t[3] + t[7];
  const float d0 = q0 + q2, d1 = q1 + q3;
  return d0 + d1;
}

enum class Acc { L2, IP };

// Accumulate one lane: L2 uses c = x - y, fma(c, c, acc) (simd.rs:836-844);
// IP uses fma(x, y, acc) (simd.rs:1588-1600).
template <Acc A>
inline float acc_lane(float x, float y, float acc) {
  if (A == Acc::L2) {
    const float c = x - y;
    return std::fmaf(c, c, acc);
  } else {
    return std::fmaf(x, y, acc);
  }
}

template <Acc A>
float simd_op_v3(const float* x, const float* y, size_t len) {
  float s[4][8];
  std::memset(s, 0, sizeof(s));
  const size_t trip = len / 32;
  const size_t epilogues = (len - 32 * trip) / 8;
  for (size_t b = 0; b < trip; ++b)
    for (int j = 0; j < 4; ++j)
      for (int l = 0; l < 8; ++l) {
        const size_t e = 32 * b + 8 * j + l;
        s[j][l] = acc_lane<A>(x[e], y[e], s[j][l]);
      }
  for (size_t j = 0; j < epilogues; ++j)
    for (int l = 0; l < 8; ++l) {
      const size_t e = 32 * trip + 8 * j + l;
      s[j][l] = acc_lane<A>(x[e], y[e], s[j][l]);
    }
  float t[8];
  for (int l = 0; l < 8; ++l) t[l] = (s[0][l] + s[1][l]) + (s[2][l] + s[3][l]);
  const size_t rem = len % 8;
  const size_t base = len - rem;
  for (size_t l = 0; l < rem; ++l) t[l] = acc_lane<A>(x[base + l], y[base + l], t[l]);
  return sum_tree8(t);
}

// Cosine: `CosineStateless` on x86-64-v3 (simd.rs:2430-2460) keeps three f32x8
// accumulators (x*x, y*y, x*y; FullCosineAccumulator::add_with, simd.rs:2307-2315) and runs
// the `Strategy2x4` main loop (simd.rs:422-482): two accumulator sets, the full 8-wide vectors
// in order alternating between them (vector k goes to set k % 2, the peeled odd block and the
// 1-3 full-width epilogues continue the same alternation), combined as s0 + s1; a remainder
// shorter than 8 is then masked-loaded into the combined set (simd.rs:686-745).  `sum`
// (simd.rs:2327-2361): norms and product via sum_tree, zero similarity if either norm is below
// f32::MIN_POSITIVE, otherwise clamp(prod / (sqrt(nx) * sqrt(ny)), -1, 1).
struct CosAcc {
  float x[8], y[8], xy[8];
};

// One `simd_op` of CosineStateless over a slice, before `sum`: the combined accumulator.
CosAcc cosine_accumulate_v3(const float* x, const float* y, size_t len) {
  float sx[2][8], sy[2][8], sxy[2][8];
  std::memset(sx, 0, sizeof(sx));
  std::memset(sy, 0, sizeof(sy));
  std::memset(sxy, 0, sizeof(sxy));
  const size_t nvec = len / 8;
  for (size_t k = 0; k < nvec; ++k)
    for (int l = 0; l < 8; ++l) {
      const float a = x[8 * k + l], b = y[8 * k + l];
      const int j = (int)(k & 1);
      sx[j][l] = std::fmaf(a, a, sx[j][l]);
      sy[j][l] = std::fmaf(b, b, sy[j][l]);
      sxy[j][l] = std::fmaf(a, b, sxy[j][l]);
    }
  CosAcc t;
  for (int l = 0; l < 8; ++l) {
    t.x[l] = sx[0][l] + sx[1][l];
    t.y[l] = sy[0][l] + sy[1][l];
    t.xy[l] = sxy[0][l] + sxy[1][l];
  }
  const size_t rem = len % 8;
  const size_t base = len - rem;
  for (size_t l = 0; l < rem; ++l) {
    const float a = x[base + l], b = y[base + l];
    t.x[l] = std::fmaf(a, a, t.x[l]);
    t.y[l] = std::fmaf(b, b, t.y[l]);
    t.xy[l] = std::fmaf(a, b, t.xy[l]);
  }
  return t;
}

float cosine_sum_v3(const CosAcc& t) {
  const float nx = sum_tree8(t.x);
  const float ny = sum_tree8(t.y);
  const float denom = std::sqrt(nx) * std::sqrt(ny);
  const float prod = sum_tree8(t.xy);
  if (nx < 1.17549435e-38f || ny < 1.17549435e-38f) return 0.0f;
  const float v = prod / denom;
  return std::max(-1.0f, std::min(1.0f, v));
}

float cosine_similarity_v3(const float* x, const float* y, size_t len) {
  return cosine_sum_v3(cosine_accumulate_v3(x, y, len));
}

}  // namespace

// diskann-vector/src/distance/implementations.rs:215-405: the post-ops.
//   L2               -> Σ(x-y)²                      (SquaredL2, no sqrt)
//   InnerProduct     -> -Σxy                         (implementations.rs:292-300)
//   Cosine           -> 1 - clamp(cos)               (implementations.rs:330-369)
//   CosineNormalized -> 1 - Σxy, no clamp            (implementations.rs:373-404)
extern "C" float orc_distance(int32_t metric, const float* x, const float* y, uint32_t len) {
  switch (metric) {
    case ORC_METRIC_L2:
      return simd_op_v3<Acc::L2>(x, y, len);
    case ORC_METRIC_INNER_PRODUCT:
      return -simd_op_v3<Acc::IP>(x, y, len);
    case ORC_METRIC_COSINE:
      return 1.0f - cosine_similarity_v3(x, y, len);
    case ORC_METRIC_COSINE_NORMALIZED:
      return 1.0f - simd_op_v3<Acc::IP>(x, y, len);
    default:
      return NAN;
  }
}

namespace {

// ---------------------------------------------------------------------------------------
// NeighborPriorityQueue (diskann/src/neighbor/queue.rs:68-519), fixed-capacity mode.
// ---------------------------------------------------------------------------------------
struct Queue {
  std::vector<uint32_t> ids;
  std::vector<uint8_t> visited;
  std::vector<float> dists;
  size_t size = 0;
  size_t capacity = 0;
  size_t cursor = 0;
  size_t search_l = 0;
  bool resizable = false;  // queue.rs:108-119 auto_resizable: never drops, grows instead

  explicit Queue(size_t cap) : capacity(cap), search_l(cap) {
    ids.reserve(cap + 1);
    visited.reserve(cap + 1);
    dists.reserve(cap + 1);
  }

  // queue.rs:229-280 `get_lower_bound`: index of the first distance >= target.
  size_t lower_bound(float d) const {
    for (size_t i = 0; i < size; ++i)
      if (dists[i] >= d) return i;
    return size;
  }

  // queue.rs:130-171 `insert`.
  void insert(uint32_t id, float d) {
    if (std::isnan(d)) return;
    if (resizable) {
      if (size == capacity) capacity += std::max<size_t>(1, capacity >> 1);  // 1.5x
    } else if (size == capacity && dists[size - 1] < d) {
      return;
    }
    const size_t idx = size > 0 ? lower_bound(d) : 0;
    if (size == capacity) {
      ids.pop_back();
      visited.pop_back();
      dists.pop_back();
      --size;
    }
    ids.insert(ids.begin() + idx, id);
    visited.insert(visited.begin() + idx, 0);
    dists.insert(dists.begin() + idx, d);
    ++size;
    if (idx < cursor) cursor = idx;
  }

  // queue.rs:316-318 `has_notvisited_node`.
  bool has_notvisited() const { return cursor < std::min(search_l, size); }

  // queue.rs:297-313 `closest_notvisited`.
  bool closest_notvisited(uint32_t* out) {
    if (!has_notvisited()) return false;
    const size_t cur = cursor;
    visited[cur] = 1;
    ++cursor;
    while (cursor < size && visited[cursor]) ++cursor;
    *out = ids[cur];
    return true;
  }

  // queue.rs:190-193 `iter`: first min(search_l, size) entries.
  size_t iter_len() const { return std::min(search_l, size); }

  // queue.rs:174-181 `drain_best`: drop the first `count` entries; the cursor restarts at 0.
  void drain_best(size_t count) {
    count = std::min(count, size);
    ids.erase(ids.begin(), ids.begin() + count);
    visited.erase(visited.begin(), visited.begin() + count);
    dists.erase(dists.begin(), dists.begin() + count);
    size -= count;
    cursor = 0;
  }
};

// Visited set: an open-addressing u32 set with linear probing that doubles at 50% load.
// Membership semantics are those of the reference's hashbrown::HashSet<u32> (scratch.rs:41-48).
struct VisitedSet {
  std::vector<uint32_t> slots;
  size_t mask = 0, count = 0;
  explicit VisitedSet(size_t hint) {
    size_t cap = 16;
    while (cap < 2 * hint) cap <<= 1;
    slots.assign(cap, 0xFFFFFFFFu);
    mask = cap - 1;
  }
  static size_t hash(uint32_t id) { return (size_t)(id * 2654435761u); }
  // Returns true if `id` was newly inserted.
  void clear() {
    std::fill(slots.begin(), slots.end(), 0xFFFFFFFFu);
    count = 0;
  }
  bool insert(uint32_t id) {
    if (2 * (count + 1) > slots.size()) grow();
    size_t h = hash(id) & mask;
    while (true) {
      const uint32_t cur = slots[h];
      if (cur == id) return false;
      if (cur == 0xFFFFFFFFu) {
        slots[h] = id;
        ++count;
        return true;
      }
      h = (h + 1) & mask;
    }
  }
  void grow() {
    std::vector<uint32_t> old;
    old.swap(slots);
    slots.assign(old.size() * 2, 0xFFFFFFFFu);
    mask = slots.size() - 1;
    count = 0;
    for (uint32_t v : old)
      if (v != 0xFFFFFFFFu) insert(v);
  }
};

inline const float* vec_row(const orc_index* ix, uint32_t id) {
  return ix->vectors + (size_t)id * ix->vector_stride;
}

// diskann-providers/src/model/pq/fixed_chunk_pq_table.rs:149-215
// `populate_chunk_distances_impl`: table[m*256 + c] = F(query_chunk_m, pivot_c_chunk_m),
// with F = SquaredL2 (L2, CosineNormalized; pq/distance/dynamic.rs:78-81) or
// InnerProduct (= -dot; IP).
void pq_table(const orc_index* ix, const float* q, std::vector<float>& table) {
  const uint32_t m_count = ix->pq_chunks;
  table.assign((size_t)m_count * 256, 0.0f);
  const bool ip = ix->metric == ORC_METRIC_INNER_PRODUCT;
  for (uint32_t c = 0; c < 256; ++c) {
    const float* pivot = ix->pq_pivots + (size_t)c * ix->dim;
    for (uint32_t m = 0; m < m_count; ++m) {
      const uint32_t start = ix->pq_offsets[m], stop = ix->pq_offsets[m + 1];
      const float v = ip ? -simd_op_v3<Acc::IP>(q + start, pivot + start, stop - start)
                         : simd_op_v3<Acc::L2>(q + start, pivot + start, stop - start);
      table[(size_t)m * 256 + c] = v;
    }
  }
}

// fixed_chunk_pq_table.rs:79-95 `pq_dist_lookup_single`: sequential f32 sum, m ascending.
inline float pq_lookup(const std::vector<float>& table, const uint8_t* code, uint32_t m_count) {
  float acc = 0.0f;
  for (uint32_t m = 0; m < m_count; ++m) acc += table[(size_t)m * 256 + code[m]];
  return acc;
}

// PQ with the Cosine metric: `DirectCosine` (pq/distance/dynamic.rs:80, cosine.rs:27-70) →
// `FixedChunkPQTable::cosine_distance` (fixed_chunk_pq_table.rs:233-243) →
// `direct_distance_impl::<ResumableCosine>` (fixed_chunk_pq_table.rs:32-56): for every chunk m
// one CosineStateless `simd_op` over (query[start..stop], pivot[code[m]][start..stop]) from a
// fresh accumulator, folded into the running one lane by lane (`combine_with`: self + chunk,
// simd.rs:3184-3190), then `sum` (the cosine similarity); distance = 1 - similarity.
float pq_direct_cosine(const orc_index* ix, const float* q, const uint8_t* code) {
  CosAcc total;
  std::memset(&total, 0, sizeof(total));
  for (uint32_t m = 0; m < ix->pq_chunks; ++m) {
    const uint32_t start = ix->pq_offsets[m], stop = ix->pq_offsets[m + 1];
    const float* pivot = ix->pq_pivots + (size_t)code[m] * ix->dim;
    const CosAcc a = cosine_accumulate_v3(q + start, pivot + start, stop - start);
    for (int l = 0; l < 8; ++l) {
      total.x[l] = total.x[l] + a.x[l];
      total.y[l] = total.y[l] + a.y[l];
      total.xy[l] = total.xy[l] + a.xy[l];
    }
  }
  return 1.0f - cosine_sum_v3(total);
}

struct Scorer {
  const orc_index* ix;
  const float* query;
  bool pq;
  std::vector<float> table;

  float operator()(uint32_t id) const {
    if (pq) {
      const uint8_t* code = ix->pq_codes + (size_t)id * ix->pq_code_stride;
      if (ix->metric == ORC_METRIC_COSINE) return pq_direct_cosine(ix, query, code);
      return pq_lookup(table, code, ix->pq_chunks);
    }
    return orc_distance(ix->metric, query, vec_row(ix, id), ix->dim);
  }
};

// One node of `expand_beam`: its adjacency list in stored order, retained by the visited-set
// insert predicate (glue.rs:524-561 NotInMut), each retained id scored, in order.
template <class Score>
void expand(const orc_index* ix, const Score& score, VisitedSet& visited, uint32_t node,
            std::vector<std::pair<uint32_t, float>>& out) {
  const uint32_t deg = ix->degrees[node];
  const uint32_t* adj = ix->adjacency + (size_t)node * ix->adjacency_stride;
  for (uint32_t t = 0; t < deg; ++t) {
    const uint32_t id = adj[t];
    if (visited.insert(id)) out.emplace_back(id, score(id));
  }
}

// The `search_internal` loop after the start points (index.rs:1964-2005).
template <class Score>
void search_loop(const orc_index* ix, const Score& score, Queue& best, VisitedSet& visited,
                 uint32_t beam_width, uint32_t& cmps, uint32_t& hops) {
  std::vector<uint32_t> beam;
  std::vector<std::pair<uint32_t, float>> neighbors;
  neighbors.reserve((size_t)ix->max_degree * beam_width);
  while (best.has_notvisited()) {
    beam.clear();
    uint32_t node;
    while (beam.size() < beam_width && best.closest_notvisited(&node)) beam.push_back(node);
    neighbors.clear();
    // expand_beam: per beam node, its adjacency list in stored order, retained by the
    // visited-set insert predicate (glue.rs:524-561 NotInMut), scored in order.
    for (uint32_t n : beam) expand(ix, score, visited, n, neighbors);
    for (const auto& nb : neighbors) best.insert(nb.first, nb.second);
    cmps += (uint32_t)neighbors.size();
    hops += (uint32_t)beam.size();
  }
}

}  // namespace

// diskann/src/graph/search/knn_search.rs:94-119 `Knn::new` validation.
extern "C" int32_t orc_validate_knn(uint32_t k, uint32_t l, uint32_t beam_width) {
  if (k == 0) return ORC_ERR_K_ZERO;
  if (l == 0) return ORC_ERR_L_ZERO;
  if (k > l) return ORC_ERR_L_LESS_THAN_K;
  if (beam_width == 0) return ORC_ERR_BEAM_WIDTH_ZERO;
  return ORC_OK;
}

// Range search (diskann/src/graph/search/range_search.rs), FullPrecision accessor:
//   Range::with_options validation (range_search.rs:63-110);
//   `search` (range_search.rs:157-247): search_internal with a queue of starting_l + #start
//     points; in_range = the first starting_l queue entries with distance <= radius; the
//     visited set is cleared and refilled with them; a second round runs when
//     |in_range| >= (starting_l as f32 * initial_slack) as usize and |in_range| < max_returned;
//     the post-processor (FilterStartPoints + copy) writes in_range through DistanceFiltered
//     (inner_radius < distance <= radius);
//   `range_search_internal` (range_search.rs:331-389): a FIFO frontier seeded with in_range;
//     pop beam_width nodes, expand them through the visited set, append every scored neighbour
//     with distance <= radius * range_slack while |in_range| < max_returned.
//   Stats: cmps of the first round only; when the second round runs, hops = the first round's
//     hops plus the scratch counter, which itself started at the first round's hops
//     (range_search.rs:204-209, 380-387), so the first round's hops count twice.
// inner_radius NaN means none; max_returned 0 means unlimited; at most `capacity` results are
// written (flags bit 2 set if more passed the filter).  flags bit 1: second round ran.
extern "C" int32_t orc_range_search(const orc_index* ix, const float* query, uint32_t starting_l,
                                    uint32_t beam_width, float radius, float inner_radius,
                                    float initial_slack, float range_slack, uint32_t max_returned,
                                    uint32_t capacity, uint32_t* ids_out, float* dists_out,
                                    orc_stats* stats) {
  if (beam_width == 0) return ORC_ERR_BEAM_WIDTH_ZERO;
  if (starting_l == 0) return ORC_ERR_L_ZERO;
  if (max_returned && max_returned < starting_l) return ORC_ERR_INVALID_ARGUMENT;
  if (!(initial_slack >= 0.0f && initial_slack <= 1.0f)) return ORC_ERR_INVALID_ARGUMENT;
  if (!(range_slack >= 1.0f)) return ORC_ERR_INVALID_ARGUMENT;
  if (!std::isnan(inner_radius) && inner_radius > radius) return ORC_ERR_INVALID_ARGUMENT;
  const size_t max_ret = max_returned ? max_returned : SIZE_MAX;

  Scorer score{ix, query, false, {}};
  const uint32_t n_start = ix->num_frozen;
  Queue best((size_t)starting_l + n_start);
  VisitedSet visited((size_t)std::ceil(1.1 * ix->max_degree * 1.3 * starting_l));
  uint32_t cmps = 0, hops = 0;
  for (uint32_t s = 0; s < n_start; ++s) {
    const uint32_t id = ix->num_points + s;
    visited.insert(id);
    best.insert(id, score(id));
    cmps += 1;
  }
  search_loop(ix, score, best, visited, beam_width, cmps, hops);

  std::vector<std::pair<uint32_t, float>> in_range;
  const size_t n_iter = std::min(best.iter_len(), (size_t)starting_l);
  for (size_t i = 0; i < n_iter; ++i)
    if (best.dists[i] <= radius) in_range.emplace_back(best.ids[i], best.dists[i]);
  visited.clear();
  for (const auto& e : in_range) visited.insert(e.first);
  const bool second = in_range.size() >= (size_t)((float)starting_l * initial_slack) &&
                      in_range.size() < max_ret;
  uint32_t total_hops = hops;
  if (second) {
    std::deque<uint32_t> frontier;
    for (const auto& e : in_range) frontier.push_back(e.first);
    const float limit = radius * range_slack;
    uint32_t scratch_hops = hops;
    std::vector<uint32_t> beam;
    std::vector<std::pair<uint32_t, float>> neighbors;
    while (!frontier.empty() && in_range.size() < max_ret) {
      beam.clear();
      while (!frontier.empty() && beam.size() < beam_width) {
        beam.push_back(frontier.front());
        frontier.pop_front();
      }
      neighbors.clear();
      for (uint32_t n : beam) expand(ix, score, visited, n, neighbors);
      for (const auto& nb : neighbors)
        if (nb.second <= limit && in_range.size() < max_ret) {
          in_range.push_back(nb);
          frontier.push_back(nb.first);
        }
      scratch_hops += (uint32_t)beam.size();
    }
    total_hops = hops + scratch_hops;
  }
  uint32_t count = 0, passed = 0;
  for (const auto& e : in_range) {
    if (e.first >= ix->num_points) continue;  // FilterStartPoints
    if (!std::isnan(inner_radius) && e.second <= inner_radius) continue;
    if (!(e.second <= radius)) continue;
    ++passed;
    if (count < capacity) {
      ids_out[count] = e.first;
      dists_out[count] = e.second;
      ++count;
    }
  }
  if (stats) {
    stats->cmps = cmps;
    stats->hops = total_hops;
    stats->result_count = count;
    stats->flags = (second ? 2u : 0u) | (passed > count ? 4u : 0u);
  }
  return ORC_OK;
}

// Paged search (diskann/src/graph/search/paged.rs; index.rs:2080-2160), FullPrecision
// accessor.  A session holds the resizable queue (capacity L + #start points, never
// dropping), the visited set, the page cache and the running comparison / hop counters.
struct orc_paged {
  const orc_index* ix;
  std::vector<float> query;
  Queue best;
  VisitedSet visited;
  std::vector<std::pair<uint32_t, float>> computed;  // computed_result
  size_t next = 0;                                    // next_result_index
  uint32_t l_value = 0;
  uint32_t cmps = 0, hops = 0;
  orc_paged(const orc_index* x, size_t qcap, size_t vcap) : ix(x), best(qcap), visited(vcap) {}
};

// index.rs:2101-2160 `paged_search_with_init_ids`: the init ids (default: the start points)
// go into the visited set, their neighbours are expanded through it and inserted in order;
// the counters start at zero (search_internal then skips the start-point step because the
// visited set is not empty, index.rs:1953-1963).
extern "C" int32_t orc_paged_create(const orc_index* ix, const float* query, uint32_t l_value,
                                    const uint32_t* init_ids, uint32_t n_init,
                                    orc_paged** out) {
  if (!ix || !query || !out) return ORC_ERR_INVALID_ARGUMENT;
  const uint32_t n_start = ix->num_frozen;
  auto* ps = new orc_paged(ix, (size_t)l_value + n_start,
                           (size_t)std::ceil(1.1 * ix->max_degree * 1.3 * l_value));
  ps->best.resizable = true;
  ps->query.assign(query, query + ix->dim);
  ps->l_value = l_value;
  std::vector<uint32_t> init;
  if (n_init) init.assign(init_ids, init_ids + n_init);
  else
    for (uint32_t s = 0; s < n_start; ++s) init.push_back(ix->num_points + s);
  for (uint32_t id : init) ps->visited.insert(id);
  Scorer score{ix, ps->query.data(), false, {}};
  std::vector<std::pair<uint32_t, float>> neighbors;
  for (uint32_t id : init) expand(ix, score, ps->visited, id, neighbors);
  for (const auto& nb : neighbors) ps->best.insert(nb.first, nb.second);
  ps->computed.assign(l_value, {0u, 0.0f});
  ps->next = l_value;
  *out = ps;
  return ORC_OK;
}

// paged.rs:52-126 `next_page` with `filter_search_candidates` (paged.rs:128-151).
extern "C" int32_t orc_paged_next(orc_paged* ps, uint32_t k, uint32_t* ids_out,
                                  float* dists_out, uint32_t* count_out, orc_stats* stats) {
  if (!ps) return ORC_ERR_INVALID_ARGUMENT;
  if (k > ps->l_value || k == 0) return ORC_ERR_INVALID_ARGUMENT;
  const orc_index* ix = ps->ix;
  uint32_t n = 0;
  const size_t available = ps->computed.size() > ps->next ? ps->computed.size() - ps->next : 0;
  const size_t from_cache = std::min<size_t>(k, available);
  for (size_t i = 0; i < from_cache; ++i) {
    ids_out[n] = ps->computed[ps->next + i].first;
    dists_out[n++] = ps->computed[ps->next + i].second;
  }
  ps->next += from_cache;
  if (n < k) {
    Scorer score{ix, ps->query.data(), false, {}};
    search_loop(ix, score, ps->best, ps->visited, 1, ps->cmps, ps->hops);
    std::vector<std::pair<uint32_t, float>> cand;
    size_t total = 0;
    for (size_t i = 0; i < ps->best.iter_len(); ++i) {
      ++total;
      if (ps->best.ids[i] < ix->num_points) {  // start points are ids N..N+F-1
        cand.emplace_back(ps->best.ids[i], ps->best.dists[i]);
        if (cand.size() >= k) break;
      }
    }
    ps->best.drain_best(total);
    ps->computed = cand;
    ps->next = 0;
    const size_t leftover = std::min<size_t>(k - n, cand.size());
    for (size_t i = 0; i < leftover; ++i) {
      ids_out[n] = cand[i].first;
      dists_out[n++] = cand[i].second;
    }
    ps->next = leftover;
  }
  *count_out = n;
  if (stats) {
    stats->cmps = ps->cmps;
    stats->hops = ps->hops;
    stats->result_count = n;
    stats->flags = 0;
  }
  return ORC_OK;
}

extern "C" void orc_paged_destroy(orc_paged* ps) { delete ps; }

// One k-NN search.
//
// diskann/src/graph/search/knn_search.rs:178-216 `<Knn as Search>::search`: the queue
// capacity is L + #start points (scratch.rs:199-207, index.rs:178-189), the loop is
// `search_internal` (index.rs:1938-2005) and the default post-processor is applied to
// the first min(search_l, size) queue entries.
//
//   strategy FULL_PRECISION: FullAccessor (inmem/full_precision.rs:251-322), post
//     process FilterStartPoints + copy (full_precision.rs:497-506, glue.rs:730-773).
//   strategy HYBRID: QuantAccessor (inmem/product.rs:267-336) PQ traversal, post process
//     FilterStartPoints + Rerank (product.rs:386-394, full_precision.rs:357-404).
//   strategy QUANTIZED: PQ traversal, FilterStartPoints + copy (product.rs:537-566).
//
// Rerank sorts with `sort_unstable_by` in the reference; this restatement uses a stable
// sort (equal full-precision distances keep queue order), which is one of the orders the
// reference may produce.  The reference's comparator calls a NaN equal to everything, which
// leaves a NaN's place unspecified; here NaN distances sort after every number, in queue order.
extern "C" int32_t orc_search(const orc_index* ix, int32_t strategy, const float* query,
                              uint32_t k, uint32_t l, uint32_t beam_width, uint32_t* ids_out,
                              float* dists_out, orc_stats* stats) {
  const int32_t verr = orc_validate_knn(k, l, beam_width);
  if (verr != ORC_OK) return verr;
  const bool pq = strategy == ORC_STRATEGY_HYBRID || strategy == ORC_STRATEGY_QUANTIZED;
  if (pq && ix->pq_chunks == 0) return ORC_ERR_NO_PQ;

  Scorer score{ix, query, pq, {}};
  if (pq && ix->metric != ORC_METRIC_COSINE) pq_table(ix, query, score.table);

  const uint32_t n_start = ix->num_frozen;
  Queue best((size_t)l + n_start);
  VisitedSet visited((size_t)std::ceil(1.1 * ix->max_degree * 1.3 * l));
  uint32_t cmps = 0, hops = 0;

  // search_internal: start points (index.rs:1956-1963).
  for (uint32_t s = 0; s < n_start; ++s) {
    const uint32_t id = ix->num_points + s;
    const float d = score(id);
    visited.insert(id);
    best.insert(id, d);
    cmps += 1;
  }

  search_loop(ix, score, best, visited, beam_width, cmps, hops);

  // Post-processing over the first min(search_l, size) candidates.
  const size_t n_cand = best.iter_len();
  uint32_t count = 0;
  if (strategy == ORC_STRATEGY_HYBRID) {
    std::vector<std::pair<uint32_t, float>> rr;
    rr.reserve(n_cand);
    for (size_t i = 0; i < n_cand; ++i) {
      const uint32_t id = best.ids[i];
      if (id >= ix->num_points) continue;  // FilterStartPoints
      rr.emplace_back(id, orc_distance(ix->metric, query, vec_row(ix, id), ix->dim));
    }
    std::stable_sort(rr.begin(), rr.end(), [](const auto& a, const auto& b) {
      const bool an = std::isnan(a.second), bn = std::isnan(b.second);
      return an != bn ? bn : (!an && a.second < b.second);
    });
    for (size_t i = 0; i < rr.size() && count < k; ++i, ++count) {
      ids_out[count] = rr[i].first;
      dists_out[count] = rr[i].second;
    }
  } else {
    for (size_t i = 0; i < n_cand && count < k; ++i) {
      const uint32_t id = best.ids[i];
      if (id >= ix->num_points) continue;  // FilterStartPoints
      ids_out[count] = id;
      dists_out[count] = best.dists[i];
      ++count;
    }
  }
  for (uint32_t i = count; i < k; ++i) {
    ids_out[i] = ORC_INVALID_ID;
    dists_out[i] = INFINITY;
  }
  if (stats) {
    stats->cmps = cmps;
    stats->hops = hops;
    stats->result_count = count;
    stats->flags = 0;
  }
  return ORC_OK;
}

// diskann-inmem provider search (diskann-inmem/src/provider.rs:380-960).  Rows are the store's
// slots: `dim` elements of `elem` then the one-byte tag (store.rs:150-260); a slot is
// readable when its tag is >= 254 (tag.rs Tag::can_read).  FP32 and FP16 data are scored by
// the FP32 restatement on the exact f32 values (the f32-by-f16 kernels, simd.rs:1121-1156,
// 1878-1912, 2716-2747, run Strategy4x2 / Strategy2x4, which feed each accumulator the same
// vectors in the same order as Strategy4x1 / Strategy2x4 over f32), so `ix->vectors` holds the
// converted rows and `query` f32 values.  u8 / i8 data are scored in exact integers
// (simd.rs:1192-1227, 1370-1405, 1947-1981, 2109-2145, 2790-2829, 2996-3035: i32 lanes, one
// lossy conversion to f32 per sum), `query` then holds `dim` bytes.
namespace {

struct IntScorer {
  const orc_index* ix;
  const uint8_t* rows;
  uint64_t row_stride;
  const uint8_t* query;
  bool is_signed;

  int64_t at(const uint8_t* p, uint32_t i) const {
    return is_signed ? (int64_t)(int8_t)p[i] : (int64_t)p[i];
  }
  float operator()(uint32_t id) const {
    const uint8_t* y = rows + (uint64_t)id * row_stride;
    int64_t xx = 0, yy = 0, xy = 0, l2 = 0;
    for (uint32_t i = 0; i < ix->dim; ++i) {
      const int64_t a = at(query, i), b = at(y, i);
      xx += a * a;
      yy += b * b;
      xy += a * b;
      l2 += (a - b) * (a - b);
    }
    // The i32 lanes wrap; the sums are converted with round-to-nearest-even.
    auto lossy = [](int64_t v) { return (float)(int32_t)(uint32_t)(uint64_t)v; };
    switch (ix->metric) {
      case ORC_METRIC_L2: return lossy(l2);
      case ORC_METRIC_INNER_PRODUCT: return -lossy(xy);
      default: {  // Cosine; the integer layers map CosineNormalized to Cosine
        const float nx = lossy(xx), ny = lossy(yy), pr = lossy(xy);
        const float denom = std::sqrt(nx) * std::sqrt(ny);
        if (nx < FLT_MIN || ny < FLT_MIN) return 1.0f;
        return 1.0f - std::max(-1.0f, std::min(1.0f, pr / denom));
      }
    }
  }
};

template <class Score>
int32_t inmem_search(const orc_index* ix, const uint8_t* rows, uint64_t row_stride,
                     uint32_t tag_offset, const uint64_t* ext, const Score& score, uint32_t k,
                     uint32_t l, uint32_t beam_width, uint64_t* ids_out, float* dists_out,
                     orc_stats* stats) {
  const int32_t verr = orc_validate_knn(k, l, beam_width);
  if (verr != ORC_OK) return verr;
  auto readable = [&](uint32_t id) { return rows[(uint64_t)id * row_stride + tag_offset] >= 254; };
  const uint32_t n_start = ix->num_frozen;
  Queue best((size_t)l + n_start);
  VisitedSet visited((size_t)std::ceil(1.1 * ix->max_degree * 1.3 * l));
  uint32_t cmps = 0, hops = 0;
  // start_point_distances (provider.rs:415-440): the frozen slots, always readable.
  for (uint32_t s = 0; s < n_start; ++s) {
    const uint32_t id = ix->num_points + s;
    visited.insert(id);
    best.insert(id, score(id));
    cmps += 1;
  }
  std::vector<uint32_t> beam;
  std::vector<std::pair<uint32_t, float>> neighbors;
  while (best.has_notvisited()) {
    beam.clear();
    uint32_t node;
    while (beam.size() < beam_width && best.closest_notvisited(&node)) beam.push_back(node);
    neighbors.clear();
    // expand_beam (provider.rs:443-478): retain(visited-set insert && in bounds), then score
    // the slots whose tag is readable, in order; the others stay visited.
    for (uint32_t n : beam) {
      const uint32_t deg = ix->degrees[n];
      const uint32_t* adj = ix->adjacency + (size_t)n * ix->adjacency_stride;
      for (uint32_t t = 0; t < deg; ++t) {
        const uint32_t id = adj[t];
        if (visited.insert(id) && readable(id)) neighbors.emplace_back(id, score(id));
      }
    }
    for (const auto& nb : neighbors) best.insert(nb.first, nb.second);
    cmps += (uint32_t)neighbors.size();
    hops += (uint32_t)beam.size();
  }
  // Translate (provider.rs:906-945): candidates with an external id, in order, up to k.
  uint32_t count = 0;
  for (size_t i = 0; i < best.iter_len() && count < k; ++i) {
    const uint64_t e = ext[best.ids[i]];
    if (e == ORC_NO_EXTERNAL_ID) continue;
    ids_out[count] = e;
    dists_out[count++] = best.dists[i];
  }
  for (uint32_t i = count; i < k; ++i) {
    ids_out[i] = ORC_NO_EXTERNAL_ID;
    dists_out[i] = INFINITY;
  }
  if (stats) {
    stats->cmps = cmps;
    stats->hops = hops;
    stats->result_count = count;
    stats->flags = 0;
  }
  return ORC_OK;
}

}  // namespace

extern "C" int32_t orc_inmem_search(const orc_index* ix, int32_t elem, const uint8_t* rows,
                                    uint64_t row_stride, const uint64_t* ext, const void* query,
                                    uint32_t k, uint32_t l, uint32_t beam_width,
                                    uint64_t* ids_out, float* dists_out, orc_stats* stats) {
  const uint32_t eb = elem == ORC_ELEM_F32 ? 4u : (elem == ORC_ELEM_F16 ? 2u : 1u);
  const uint32_t tag_offset = ix->dim * eb;
  if (elem == ORC_ELEM_U8 || elem == ORC_ELEM_I8) {
    const IntScorer score{ix, rows, row_stride, static_cast<const uint8_t*>(query), elem == ORC_ELEM_I8};
    return inmem_search(ix, rows, row_stride, tag_offset, ext, score, k, l, beam_width, ids_out,
                        dists_out, stats);
  }
  const Scorer score{ix, static_cast<const float*>(query), false, {}};
  return inmem_search(ix, rows, row_stride, tag_offset, ext, score, k, l, beam_width, ids_out,
                      dists_out, stats);
}

// Many queries on `num_threads` host threads.  Queries are split into contiguous ranges,
// one per thread, as the reference benchmark's task partitioning does
// (diskann/src/utils/async_tools.rs:311-351 PartitionIter).
extern "C" int32_t orc_search_batch(const orc_index* ix, int32_t strategy, const float* queries,
                                    uint32_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                                    uint32_t beam_width, uint32_t* ids_out, float* dists_out,
                                    orc_stats* stats, uint32_t num_threads) {
  const int32_t verr = orc_validate_knn(k, l, beam_width);
  if (verr != ORC_OK) return verr;
  if (num_threads == 0) num_threads = 1;
  if (num_threads > nq) num_threads = nq > 0 ? nq : 1;
  std::atomic<int32_t> status{ORC_OK};
  auto work = [&](uint32_t t) {
    const uint64_t lo = (uint64_t)nq * t / num_threads, hi = (uint64_t)nq * (t + 1) / num_threads;
    for (uint64_t i = lo; i < hi; ++i) {
      const int32_t rc = orc_search(ix, strategy, queries + i * query_stride, k, l, beam_width,
                                    ids_out + i * k, dists_out + i * k, stats ? stats + i : nullptr);
      if (rc != ORC_OK) status.store(rc);
    }
  };
  if (num_threads == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    pool.reserve(num_threads);
    for (uint32_t t = 0; t < num_threads; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  return status.load();
}

// Brute-force exact k-NN in float64 (the ground-truth restatement used to check the GPU
// ground-truth kernel on small cases).  Distances follow the metric definitions above but
// in double precision with a plain sequential sum.  Ties are broken by smaller id.
extern "C" void orc_bruteforce_f64(const float* base, uint32_t n, uint32_t dim, uint32_t stride,
                                   const float* queries, uint32_t nq, uint32_t k, int32_t metric,
                                   uint32_t* ids_out, double* dists_out) {
  std::vector<std::pair<double, uint32_t>> all(n);
  for (uint32_t qi = 0; qi < nq; ++qi) {
    const float* q = queries + (size_t)qi * dim;
    double qq = 0.0;
    for (uint32_t d = 0; d < dim; ++d) qq += (double)q[d] * q[d];
    for (uint32_t i = 0; i < n; ++i) {
      const float* x = base + (size_t)i * stride;
      double acc = 0.0, xx = 0.0;
      for (uint32_t d = 0; d < dim; ++d) {
        if (metric == ORC_METRIC_L2) {
          const double c = (double)q[d] - (double)x[d];
          acc += c * c;
        } else {
          acc += (double)q[d] * x[d];
          xx += (double)x[d] * x[d];
        }
      }
      double v;
      if (metric == ORC_METRIC_L2) v = acc;
      else if (metric == ORC_METRIC_INNER_PRODUCT) v = -acc;
      else if (metric == ORC_METRIC_COSINE_NORMALIZED) v = 1.0 - acc;
      else v = (qq > 0 && xx > 0) ? 1.0 - acc / (std::sqrt(qq) * std::sqrt(xx)) : 1.0;
      all[i] = {v, i};
    }
    const uint32_t kk = std::min(k, n);
    std::partial_sort(all.begin(), all.begin() + kk, all.end());
    for (uint32_t j = 0; j < k; ++j) {
      ids_out[(size_t)qi * k + j] = j < kk ? all[j].second : ORC_INVALID_ID;
      dists_out[(size_t)qi * k + j] = j < kk ? all[j].first : INFINITY;
    }
  }
}

// PQ lookup table for one query, exposed for table-level checks.
extern "C" void orc_pq_table(const orc_index* ix, const float* query, float* table_out) {
  std::vector<float> t;
  pq_table(ix, query, t);
  std::memcpy(table_out, t.data(), t.size() * sizeof(float));
}
