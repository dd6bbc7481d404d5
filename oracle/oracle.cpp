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
    if (size == capacity && dists[size - 1] < d) return;
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
// reference may produce.
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
      return a.second < b.second;
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
