// ORACLE — TEST INFRASTRUCTURE ONLY (see oracle.cpp for what this restates).
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

// Metric codes follow the reference's i32 encoding
// (diskann-vector/src/distance/metric.rs:34-52).
enum {
  ORC_METRIC_COSINE = 0,
  ORC_METRIC_INNER_PRODUCT = 1,
  ORC_METRIC_L2 = 2,
  ORC_METRIC_COSINE_NORMALIZED = 3,
};

enum {
  ORC_STRATEGY_FULL_PRECISION = 0,
  ORC_STRATEGY_HYBRID = 1,
  ORC_STRATEGY_QUANTIZED = 2,
};

enum {
  ORC_OK = 0,
  ORC_ERR_K_ZERO = 1,
  ORC_ERR_L_ZERO = 2,
  ORC_ERR_L_LESS_THAN_K = 3,
  ORC_ERR_BEAM_WIDTH_ZERO = 4,
  ORC_ERR_NO_PQ = 5,
  ORC_ERR_INVALID_ARGUMENT = 6,
};

#define ORC_INVALID_ID 0xFFFFFFFFu
#define ORC_NO_EXTERNAL_ID 0xFFFFFFFFFFFFFFFFull

enum { ORC_ELEM_F32 = 0, ORC_ELEM_F16 = 1, ORC_ELEM_U8 = 2, ORC_ELEM_I8 = 3 };

// An in-memory index: ids 0..num_points-1 are data, num_points..num_points+num_frozen-1
// are frozen start points.  All arrays have num_points + num_frozen rows.
typedef struct orc_index {
  uint32_t num_points;
  uint32_t num_frozen;
  uint32_t dim;
  int32_t metric;
  const float* vectors;        // rows of `vector_stride` floats
  uint32_t vector_stride;
  const uint32_t* adjacency;   // rows of `adjacency_stride` ids
  const uint32_t* degrees;     // adjacency list lengths
  uint32_t adjacency_stride;
  uint32_t max_degree;
  uint32_t pq_chunks;          // 0 when no PQ
  const uint32_t* pq_offsets;  // pq_chunks + 1 dimension offsets
  const float* pq_pivots;      // 256 x dim
  const uint8_t* pq_codes;     // rows of `pq_code_stride` bytes
  uint32_t pq_code_stride;
} orc_index;

typedef struct orc_stats {
  uint32_t cmps;
  uint32_t hops;
  uint32_t result_count;
  uint32_t flags;
} orc_stats;

float orc_distance(int32_t metric, const float* x, const float* y, uint32_t len);
int32_t orc_validate_knn(uint32_t k, uint32_t l, uint32_t beam_width);
int32_t orc_search(const orc_index* ix, int32_t strategy, const float* query, uint32_t k,
                   uint32_t l, uint32_t beam_width, uint32_t* ids_out, float* dists_out,
                   orc_stats* stats);
int32_t orc_inmem_search(const orc_index* ix, int32_t elem, const uint8_t* rows,
                         uint64_t row_stride, const uint64_t* ext, const void* query, uint32_t k,
                         uint32_t l, uint32_t beam_width, uint64_t* ids_out, float* dists_out,
                         orc_stats* stats);
typedef struct orc_paged orc_paged;
int32_t orc_paged_create(const orc_index* ix, const float* query, uint32_t l_value,
                         const uint32_t* init_ids, uint32_t n_init, orc_paged** out);
int32_t orc_paged_next(orc_paged* ps, uint32_t k, uint32_t* ids_out, float* dists_out,
                       uint32_t* count_out, orc_stats* stats);
void orc_paged_destroy(orc_paged* ps);
int32_t orc_range_search(const orc_index* ix, const float* query, uint32_t starting_l,
                         uint32_t beam_width, float radius, float inner_radius,
                         float initial_slack, float range_slack, uint32_t max_returned,
                         uint32_t capacity, uint32_t* ids_out, float* dists_out, orc_stats* stats);
int32_t orc_search_batch(const orc_index* ix, int32_t strategy, const float* queries,
                         uint32_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                         uint32_t beam_width, uint32_t* ids_out, float* dists_out,
                         orc_stats* stats, uint32_t num_threads);
void orc_bruteforce_f64(const float* base, uint32_t n, uint32_t dim, uint32_t stride,
                        const float* queries, uint32_t nq, uint32_t k, int32_t metric,
                        uint32_t* ids_out, double* dists_out);
void orc_pq_table(const orc_index* ix, const float* query, float* table_out);

// Graph construction (build.cpp): the reference's insert rules with a deterministic batch
// schedule; ids num_points.. are the frozen start points (their vectors must be set).
typedef struct orc_build_params {
  uint32_t pruned_degree;  // R
  uint32_t max_degree;     // slot width (list length allowed before a back edge prunes)
  uint32_t l_build;
  float alpha;
  uint32_t max_backedges;
  uint32_t max_occlusion;  // 0 = 750
  uint32_t num_threads;    // 0 = all hardware threads
  uint32_t max_batch;      // 0 = max(64, num_points / 64)
} orc_build_params;
int32_t orc_build_vamana(const float* vectors, uint32_t vector_stride, uint32_t num_points,
                         uint32_t num_frozen, uint32_t dim, int32_t metric,
                         const orc_build_params* params, uint32_t* adjacency,
                         uint32_t adjacency_stride, uint32_t* degrees);
uint32_t orc_medoid(const float* vectors, uint32_t stride, uint32_t n, uint32_t dim);

#ifdef __cplusplus
}
#endif
