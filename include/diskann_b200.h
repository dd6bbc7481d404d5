/*
 * diskann_b200 — C ABI of the B200 in-memory graph-search engine.
 *
 * This is the drop-in boundary for the reference's in-memory search call.  In the
 * reference (a Rust workspace) a search is
 *
 *     DiskANNIndex::search(Knn::new(k, l, beam)?, &strategy, &ctx, query, &mut output)
 *       diskann/src/graph/index.rs:2034-2070  ->  <Knn as Search>::search
 *       diskann/src/graph/search/knn_search.rs:178-216
 *
 * run against an in-memory `DefaultProvider` (diskann-providers/src/model/graph/provider/
 * async_/inmem/provider.rs:227-352) with one of the strategies `FullPrecision`
 * (inmem/full_precision.rs:476-506), `Hybrid` (inmem/product.rs:363-394) or `Quantized`
 * (inmem/product.rs:537-566).  The per-hop `SearchAccessor::expand_beam` callback
 * (diskann/src/graph/glue.rs:125-254) is far too fine-grained to cross into a GPU, so the
 * boundary sits at `Search::search` granularity and is batched: one call searches many
 * queries.  The reference's own C FFI precedent is diskann-garnet/src/lib.rs:218-807
 * (plain `extern "C"` functions over raw pointers and sizes, integer status codes).
 *
 * Conventions
 *  - Every function returns an int32_t status (DK_OK == 0).  `dk_last_error` gives the
 *    calling thread's last error message.
 *  - Ids 0..num_points-1 are data points; ids num_points..num_points+num_frozen-1 are the
 *    frozen start points (inmem/provider.rs:312-319), which are searched from and filtered
 *    out of results (diskann/src/graph/glue.rs:730-773 FilterStartPoints).
 *  - Output buffers are caller-allocated, k entries per query (the reference's
 *    caller-allocated `SearchOutputBuffer`, diskann/src/graph/search_output_buffer.rs:100-140).
 *    Entries past a query's result_count are id 0xFFFFFFFF, distance +inf.
 *  - Thread safety: create/destroy are exclusive; search calls on one index are safe from
 *    several host threads and streams at once (the index is read-only after creation).
 */
#ifndef DISKANN_B200_H
#define DISKANN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DK_ABI_VERSION 1
#define DK_INVALID_ID 0xFFFFFFFFu

/* Metric codes are the reference's i32 encoding (diskann-vector/src/distance/metric.rs:34-52). */
enum dk_metric {
  DK_METRIC_COSINE = 0,
  DK_METRIC_INNER_PRODUCT = 1,
  DK_METRIC_L2 = 2,
  DK_METRIC_COSINE_NORMALIZED = 3,
};

/* Search strategies (the reference's strategy types and their default post-processors). */
enum dk_strategy {
  DK_STRATEGY_FULL_PRECISION = 0, /* FullPrecision: FP32 traversal, FilterStartPoints + copy */
  DK_STRATEGY_HYBRID = 1,         /* Hybrid: PQ traversal, FilterStartPoints + FP32 Rerank  */
  DK_STRATEGY_QUANTIZED = 2,      /* Quantized: PQ traversal, FilterStartPoints + copy      */
  /* Hybrid-style strategies over low-precision copies of the vectors (no counterpart in the
   * reference): candidates are scored from BF16 rows, or from FP8-E4M3 rows with one FP32
   * scale per vector, accumulating in FP32; the queue is then re-ranked with exact FP32
   * distances (the reference's Rerank, inmem/full_precision.rs:357-404).
   * Rerank order, every reranking strategy: ascending exact distance, ties in queue order, NaN
   * distances (rows holding a NaN) after every number, in queue order. */
  DK_STRATEGY_BF16 = 3,
  DK_STRATEGY_FP8 = 4,
};

/* dk_index_desc.flags: which low-precision copies dk_index_create derives from `vectors`. */
#define DK_INDEX_BF16 1u
#define DK_INDEX_FP8 2u

/* Status codes.  1..4 mirror `KnnSearchError` (diskann/src/graph/search/knn_search.rs:39-44). */
enum dk_status {
  DK_OK = 0,
  DK_ERR_K_ZERO = 1,
  DK_ERR_L_ZERO = 2,
  DK_ERR_L_LESS_THAN_K = 3,
  DK_ERR_BEAM_WIDTH_ZERO = 4,
  DK_ERR_NO_PQ = 5,              /* PQ strategy on an index created without PQ data */
  DK_ERR_INVALID_ARGUMENT = 6,   /* null pointer, zero dimension, unsupported size */
  DK_ERR_INVALID_GRAPH = 7,      /* neighbour id out of range or degree above max_degree */
  DK_ERR_DIMENSION_MISMATCH = 8,
  DK_ERR_OUT_OF_MEMORY = 9,
  DK_ERR_CUDA = 10,
  DK_ERR_DEVICE_TIMEOUT = 11,    /* a bounded device-side wait gave up */
  DK_ERR_UNSUPPORTED = 12,
  DK_ERR_ADMISSION = 13,         /* serving loop: request rejected (no slot / memory) */
  DK_ERR_CANCELLED = 14,
  DK_ERR_NOT_FOUND = 15,
  DK_ERR_NO_LOW_PRECISION = 16,  /* BF16/FP8 strategy on an index created without that copy */
  DK_ERR_NOT_READY = 17,         /* serving: the request has not completed yet */
};

/* Per-query statistics: the reference's `SearchStats` (diskann/src/graph/index.rs:90-102). */
typedef struct dk_search_stats {
  uint32_t cmps;         /* distance computations, start points included */
  uint32_t hops;         /* expanded nodes */
  uint32_t result_count; /* results written (<= k) */
  uint32_t flags;        /* internal: bit 0 = visited set spilled to the global-memory pass */
} dk_search_stats;

/* Host-side description of an in-memory index.  All arrays are host memory with
 * num_points + num_frozen rows; dk_index_create copies them to device memory and the
 * caller keeps ownership. */
typedef struct dk_index_desc {
  uint32_t num_points;        /* N data points */
  uint32_t num_frozen;        /* F >= 1 frozen start points, ids N..N+F-1 */
  uint32_t dim;               /* D */
  int32_t metric;             /* enum dk_metric */
  const float* vectors;       /* (N+F) rows of `vector_stride` floats; first D used */
  uint64_t vector_stride;
  const uint32_t* adjacency;  /* (N+F) rows of `adjacency_stride` ids */
  uint64_t adjacency_stride;
  const uint32_t* degrees;    /* (N+F) list lengths, each <= max_degree */
  uint32_t max_degree;        /* adjacency slot width (the reference's max_degree with slack) */
  /* Optional product quantisation (pq_chunks == 0: none).  Layout of the reference's
   * FixedChunkPQTable (diskann-providers/src/model/pq/fixed_chunk_pq_table.rs:100-133). */
  uint32_t pq_chunks;         /* M */
  const uint32_t* pq_offsets; /* M+1 dimension offsets, 0 .. D, strictly increasing */
  const float* pq_pivots;     /* 256 x D, row-major */
  const uint8_t* pq_codes;    /* (N+F) rows of `pq_code_stride` bytes, first M used */
  uint64_t pq_code_stride;
  uint32_t flags;             /* DK_INDEX_BF16 | DK_INDEX_FP8 */
} dk_index_desc;

typedef struct dk_index dk_index;

typedef struct dk_index_info {
  uint32_t num_points, num_frozen, dim, max_degree, pq_chunks;
  int32_t metric;
  int32_t device;
  uint64_t device_bytes;       /* HBM held by the index */
} dk_index_info;

/* Library ABI version (DK_ABI_VERSION). */
int32_t dk_abi_version(void);

/* Message of the calling thread's most recent error (NUL-terminated, truncated to len).
 * Returns the status that produced it. */
int32_t dk_last_error(char* buf, uint64_t len);

/* `Knn::new` validation (diskann/src/graph/search/knn_search.rs:94-119). */
int32_t dk_knn_validate(uint32_t k, uint32_t l, uint32_t beam_width);

/* Build a device-resident index from host arrays (replaces constructing a
 * `DefaultProvider` + `DiskANNIndex`, inmem/provider.rs:301-352 and index.rs:59-66). */
int32_t dk_index_create(const dk_index_desc* desc, int32_t device, dk_index** out);
int32_t dk_index_destroy(dk_index* index);
int32_t dk_index_get_info(const dk_index* index, dk_index_info* info);

/* Batched k-NN search with HOST buffers: copies the queries in, searches, copies results
 * out and returns when they are in `ids`, `dists`, `stats` (stats may be NULL).
 * Replaces `nq` calls of DiskANNIndex::search with Knn{k, l, beam_width}
 * (diskann/src/graph/index.rs:2034-2070). */
int32_t dk_search(dk_index* index, int32_t strategy, const float* queries, uint64_t query_stride,
                  uint32_t nq, uint32_t k, uint32_t l, uint32_t beam_width, uint32_t* ids,
                  float* dists, dk_search_stats* stats);

/* Same search with DEVICE buffers, asynchronous on `stream` (a cudaStream_t; NULL = the
 * legacy default stream).  `stats` is required here: the visited-set spill pass reads it. */
int32_t dk_search_device(dk_index* index, int32_t strategy, const float* queries,
                         uint64_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                         uint32_t beam_width, uint32_t* ids, float* dists,
                         dk_search_stats* stats, void* stream);

/* The distance each strategy scores a candidate with, for `nq` queries (rows of
 * `query_stride` floats) and `per_query` candidate ids each (row-major, nq x per_query),
 * written to `dists` (same shape).  DEVICE buffers, asynchronous on `stream`.  This is the
 * accessor's per-candidate distance, batched (replaces the preprocessed query distance of
 * diskann/src/utils/vector_repr.rs:48-93 for FullPrecision, bit-exact; the PQ QueryComputer of
 * diskann-providers/src/model/pq/distance/dynamic.rs:64-84 for Hybrid / Quantized; for BF16 /
 * FP8, which have no counterpart in the reference, the low-precision distance their traversal
 * uses).  An id outside the index scores NaN. */
int32_t dk_score_candidates(dk_index* index, int32_t strategy, const float* queries,
                            uint64_t query_stride, uint32_t nq, const uint32_t* ids,
                            uint32_t per_query, float* dists, void* stream);

/* Range search with the FullPrecision strategy (replaces DiskANNIndex::search with the
 * reference's `Range` parameters, diskann/src/graph/search/range_search.rs:63-389): a first
 * greedy search with a queue of starting_l + F entries, then - when at least
 * (starting_l * initial_slack) of its first starting_l entries lie within `radius` and fewer
 * than max_returned - a breadth-first second round from them that adds every neighbour within
 * radius * range_slack; results are the start-point-free entries with
 * inner_radius < distance <= radius, in the reference's order.  inner_radius NaN = none;
 * max_returned 0 = unlimited.  Each query gets `capacity` (>= starting_l, >= max_returned) output
 * slots: result_count in stats says how many are filled (this host entry point copies back the
 * filled slots only and leaves the rest of each row unspecified; the device entry point pads
 * them with id 0xFFFFFFFF, distance +inf); with max_returned unlimited, flags
 * bit 2 marks a query whose results reached the capacity (possibly incomplete); flags bit 1:
 * the second round ran.  Stats follow the reference (cmps of the first round; with a second
 * round, hops counts the first round twice, as the reference's scratch counter does). */
int32_t dk_range_search(dk_index* index, const float* queries, uint64_t query_stride,
                        uint32_t nq, uint32_t starting_l, uint32_t beam_width, float radius,
                        float inner_radius, float initial_slack, float range_slack,
                        uint32_t max_returned, uint32_t capacity, uint32_t* ids, float* dists,
                        dk_search_stats* stats);
/* The same with device buffers, asynchronous on `stream`; `stats` is required. */
int32_t dk_range_search_device(dk_index* index, const float* queries, uint64_t query_stride,
                               uint32_t nq, uint32_t starting_l, uint32_t beam_width,
                               float radius, float inner_radius, float initial_slack,
                               float range_slack, uint32_t max_returned, uint32_t capacity,
                               uint32_t* ids, float* dists, dk_search_stats* stats, void* stream);

/* Paged search with the FullPrecision strategy, one session per query of a batch.
 * dk_paged_search_create replaces DiskANNIndex::paged_search / paged_search_with_init_ids
 * (diskann/src/graph/index.rs:2080-2160): the init ids (init_ids = NULL / n_init = 0: the start
 * points; else n_init ids per query, row-major) enter the visited set and their neighbours
 * seed a queue that keeps every scored id (the reference's resizable queue; search window
 * l_value + F).  dk_paged_search_next replaces PagedSearch::next_page
 * (diskann/src/graph/search/paged.rs:52-151) for every session at once: up to k results per
 * session (ids / dists: nq x k host arrays; result_count in stats says how many, 0 once the
 * session is exhausted), resuming the search where the previous page stopped; pages never
 * repeat an id.  Errors: k == 0 or k > l_value -> DK_ERR_INVALID_ARGUMENT (the reference's
 * paged-search error).  stats carry each session's running comparison and hop counts.  The
 * queue holds queue_capacity entries per session (0 = N + F, which can never fill); a session
 * whose queue filled keeps its best entries and reports flags bit 2.  Device memory per
 * session: 8 * queue_capacity + (N + F) / 8 + 16 * l_value bytes, plus the query. */
typedef struct dk_paged dk_paged;
int32_t dk_paged_search_create(dk_index* index, const float* queries, uint64_t query_stride,
                               uint32_t nq, uint32_t l_value, const uint32_t* init_ids,
                               uint32_t n_init, uint32_t queue_capacity, dk_paged** out);
int32_t dk_paged_search_next(dk_paged* search, uint32_t k, uint32_t* ids, float* dists,
                             dk_search_stats* stats);
int32_t dk_paged_search_destroy(dk_paged* search);

/* The diskann-inmem provider (diskann-inmem/src/provider.rs), its store and search.
 *
 * dk_inmem_index_create replaces diskann_inmem::Provider::new plus the inserts that filled it:
 * it takes the provider's store as it lies in memory - one slot of `row_stride` bytes per id,
 * `dim` elements of `elem` followed by the one-byte concurrency tag (store.rs:150-260; the
 * frozen start points are the last `num_frozen` slots, store.rs:248-251) - its adjacency
 * lists and, per slot, the external id (ids.rs IdMap; DK_NO_EXTERNAL_ID: no mapping, as for
 * the frozen slots and deleted or empty ones).  A slot is readable when its tag is PUBLISHED
 * (254) or FROZEN (255) (tag.rs Tag::can_read); every frozen slot must be.
 *
 * dk_inmem_search replaces DiskANNIndex::search with the provider's Strategy and default
 * post-processor (provider.rs:855-960): the search loop of dk_search where a neighbour whose
 * slot is not readable enters the visited set but is not scored (provider.rs:451-473), and
 * results are the queue's entries that have an external id, in order, translated (Translate,
 * provider.rs:906-945); `ids` receives the external ids.  Queries are `elem` values
 * (query_stride in elements); f16 data is searched with f32 queries converted from f16, as
 * the f16 layer does (layers/full.rs:404-437).  u8 / i8 with CosineNormalized use cosine, as
 * the layers do.  Host buffers; returns when the results are written.
 * dk_inmem_set_tags updates the tags of slots [first, first + count) (deletes, inserts). */
enum dk_elem { DK_ELEM_F32 = 0, DK_ELEM_F16 = 1, DK_ELEM_U8 = 2, DK_ELEM_I8 = 3 };
#define DK_NO_EXTERNAL_ID 0xFFFFFFFFFFFFFFFFull
typedef struct dk_inmem_desc {
  uint32_t capacity;          /* data slots 0..capacity-1 (the provider's Config::capacity) */
  uint32_t num_frozen;        /* start points: slots capacity..capacity+num_frozen-1 */
  uint32_t dim;
  int32_t metric;             /* enum dk_metric */
  int32_t elem;               /* enum dk_elem */
  const uint8_t* rows;        /* (capacity + num_frozen) slots of row_stride bytes */
  uint64_t row_stride;        /* >= dim * element size + 1 */
  const uint32_t* adjacency;  /* (capacity + num_frozen) rows of adjacency_stride ids */
  uint64_t adjacency_stride;
  const uint32_t* degrees;
  uint32_t max_degree;
  const uint64_t* external_ids; /* per slot */
} dk_inmem_desc;
int32_t dk_inmem_index_create(const dk_inmem_desc* desc, int32_t device, dk_index** out);
int32_t dk_inmem_set_tags(dk_index* index, uint32_t first, uint32_t count, const uint8_t* tags);
int32_t dk_inmem_search(dk_index* index, const void* queries, uint64_t query_stride, uint32_t nq,
                        uint32_t k, uint32_t l, uint32_t beam_width, uint64_t* ids, float* dists,
                        dk_search_stats* stats);

/* Same search, arguments and results as dk_search_device, for callers that cannot allocate
 * device memory while they search: for example a process whose own caching allocator took the
 * GPU's free memory at start-up (so the allocation inside dk_search_device would fail), or a
 * latency-critical path that must not enter the CUDA allocator.  This entry point allocates
 * nothing: its scratch (work counter, per-warp visited tables, spill bitmaps) comes from one
 * fixed device array of DK_NOALLOC_SCRATCH_BYTES that the library declares statically, which
 * every GPU that loads the library holds until the process exits.  No counterpart in the
 * reference.
 *  - Set-up: the first call on a device, made with that device current, looks up the array's
 *    device address; make that first call (nq = 0 is enough) before any stream capture.  With
 *    CUDA's lazy module loading the array's memory is committed by that look-up, so make the
 *    set-up call before your own allocator reserves the GPU's memory; a set-up that finds no
 *    room returns DK_ERR_CUDA (out of memory).
 *  - Visited tables are sized from the index's visited-size estimate, which only
 *    dk_search_device calls update; this entry point reads it and never changes it.
 *  - The spill pass (queries whose visited set outgrows the tables) runs at most one CTA per
 *    SM here, against up to eight in dk_search_device, so spill-heavy batches run slower.
 *  - Limit: a search whose scratch would not fit the array (one spill bitmap of (N+F)/8
 *    bytes plus one CTA's visited tables at least) is refused with DK_ERR_UNSUPPORTED and a
 *    message giving the bytes it needs; large batches run with fewer warps when not all of
 *    their tables fit.
 *  - Every call on a device shares the array and it keeps the last call's contents; each call
 *    clears what must start at zero.  Calls whose work overlaps on the GPU race on the array:
 *    issue them on one stream, or let one finish before the next starts. */
#define DK_NOALLOC_SCRATCH_BYTES (32u << 20)
int32_t dk_search_device_noalloc(dk_index* index, int32_t strategy, const float* queries,
                                 uint64_t query_stride, uint32_t nq, uint32_t k, uint32_t l,
                                 uint32_t beam_width, uint32_t* ids, float* dists,
                                 dk_search_stats* stats, void* stream);


/* ---- Serving: continuous admission of single requests (no counterpart in the reference,
 * whose searches are one async call per query scheduled by the caller's runtime) ----
 *
 * dk_server_submit queues one request (its own k and L, up to max_k / max_l) and returns a
 * ticket.  Queued requests are launched as soon as one of the server's `streams` launch
 * contexts is free: a request that arrives while others are on the GPU goes out in the next
 * launch on another stream, and the launches overlap on the device (each a warp-per-request
 * search whose beam state and visited set stay in shared memory and HBM for the whole
 * search).  Requests that arrive while every context is busy are launched together when the
 * first one frees up.  dk_server_poll returns DK_OK once the request's results are in the
 * caller's buffers, else DK_ERR_NOT_READY; polling also reaps finished launches and starts
 * queued ones.  Admission: a submit is rejected with DK_ERR_ADMISSION while queue_depth
 * requests are outstanding (submitted, not yet collected), or when the device memory its
 * beam state needs at its own L (a double-buffered queue of L + F entries and a visited table
 * for the expected visited set) does not fit the server's beam-state memory beside the
 * reservations of the requests outstanding; a larger L therefore takes more of it.  All device memory (per-context
 * query, result and visited-table buffers) is taken at creation, sized from max_l, the
 * contexts' slots and the free device memory; no device code waits on the host.
 * A server's calls are serialised by an internal lock. */
typedef struct dk_server dk_server;

typedef struct dk_server_config {
  int32_t strategy;      /* enum dk_strategy, for every request */
  uint32_t max_k;        /* per-request k <= max_k */
  uint32_t max_l;        /* per-request L <= max_l */
  uint32_t beam_width;   /* for every request (<= 4) */
  uint32_t queue_depth;  /* outstanding requests accepted */
  uint32_t max_slots;    /* concurrent searches per launch (0 = all resident warps) */
  uint32_t streams;      /* launch contexts that overlap on the device (0 = 16) */
  uint32_t pad;
  uint64_t memory_bytes; /* device memory for beam state that admission fills (0 = the
                            visited tables the server allocates) */
} dk_server_config;

typedef struct dk_server_info {
  uint32_t slots;            /* concurrent searches per launch */
  uint32_t queue_depth;
  uint32_t streams;
  uint32_t pad;
  uint64_t device_bytes;     /* HBM held by the server */
  uint64_t launches;         /* kernel launches so far */
  uint64_t memory_bytes;     /* device memory for beam state (admission budget) */
  uint64_t reserved_bytes;   /* reserved by the outstanding requests now */
} dk_server_info;

int32_t dk_server_create(dk_index* index, const dk_server_config* config, dk_server** out);
int32_t dk_server_submit(dk_server* server, const float* query, uint32_t k, uint32_t l,
                         uint64_t* ticket);
int32_t dk_server_poll(dk_server* server, uint64_t ticket, uint32_t* ids, float* dists,
                       dk_search_stats* stats);
/* Cancel an outstanding request (the serving analogue of dropping the reference's search
 * future; its errors rank a cancellation as transient, diskann/src/error/ranked.rs:91-159):
 * a queued request never reaches the device; one already on the device finishes its launch
 * and its results are dropped.  The next dk_server_poll of the ticket returns
 * DK_ERR_CANCELLED and frees its slot and memory reservation; the server stays usable.
 * DK_ERR_NOT_FOUND for an unknown or collected ticket. */
int32_t dk_server_cancel(dk_server* server, uint64_t ticket);
/* Load-test driver (no counterpart in the reference; the role of its benchmark runner): replay
 * a request stream through the server from the calling host thread.  Request i uses query row
 * i % nq, k[i] and L[i], and is submitted arrival_ns[i] nanoseconds after the call starts (not
 * decreasing; a request that finds queue_depth requests outstanding waits for admission);
 * latency_ns[i] = when the calling thread sees its results - arrival_ns[i].  ids / dists (may
 * be NULL) receive n x max_k entries.  The thread spins between events; returns when every
 * request is done. */
int32_t dk_server_replay(dk_server* server, const float* queries, uint64_t query_stride,
                         uint32_t nq, const uint32_t* k, const uint32_t* l,
                         const uint64_t* arrival_ns, uint32_t n, uint64_t* latency_ns,
                         uint32_t* ids, float* dists);
int32_t dk_server_get_info(const dk_server* server, dk_server_info* info);
int32_t dk_server_destroy(dk_server* server);

/* ---- Data tooling on either side of the search path (host code, no GPU needed) ---- */

/* Distance with the reference's float rounding sequence (x86-64-v3 kernels,
 * diskann-vector/src/distance/simd.rs:321-363, 686-846; post-ops implementations.rs:215-405). */
int32_t dk_distance(int32_t metric, const float* x, const float* y, uint32_t len, float* out);

/* Medoid start point: index of the first row nearest (squared L2) to the f64 mean
 * (diskann-utils/src/sampling/medoid.rs:15-45). */
int32_t dk_compute_medoid(const float* vectors, uint64_t stride, uint32_t n, uint32_t dim,
                          uint32_t* medoid);

/* Vamana construction parameters (diskann/src/graph/config/mod.rs:182-331; defaults in
 * config/defaults.rs: alpha 1.2, max_occlusion 750). */
typedef struct dk_build_params {
  uint32_t pruned_degree;  /* R */
  uint32_t max_degree;     /* slot width, floor(1.3 R) in the reference benchmark */
  uint32_t l_build;
  float alpha;
  uint32_t max_backedges;  /* ceil(backedge_ratio * R) */
  uint32_t max_occlusion;  /* 0 = 750 */
  uint32_t num_threads;    /* 0 = all hardware threads */
  uint32_t max_batch;      /* 0 = max(64, N / 64) */
} dk_build_params;

/* Build a Vamana graph over `vectors` ((num_points + num_frozen) rows; the frozen rows are
 * the start points) by deterministic batched insertion (insert / occlude_list /
 * add_edge_and_prune, diskann/src/graph/index.rs:226-341, 2269-2346, 2570-2782).  Writes
 * (N+F) rows of `adjacency_stride` ids and their lengths. */
int32_t dk_build_vamana(const float* vectors, uint64_t stride, uint32_t num_points,
                        uint32_t num_frozen, uint32_t dim, int32_t metric,
                        const dk_build_params* params, uint32_t* adjacency,
                        uint64_t adjacency_stride, uint32_t* degrees);

/* The same build with the greedy searches of every batch of 256 points or more run on CUDA
 * device `device` (the search kernels of dk_search, bit-exact), pruning and back edges on the
 * host threads.  Produces exactly the graph dk_build_vamana produces. */
int32_t dk_build_vamana_device(const float* vectors, uint64_t stride, uint32_t num_points,
                               uint32_t num_frozen, uint32_t dim, int32_t metric,
                               const dk_build_params* params, uint32_t* adjacency,
                               uint64_t adjacency_stride, uint32_t* degrees, int32_t device);

/* Product-quantisation schema: 256 centres per chunk by k-means++ and Lloyd iterations on
 * the given rows; chunk offsets split dim with the first dim % chunks chunks one longer
 * (the reference's FixedChunkPQTable layout, fixed_chunk_pq_table.rs:100-133). */
int32_t dk_pq_train(const float* data, uint64_t stride, uint32_t n, uint32_t dim, uint32_t chunks,
                    uint32_t iters, uint64_t seed, uint32_t num_threads, uint32_t* offsets,
                    float* pivots);

/* Encode rows to PQ codes (nearest centre per chunk). */
int32_t dk_pq_encode(const float* data, uint64_t stride, uint32_t n, uint32_t dim, uint32_t chunks,
                     const uint32_t* offsets, const float* pivots, uint32_t num_threads,
                     uint8_t* codes, uint64_t code_stride);

#ifdef __cplusplus
}
#endif
#endif /* DISKANN_B200_H */
