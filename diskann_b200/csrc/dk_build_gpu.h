// Device side of graph construction (dk_build_vamana_device).  For a batch of points: the
// greedy searches run on the GPU against the graph as it stood before the batch, with the same
// kernel as dk_search (bit-exact), recording each point's visited nodes; each point's out-list
// is pruned from its record on the GPU (occlude_list restated, bit-exact with the host
// version); the host groups the back edges by target; the GPU appends them and re-prunes the
// lists that overflow.  While batches run on the GPU its adjacency is the current graph; the
// host reads it back (dk_build_gpu_get_rows) before it works on the graph itself again.
#pragma once

#include <cstdint>
#include <vector>

#include "diskann_b200.h"

struct dk_build_gpu;

int32_t dk_build_gpu_create(const float* vectors, uint64_t stride, uint32_t num_points,
                            uint32_t num_frozen, uint32_t dim, int32_t metric,
                            uint32_t max_degree, uint32_t l_build, uint32_t max_batch,
                            int32_t device, dk_build_gpu** out);

// Search points [start, start + count).  On return hops[i] is how many nodes point i expanded
// (a point with hops[i] > rec_cap must be searched again on the host); with `copy_records`
// rec_ids / rec_d also hold, for point i, its expanded nodes in order with their distances at
// i * rec_cap (else they are left on the device for dk_build_gpu_prune_forward).
int32_t dk_build_gpu_search(dk_build_gpu* g, uint32_t start, uint32_t count, bool copy_records,
                            const uint32_t** rec_ids, const float** rec_d,
                            const uint32_t** hops, uint32_t* rec_cap);

// occlude_list parameters (index.rs:2570-2782).
struct dk_build_prune_cfg {
  float alpha;
  uint32_t degree;         // pruned degree R
  uint32_t max_occlusion;  // pool size cap
  uint32_t occluding;      // PruneKind::Occluding (inner product) instead of the triangle rule
};

// Prune the out-list of every point of the last searched batch from its device record.  On
// return out[i * cfg.degree ...] holds point i's list and counts[i] its length, or UINT32_MAX
// for a point whose record overflowed (the caller prunes those on the host).
int32_t dk_build_gpu_prune_forward(dk_build_gpu* g, uint32_t count, const dk_build_prune_cfg& cfg,
                                   const uint32_t** out, const uint32_t** counts);

// Back edges (add_edge_and_prune, index.rs:2269-2346) on the device graph: group i appends
// sources src[off[i] .. off[i+1]) (in order, skipping ids already present) to node
// targets[i]'s list and re-prunes a list that exceeds max_degree.  Groups whose list would not
// fit the kernel's pool are left untouched and returned in `oversize` for the caller.
int32_t dk_build_gpu_backedges(dk_build_gpu* g, const uint32_t* targets, const uint32_t* off,
                               const uint32_t* src, uint32_t groups, uint32_t max_group,
                               const dk_build_prune_cfg& cfg, std::vector<uint32_t>& oversize);

// The device graph's rows: all of them into adj, or one.
int32_t dk_build_gpu_get_rows(dk_build_gpu* g, std::vector<std::vector<uint32_t>>& adj);
int32_t dk_build_gpu_get_row(dk_build_gpu* g, uint32_t node, std::vector<uint32_t>& row);

// Write the adjacency lists adj[nodes[i]] into the device graph.
int32_t dk_build_gpu_set_rows(dk_build_gpu* g, const uint32_t* nodes, uint32_t count,
                              const std::vector<std::vector<uint32_t>>& adj);

void dk_build_gpu_destroy(dk_build_gpu* g);
