// Device side of graph construction (dk_build_vamana_device): the greedy searches of a batch of
// points run on the GPU against the graph as it stood before the batch, with the same kernel
// as dk_search (bit-exact), returning each point's visited search record.  Host code prunes
// and adds back edges, then writes the changed adjacency rows back with dk_build_gpu_set_rows.
#pragma once

#include <cstdint>
#include <vector>

#include "diskann_b200.h"

struct dk_build_gpu;

int32_t dk_build_gpu_create(const float* vectors, uint64_t stride, uint32_t num_points,
                            uint32_t num_frozen, uint32_t dim, int32_t metric,
                            uint32_t max_degree, uint32_t l_build, uint32_t max_batch,
                            int32_t device, dk_build_gpu** out);

// Search points [start, start + count).  On return rec_ids / rec_d hold, for point i, its
// expanded nodes in order with their distances at i * rec_cap; hops[i] is how many there were
// (a point with hops[i] > rec_cap must be searched again on the host).
int32_t dk_build_gpu_search(dk_build_gpu* g, uint32_t start, uint32_t count,
                            const uint32_t** rec_ids, const float** rec_d,
                            const uint32_t** hops, uint32_t* rec_cap);

// Write the adjacency lists adj[nodes[i]] into the device graph.
int32_t dk_build_gpu_set_rows(dk_build_gpu* g, const uint32_t* nodes, uint32_t count,
                              const std::vector<std::vector<uint32_t>>& adj);

void dk_build_gpu_destroy(dk_build_gpu* g);
