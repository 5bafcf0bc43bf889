// Host-side graph utilities shared by the C ABI translation units.
#pragma once
#include <cstdint>
#include <vector>
#include "../../include/i2b200.h"

namespace i2 {

// Check that a host CSR is well formed: nodes >= 1, edges >= 0, nindex[0] == 0,
// nindex non-decreasing, nindex[nodes] == edges, every nlist entry in [0, nodes).
// The reference performs only the first two checks (include/ECLgraph.h:57).
int validate_host_csr(const i2_eclgraph* g);

// Degree statistics of a host CSR.
void host_degree_stats(const i2_eclgraph* g, int heavy, int* maxdeg, int* nheavy, float* avgdeg,
                       float* degcv);

// Build a symmetric, deduplicated, loop-free CSR with sorted adjacency from a
// list of undirected pairs (each pair is inserted in both directions).
// weight_seed >= 0 adds the per-edge weights of edge_weight().
int csr_from_pairs(int nodes, const std::vector<uint64_t>& pairs, bool weighted, uint64_t weight_seed,
                   i2_eclgraph* out);

}  // namespace i2
