// ORACLE — test infrastructure only.
// Exposes the reference's own serial checker CPUserialDijkstra (compiled
// unchanged from the reference harness header named by REF_HEADER) as a C
// function, so tests can pin oracle.c against it on many graphs.
//   REF_HEADER=bfs_vertex_omp.h   -> include/bfs_vertex_omp.h:105-130 (unit weights)
//   REF_HEADER=sssp_vertex_omp.h  -> include/sssp_vertex_omp.h:105-130 (max-heap on -d)
//   REF_HEADER=sssp_edge_omp.h    -> include/sssp_edge_omp.h:105-130 (min-heap)
// The harness's main() is renamed so that it does not clash with the caller's.
typedef int data_type;
#define main i2ref_harness_main
#include REF_HEADER
#undef main
#include "ref_stub.h"

extern "C" int ref_serial(int nodes, int edges, int* nindex, int* nlist, int* eweight, int src, int* dist) {
  ECLgraph g;
  g.nodes = nodes;
  g.edges = edges;
  g.nindex = nindex;
  g.nlist = nlist;
  g.eweight = eweight;
  CPUserialDijkstra(src, g, dist);
  return 0;
}
