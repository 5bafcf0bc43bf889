// ORACLE — test infrastructure only (CPU baseline of bench.py).
// One reference CPU program (REF_VARIANT, a codes/omp or codes/cpp file),
// compiled unchanged with its harness main() renamed, exposing a single call
// of its host driver so that each benchmark step is exactly one traversal.
#include <omp.h>
#define main i2ref_harness_main
#include REF_VARIANT
#undef main

extern "C" double ref_cpu_run(int nodes, int edges, int* nindex, int* nlist, int* eweight, int src, int* dist,
                              const int* sp, int threads) {
  ECLgraph g;
  g.nodes = nodes;
  g.edges = edges;
  g.nindex = nindex;
  g.nlist = nlist;
  g.eweight = eweight;
  (void)sp;
  (void)src;
#if defined(REF_CPP_SSSP_EDGE)
  return CPUsssp_edge(src, g, dist, sp, threads);
#elif defined(REF_CPP_SSSP_VERTEX)
  return CPUsssp_vertex(src, g, dist, threads);
#elif defined(REF_OMP_SSSP_EDGE)
  omp_set_num_threads(threads);
  return CPUsssp_edge(src, g, dist, sp);
#elif defined(REF_CPP_BFS_VERTEX)
  return CPPbfs_vertex(src, g, dist, threads);
#elif defined(REF_OMP_BFS_VERTEX)
  omp_set_num_threads(threads);
  return CPUbfs_vertex(src, g, dist);
#elif defined(REF_CPP_CC_VERTEX)
  return CPUcc_vertex(g, dist, threads);
#elif defined(REF_OMP_CC_VERTEX)
  omp_set_num_threads(threads);
  return CPUcc_vertex(g, dist);
#elif defined(REF_CPP_MIS_VERTEX)
  // the MIS driver fills a byte status per vertex (1 in the set, 2 excluded)
  data_type* priority = new data_type[nodes > 0 ? nodes : 1];
  unsigned char* st = new unsigned char[nodes > 0 ? nodes : 1];
  const double t = CPPmis_vertex(g, priority, st, threads);
  for (int v = 0; v < nodes; ++v) dist[v] = st[v];
  delete[] priority;
  delete[] st;
  return t;
#endif
}
