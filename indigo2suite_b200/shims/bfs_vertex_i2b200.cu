// Drop-in variant body for the Indigo2 harness include/bfs_vertex_cuda.h,
// implementing GPUbfs_vertex(const int src, const ECLgraph& g, basic_t* const dist) (include/bfs_vertex_cuda.h:61) on libi2b200. See shim_common.h.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
typedef int basic_t;
static const int ThreadsPerBlock = 512;
#include "bfs_vertex_cuda.h"
#include "shim_common.h"

static double GPUbfs_vertex(const int src, const ECLgraph& g, basic_t* const dist)
{
  return i2shim_run(I2_BFS, src, g.nodes, g.edges, g.nindex, g.nlist, nullptr, dist, I2_AUTO_HEURISTIC);
}
