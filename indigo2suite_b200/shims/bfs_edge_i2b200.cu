// Drop-in variant body for the Indigo2 harness include/bfs_edge_cuda.h,
// implementing GPUbfs_edge(const int src, const ECLgraph& g, basic_t* const dist, const int* const sp) (include/bfs_edge_cuda.h:61) on libi2b200. See shim_common.h.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
typedef int basic_t;
static const int ThreadsPerBlock = 512;
#include "bfs_edge_cuda.h"
#include "shim_common.h"

static double GPUbfs_edge(const int src, const ECLgraph& g, basic_t* const dist, const int* const sp)
{
  (void)sp;  // the engine builds its own starting-point array on the device when needed
  return i2shim_run(I2_BFS, src, g.nodes, g.edges, g.nindex, g.nlist, nullptr, dist, I2_VP_CTA);
}
