// Drop-in variant body for the Indigo2 harness include/sssp_vertex_cuda.h,
// implementing GPUsssp_vertex(const int src, const ECLgraph& g, basic_t* const dist) (include/sssp_vertex_cuda.h:60) on libi2b200. See shim_common.h.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
typedef int basic_t;
static const int ThreadsPerBlock = 512;
#include "sssp_vertex_cuda.h"
#include "shim_common.h"

static double GPUsssp_vertex(const int src, const ECLgraph& g, basic_t* const dist)
{
  return i2shim_run(I2_SSSP, src, g.nodes, g.edges, g.nindex, g.nlist, g.eweight, dist, I2_AUTO_HEURISTIC);
}
