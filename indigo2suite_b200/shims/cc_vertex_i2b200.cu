// Drop-in variant body for the Indigo2 harness include/cc_vertex_cuda.h,
// implementing GPUcc_vertex(const ECLgraph& g, basic_t* const label) (include/cc_vertex_cuda.h:57) on libi2b200. See shim_common.h.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
typedef int basic_t;
static const int ThreadsPerBlock = 512;
#include "cc_vertex_cuda.h"
#include "shim_common.h"

static double GPUcc_vertex(const ECLgraph& g, basic_t* const label)
{
  return i2shim_run(I2_CC, 0, g.nodes, g.edges, g.nindex, g.nlist, nullptr, label, I2_AUTO_HEURISTIC);
}
