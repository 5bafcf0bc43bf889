// Drop-in variant body for the Indigo2 harness include/cc_edge_cuda.h,
// implementing GPUcc_edge(const ECLgraph& g, basic_t* const label, const int* const sp) (include/cc_edge_cuda.h:57) on libi2b200. See shim_common.h.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
typedef int basic_t;
static const int ThreadsPerBlock = 512;
#include "cc_edge_cuda.h"
#include "shim_common.h"

static double GPUcc_edge(const ECLgraph& g, basic_t* const label, const int* const sp)
{
  (void)sp;  // the engine builds its own starting-point array on the device when needed
  return i2shim_run(I2_CC, 0, g.nodes, g.edges, g.nindex, g.nlist, nullptr, label, I2_EDGE_TOPO);
}
