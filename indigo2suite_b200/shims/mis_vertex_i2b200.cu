// Drop-in variant body for the Indigo2 harness include/mis_vertex_cuda.h,
// implementing GPUmis_vertex(const ECLgraph& g, data_type* const priority, int* const status)
// (include/mis_vertex_cuda.h:52) on libi2b200. See shim_common.h. Like the
// reference's own GPU bodies, it leaves the host priority array untouched (the
// priorities live on the device only).
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
static const int ThreadsPerBlock = 512;
#include "mis_vertex_cuda.h"
#include "shim_common.h"

static double GPUmis_vertex(const ECLgraph& g, data_type* const priority, int* const status)
{
  (void)priority;
  return i2shim_run(I2_MIS, 0, g.nodes, g.edges, g.nindex, g.nlist, nullptr, status, I2_VP_WARP);
}
