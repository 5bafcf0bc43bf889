// Drop-in variant body for the Indigo2 harness include/mis_edge_cuda.h,
// implementing GPUmis_edge(const ECLgraph& g, const int* const sp, data_type* const priority,
// int* const status) (include/mis_edge_cuda.h:54) on libi2b200. See shim_common.h.
// The engine's MIS needs no starting-point array; the priority array is left
// untouched, as the reference's own GPU bodies do.
#include <cuda/atomic>
typedef int flag_t;
typedef int data_type;
static const int ThreadsPerBlock = 512;
#include "mis_edge_cuda.h"
#include "shim_common.h"

static double GPUmis_edge(const ECLgraph& g, const int* const sp, data_type* const priority, int* const status)
{
  (void)sp;
  (void)priority;
  return i2shim_run(I2_MIS, 0, g.nodes, g.edges, g.nindex, g.nlist, nullptr, status, I2_VP_WARP);
}
