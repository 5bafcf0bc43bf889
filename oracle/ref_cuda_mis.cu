// ORACLE — test infrastructure only (GPU tests). One reference CUDA MIS
// variant (REF_VARIANT, a codes/cuda/mis-cuda file), compiled unchanged with its
// harness main() renamed, exposing its host driver GPUmis_vertex on host CSR
// arrays, so that a GPU test can compare the reference's own status array with
// the oracle's and the engine's.
#define main i2ref_harness_main
#include REF_VARIANT
#undef main

extern "C" double ref_cuda_mis(int nodes, int edges, const int* nindex, const int* nlist, int* status) {
  ECLgraph d_g;
  d_g.nodes = nodes;
  d_g.edges = edges;
  d_g.eweight = nullptr;
  if (cudaMalloc((void**)&d_g.nindex, sizeof(int) * (nodes + 1)) != cudaSuccess) return -1.0;
  if (cudaMalloc((void**)&d_g.nlist, sizeof(int) * (edges > 0 ? edges : 1)) != cudaSuccess) return -1.0;
  cudaMemcpy(d_g.nindex, nindex, sizeof(int) * (nodes + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_g.nlist, nlist, sizeof(int) * edges, cudaMemcpyHostToDevice);
  data_type* priority = new data_type[nodes > 0 ? nodes : 1];
  const double t = GPUmis_vertex(d_g, priority, status);
  delete[] priority;
  cudaFree(d_g.nindex);
  cudaFree(d_g.nlist);
  return t;
}
