// Internal interface between the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include "../../include/i2b200.h"
#include "common.cuh"

namespace i2 {

typedef void (*KernelFn)(Ctx);

int cuda_status(cudaError_t e);
int grid_for(KernelFn fn, int max_per_sm);
KernelFn relax_kernel(int algo, int variant, bool near_far = false);
// Resident traversal kernel: fixed style `variant`, or the per-iteration pick
// when variant < 0, in the form compiled for more resident blocks when `wide`
// (resident.cu).
KernelFn resident_kernel(int algo, int variant, bool near_far, bool wide = false);
const float* mlp_device_params();
int mlp_install(const float* params, int count);

// One traversal of a device graph from one source (srcs_host == nullptr) or
// from nsrc sources at once (batched graphs). The result stays in the graph's
// workspace.
int run_traversal(i2_graph* g, int algo, int src, const int* srcs_host, int nsrc, const i2_opts* opts,
                  i2_report* rep);

// True when [p, p + bytes) lies inside one allocation of the current device
// (or managed memory); host pointers and other GPUs' memory are refused.
bool device_range_ok(const void* p, size_t bytes);

// Take ownership of CSR arrays already on the device and build a graph handle.
int graph_adopt(int nodes, int edges, int* d_nindex, int* d_nlist, int* d_eweight, i2_graph** out);

// The device CSR arrays of a graph (weights null when it has none).
int graph_device_csr(const i2_graph* g, int* nodes, int* edges, const int** nindex, const int** nlist,
                     const int** eweight);

// A copy of g with its vertices renumbered by descending degree, ties by
// ascending ID (gen_device.cu): *twin is a new graph, *inv (g.nodes ints,
// from dev_alloc) maps each original ID to the copy's.
int degree_ordered_copy(const i2_graph* g, i2_graph** twin, int** inv);

// Copy the last traversal's values to a host array of g.nodes ints.
int graph_copy_result(i2_graph* g, int* host_out, const i2_opts* opts);

// Device memory of graphs (CSR arrays, workspaces, scratch) comes from one
// stream-ordered pool per device that keeps freed blocks reserved: a graph
// uploaded after another was freed reuses that memory instead of paying a
// cudaMalloc and a cudaFree (a change of the device's mappings, milliseconds
// per GB) for every array. dev_alloc returns memory every stream may use;
// dev_free keeps cudaFree's contract (the device finishes its work before the
// block goes back to the pool). Every pointer dev_free gets must come from
// dev_alloc.
cudaError_t dev_alloc_bytes(void** p, size_t bytes);
void dev_free(void* p);
template <class T>
inline cudaError_t dev_alloc(T** p, size_t bytes) {
  return dev_alloc_bytes(reinterpret_cast<void**>(p), bytes);
}

}  // namespace i2
