// Batches of graphs traversed together.
//
// The graphs of a batch are laid out as one disjoint-union CSR in HBM (graph k's
// vertices at offset voff[k], its CSR entries at offset eoff[k]). A traversal
// of the union from one source per graph is the same as one traversal per
// graph: no edge crosses two graphs, so every graph reaches the same fixed point
// as on its own. One persistent relax launch per iteration then drains frontier
// chunks of all graphs from the same device-side chunk counter, and the whole
// loop is one CUDA graph, instead of one launch sequence (with a host round trip
// per iteration) per graph.
#include <cuda_runtime.h>
#include <cstring>
#include <vector>
#include "engine.h"

namespace i2 {

__global__ void k_shift(int* a, long long n, int delta) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < n; k += stride) a[k] += delta;
}

// dst[k] = src[k] + delta (device to device, one graph of a batch).
__global__ void k_copy_shift(int* __restrict__ dst, const int* __restrict__ src, long long n, int delta) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < n; k += stride) dst[k] = src[k] + delta;
}

}  // namespace i2

using namespace i2;

struct i2_batch {
  i2_graph* g = nullptr;
  std::vector<long long> voff;
  std::vector<long long> eoff;
  int n = 0;
};

extern "C" {

int i2_batch_upload(const i2_eclgraph* graphs, int n, i2_batch** out) {
  if (!graphs || n < 1 || !out) return I2_ERR_ARG;
  *out = nullptr;
  long long V = 0, E = 0;
  int weighted = 1;
  for (int k = 0; k < n; ++k) {
    const i2_eclgraph& h = graphs[k];
    if (h.nodes < 1 || h.edges < 0 || !h.nindex || (h.edges && !h.nlist)) return I2_ERR_ARG;
    if (h.nindex[0] != 0 || h.nindex[h.nodes] != h.edges) return I2_ERR_FORMAT;
    V += h.nodes;
    E += h.edges;
    if (!h.eweight) weighted = 0;
  }
  if (V > 0x7ffffffeLL || E > 0x7ffffffbLL) return I2_ERR_OVERFLOW;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  int *nindex = nullptr, *nlist = nullptr, *w = nullptr;
  cudaError_t e = dev_alloc(&nindex, sizeof(int) * (V + 1));
  if (e == cudaSuccess) e = dev_alloc(&nlist, sizeof(int) * (E + 4));
  if (e == cudaSuccess && weighted) e = dev_alloc(&w, sizeof(int) * (E + 4));
  i2_batch* b = new i2_batch();
  b->n = n;
  // Entry ranges must be valid before anything indexes through them (all
  // graphs checked in parallel).
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int k = 0; k < n; ++k) {
    const i2_eclgraph& h = graphs[k];
    for (long long x = 0; x < h.edges; ++x) bad |= (unsigned)h.nlist[x] >= (unsigned)h.nodes;
    for (int v = 0; v < h.nodes; ++v) bad |= h.nindex[v + 1] < h.nindex[v];
  }
  if (bad) e = cudaErrorInvalidValue;
  long long vo = 0, eo = 0;
  for (int k = 0; k < n && e == cudaSuccess; ++k) {
    const i2_eclgraph& h = graphs[k];
    b->voff.push_back(vo);
    b->eoff.push_back(eo);
    e = cudaMemcpy(nindex + vo, h.nindex, sizeof(int) * h.nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && h.edges) e = cudaMemcpy(nlist + eo, h.nlist, sizeof(int) * h.edges, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && weighted && h.edges)
      e = cudaMemcpy(w + eo, h.eweight, sizeof(int) * h.edges, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && eo) k_shift<<<256, 256>>>(nindex + vo, h.nodes, (int)eo);
    if (e == cudaSuccess && vo && h.edges) k_shift<<<256, 256>>>(nlist + eo, h.edges, (int)vo);
    vo += h.nodes;
    eo += h.edges;
  }
  if (e == cudaSuccess) {
    const int Ei = (int)E;
    e = cudaMemcpy(nindex + V, &Ei, sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    const bool bad_input = e == cudaErrorInvalidValue;
    cudaGetLastError();
    dev_free(nindex);
    dev_free(nlist);
    dev_free(w);
    delete b;
    return bad_input ? I2_ERR_FORMAT : cuda_status(e);
  }
  int st = graph_adopt((int)V, (int)E, nindex, nlist, w, &b->g);
  if (st) {
    delete b;
    return st;
  }
  *out = b;
  return I2_OK;
}

int i2_batch_from_device(i2_graph* const* graphs, int n, i2_batch** out) {
  if (!graphs || n < 1 || !out) return I2_ERR_ARG;
  *out = nullptr;
  std::vector<int> nv(n), ne(n);
  std::vector<const int*> ni(n), nl(n), nw(n);
  long long V = 0, E = 0;
  int weighted = 1;
  for (int k = 0; k < n; ++k) {
    if (!graphs[k] || graph_device_csr(graphs[k], &nv[k], &ne[k], &ni[k], &nl[k], &nw[k])) return I2_ERR_ARG;
    V += nv[k];
    E += ne[k];
    if (!nw[k]) weighted = 0;
  }
  if (V > 0x7ffffffeLL || E > 0x7ffffffbLL) return I2_ERR_OVERFLOW;
  int *nindex = nullptr, *nlist = nullptr, *w = nullptr;
  cudaError_t e = dev_alloc(&nindex, sizeof(int) * (V + 1));
  if (e == cudaSuccess) e = dev_alloc(&nlist, sizeof(int) * (E + 4));
  if (e == cudaSuccess && weighted) e = dev_alloc(&w, sizeof(int) * (E + 4));
  i2_batch* b = new i2_batch();
  b->n = n;
  long long vo = 0, eo = 0;
  for (int k = 0; k < n && e == cudaSuccess; ++k) {
    b->voff.push_back(vo);
    b->eoff.push_back(eo);
    // each graph's arrays were validated when it was built or uploaded
    k_copy_shift<<<256, 256>>>(nindex + vo, ni[k], nv[k], (int)eo);
    if (ne[k]) k_copy_shift<<<1024, 256>>>(nlist + eo, nl[k], ne[k], (int)vo);
    if (weighted && ne[k]) e = cudaMemcpyAsync(w + eo, nw[k], sizeof(int) * ne[k], cudaMemcpyDeviceToDevice);
    vo += nv[k];
    eo += ne[k];
  }
  if (e == cudaSuccess) {
    const int Ei = (int)E;
    e = cudaMemcpy(nindex + V, &Ei, sizeof(int), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    cudaGetLastError();
    dev_free(nindex);
    dev_free(nlist);
    dev_free(w);
    delete b;
    return cuda_status(e);
  }
  int st = graph_adopt((int)V, (int)E, nindex, nlist, w, &b->g);
  if (st) {
    delete b;
    return st;
  }
  *out = b;
  return I2_OK;
}

int i2_batch_offsets(const i2_batch* b, long long* voff) {
  if (!b || !voff) return I2_ERR_ARG;
  i2_graph_info info;
  i2_graph_info_get(b->g, &info);
  for (int k = 0; k < b->n; ++k) voff[k] = b->voff[k];
  voff[b->n] = info.nodes;
  return I2_OK;
}

int i2_batch_run(i2_batch* b, int algo, const int* srcs, int* dist, const i2_opts* opts, i2_report* rep) {
  if (!b || !dist) return I2_ERR_ARG;
  if (algo != I2_CC && !srcs) return I2_ERR_ARG;
  i2_graph_info info;
  i2_graph_info_get(b->g, &info);
  std::vector<int> global;
  if (algo != I2_CC) {
    global.resize(b->n);
    for (int k = 0; k < b->n; ++k) {
      const long long nk = (k + 1 < b->n ? b->voff[k + 1] : info.nodes) - b->voff[k];
      if (srcs[k] < 0 || srcs[k] >= nk) return I2_ERR_ARG;
      global[k] = (int)(b->voff[k] + srcs[k]);
    }
  }
  int st = run_traversal(b->g, algo, 0, algo == I2_CC ? nullptr : global.data(), b->n, opts, rep);
  if (st && st != I2_ERR_ITER_CAP) return st;
  const int st2 = graph_copy_result(b->g, dist, opts);
  return st2 ? st2 : st;
}

int i2_batch_run_device(i2_batch* b, int algo, const int* srcs, const i2_opts* opts, i2_report* rep) {
  if (!b) return I2_ERR_ARG;
  if (algo != I2_CC && !srcs) return I2_ERR_ARG;
  i2_graph_info info;
  int n = 0, e = 0;
  i2_graph_size(b->g, &n, &e);
  (void)info;
  std::vector<int> global;
  if (algo != I2_CC) {
    global.resize(b->n);
    for (int k = 0; k < b->n; ++k) {
      const long long nk = (k + 1 < b->n ? b->voff[k + 1] : n) - b->voff[k];
      if (srcs[k] < 0 || srcs[k] >= nk) return I2_ERR_ARG;
      global[k] = (int)(b->voff[k] + srcs[k]);
    }
  }
  return run_traversal(b->g, algo, 0, algo == I2_CC ? nullptr : global.data(), b->n, opts, rep);
}

int i2_batch_result(i2_batch* b, int* dist, const i2_opts* opts) {
  if (!b || !dist) return I2_ERR_ARG;
  return graph_copy_result(b->g, dist, opts);
}

int i2_batch_tune(i2_batch* b, int heavy_threshold, int blocks_per_sm, int smem_carveout) {
  if (!b) return I2_ERR_ARG;
  return i2_graph_tune(b->g, heavy_threshold, blocks_per_sm, smem_carveout);
}

int i2_batch_free(i2_batch* b) {
  if (!b) return I2_ERR_ARG;
  i2_graph_free(b->g);
  delete b;
  return I2_OK;
}

}  // extern "C"
