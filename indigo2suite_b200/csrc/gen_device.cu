// Device-side construction of RMAT graphs: sample, relabel and symmetrise the
// edges with the same counter-based hashes as the host generator, sort the
// 64-bit (u, v) keys with a CUB radix sort, drop duplicates, and cut the CSR.
// The resulting graph is identical to i2_gen_rmat's.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include "engine.h"
#include "gen_rng.h"

namespace i2 {

__global__ void k_rmat_keys(uint64_t seed, int scale, RmatThresholds t, RmatPerm p, long long samples, int n,
                            unsigned long long* keys) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = tid; i < samples; i += stride) {
    uint64_t u, v;
    rmat_sample(seed, scale, t, (uint64_t)i, &u, &v);
    u = perm_apply(p, u);
    v = perm_apply(p, v);
    unsigned long long a = ~0ull, b = ~0ull;
    if (u != v && u < (uint64_t)n && v < (uint64_t)n) {
      a = (u << 32) | v;
      b = (v << 32) | u;
    }
    keys[2 * i] = a;
    keys[2 * i + 1] = b;
  }
}

__global__ void k_cut_csr(const unsigned long long* __restrict__ keys, long long E, int nodes, uint64_t seed,
                          int weighted, int* __restrict__ nindex, int* __restrict__ nlist, int* __restrict__ w) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < E; k += stride) {
    const unsigned long long key = keys[k];
    const int u = (int)(key >> 32), v = (int)(key & 0xffffffffu);
    nlist[k] = v;
    if (weighted) w[k] = edge_weight(seed, u, v);
  }
  for (long long v = tid; v <= nodes; v += stride) {
    const unsigned long long target = (unsigned long long)v << 32;
    long long lo = 0, hi = E;  // first k with keys[k] >= target
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (keys[mid] < target) lo = mid + 1; else hi = mid;
    }
    nindex[v] = (int)lo;
  }
}

}  // namespace i2

using namespace i2;

extern "C" int i2_graph_generate_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                                      int weighted, i2_graph** out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return I2_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  const long long n = 1LL << scale;
  if (n > 0x7fffffffLL) return I2_ERR_OVERFLOW;
  const long long samples = (long long)edge_factor * n;
  const long long nkeys = 2 * samples;
  const RmatThresholds t = make_thresholds(a, b, c);
  const RmatPerm p = make_perm(seed, scale);
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  long long* d_num = nullptr;
  void* tmp = nullptr;
  int *nindex = nullptr, *nlist = nullptr, *w = nullptr;
  int st = I2_OK;
  size_t tb = 0, tb2 = 0;
  long long num = 0, E = 0;
  unsigned long long last = 0;
  cudaError_t e = cudaMalloc(&k0, sizeof(unsigned long long) * nkeys);
  if (e == cudaSuccess) e = cudaMalloc(&k1, sizeof(unsigned long long) * nkeys);
  if (e == cudaSuccess) e = cudaMalloc(&d_num, sizeof(long long));
  if (e != cudaSuccess) goto done;
  k_rmat_keys<<<4096, 256>>>(seed, scale, t, p, samples, (int)n, k0);
  {
    cub::DoubleBuffer<unsigned long long> db(k0, k1);
    e = cub::DeviceRadixSort::SortKeys(nullptr, tb, db, nkeys);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(nullptr, tb2, k0, k1, d_num, nkeys);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, std::max(tb, tb2));
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortKeys(tmp, tb, db, nkeys);
    if (e != cudaSuccess) goto done;
    unsigned long long* sorted = db.Current();
    unsigned long long* other = db.Alternate();
    e = cub::DeviceSelect::Unique(tmp, tb2, sorted, other, d_num, nkeys);
    if (e == cudaSuccess) e = cudaMemcpy(&num, d_num, sizeof(long long), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) goto done;
    if (num > 0) e = cudaMemcpy(&last, other + num - 1, sizeof(last), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) goto done;
    E = num - ((num > 0 && last == ~0ull) ? 1 : 0);
    if (E > 0x7fffffffLL) {
      st = I2_ERR_OVERFLOW;
      goto done;
    }
    e = dev_alloc(&nindex, sizeof(int) * (n + 1));
    if (e == cudaSuccess) e = dev_alloc(&nlist, sizeof(int) * (E + 4));
    if (e == cudaSuccess && weighted) e = dev_alloc(&w, sizeof(int) * (E + 4));
    if (e != cudaSuccess) goto done;
    k_cut_csr<<<4096, 256>>>(other, E, (int)n, seed, weighted, nindex, nlist, w);
    e = cudaDeviceSynchronize();
  }
done:
  // the sort's scratch is transient: plain allocations, returned at once;
  // the graph's arrays come from the engine's pool
  cudaFree(k0);
  cudaFree(k1);
  cudaFree(d_num);
  cudaFree(tmp);
  if (st == I2_OK && e != cudaSuccess) {
    cudaGetLastError();
    st = cuda_status(e);
  }
  if (st != I2_OK) {
    dev_free(nindex);
    dev_free(nlist);
    dev_free(w);
    return st;
  }
  return graph_adopt((int)n, (int)E, nindex, nlist, w, out);
}
