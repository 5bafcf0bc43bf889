// Device-side construction of CSR graphs.
//
// One builder turns 64-bit (u << 32 | v) keys (~0: dropped) into a CSR: a CUB
// radix sort of the keys (of key/weight pairs when the weights come with the
// edges), duplicates merged (keeping the smallest weight), then the CSR cut by
// a binary search per vertex. On top of it:
//  * i2_graph_from_coo_device: a graph from COO pairs already in device memory;
//  * the seeded RMAT, ER and grid generators, which sample their edges with the
//    same counter-based hashes as the host generators (graph_host.cpp), so that
//    each device graph is identical to the host one. ER and the grid's
//    long-range edges take "the first m distinct pairs of the hash stream":
//    candidates are sorted by (pair, index), the first index of each pair
//    kept, and the survivors sorted by index again.
#include <cuda_runtime.h>
#include <cmath>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_select.cuh>
#include "engine.h"
#include "gen_rng.h"

namespace i2 {

constexpr unsigned long long kDropKey = ~0ull;

__global__ void k_rmat_keys(uint64_t seed, int scale, RmatThresholds t, RmatPerm p, long long samples, int n,
                            unsigned long long* keys) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = tid; i < samples; i += stride) {
    uint64_t u, v;
    rmat_sample(seed, scale, t, (uint64_t)i, &u, &v);
    u = perm_apply(p, u);
    v = perm_apply(p, v);
    unsigned long long a = kDropKey, b = kDropKey;
    if (u != v && u < (uint64_t)n && v < (uint64_t)n) {
      a = (u << 32) | v;
      b = (v << 32) | u;
    }
    keys[2 * i] = a;
    keys[2 * i + 1] = b;
  }
}

// Weights of the cut CSR: none, the seeded generator weight of {u, v}, or
// given per sorted key.
struct CutWeights {
  int mode;          // 0 none, 1 seeded, 2 given
  uint64_t seed;
  const int* given;  // mode 2: weight of keys[k]
};

__global__ void k_cut_csr(const unsigned long long* __restrict__ keys, long long E, int nodes, CutWeights cw,
                          int* __restrict__ nindex, int* __restrict__ nlist, int* __restrict__ w) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < E; k += stride) {
    const unsigned long long key = keys[k];
    const int u = (int)(key >> 32), v = (int)(key & 0xffffffffu);
    nlist[k] = v;
    if (cw.mode == 1) w[k] = edge_weight(cw.seed, u, v);
    else if (cw.mode == 2) w[k] = cw.given[k];
  }
  for (long long v = tid; v <= nodes; v += stride) {
    const unsigned long long target = (unsigned long long)v << 32;
    long long lo = 0, hi = E;  // first k with keys[k] >= target
    while (lo < hi) {
      const long long mid = lo + ((hi - lo) >> 1);
      if (keys[mid] < target) lo = mid + 1; else hi = mid;
    }
    nindex[v] = (int)lo;
  }
}

struct MinOp {
  __device__ __forceinline__ int operator()(int a, int b) const { return a < b ? a : b; }
};

// Scratch of a build, freed on every path (plain allocations: transient, so
// the engine's pool never keeps them).
struct Scratch {
  static constexpr int kMax = 16;
  void* p[kMax] = {nullptr};
  int n = 0;
  template <class T>
  cudaError_t get(T** out, size_t bytes) {
    *out = nullptr;
    if (n == kMax) return cudaErrorMemoryAllocation;  // more buffers than one build takes
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes > 0 ? bytes : 1);
    if (e == cudaSuccess) p[n++] = q;
    *out = static_cast<T*>(q);
    return e;
  }
  ~Scratch() {
    for (int k = 0; k < n; ++k) cudaFree(p[k]);
  }
};

// CSR of `nodes` vertices from nkeys keys in k0 (k1: a buffer of the same
// size; both are overwritten). Weights: cw.mode 1 seeded; cw.mode 2 given per
// key in w0 (w1: a buffer of the same size), duplicates keeping the smallest.
static int csr_from_keys(unsigned long long* k0, unsigned long long* k1, int* w0, int* w1, long long nkeys,
                         int nodes, CutWeights cw, i2_graph** out) {
  Scratch sc;
  long long* d_num = nullptr;
  void* tmp = nullptr;
  size_t tb = 0, tb2 = 0;
  cudaError_t e = sc.get(&d_num, sizeof(long long));
  if (e == cudaSuccess) e = cudaMemset(d_num, 0, sizeof(long long));  // stays 0 for an empty key set
  if (e != cudaSuccess) return cuda_status(e);
  const bool given = cw.mode == 2;
  cub::DoubleBuffer<unsigned long long> dk(k0, k1);
  cub::DoubleBuffer<int> dw(w0, w1);
  if (given) {
    e = cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dw, nkeys);
    if (e == cudaSuccess) e = cub::DeviceReduce::ReduceByKey(nullptr, tb2, k0, k1, w0, w1, d_num, MinOp(), nkeys);
  } else {
    e = cub::DeviceRadixSort::SortKeys(nullptr, tb, dk, nkeys);
    if (e == cudaSuccess) e = cub::DeviceSelect::Unique(nullptr, tb2, k0, k1, d_num, nkeys);
  }
  if (e == cudaSuccess) e = sc.get(&tmp, std::max(tb, tb2));
  if (e != cudaSuccess) return cuda_status(e);
  if (given) e = cub::DeviceRadixSort::SortPairs(tmp, tb, dk, dw, nkeys);
  else e = cub::DeviceRadixSort::SortKeys(tmp, tb, dk, nkeys);
  if (e != cudaSuccess) return cuda_status(e);
  unsigned long long* sorted = dk.Current();
  unsigned long long* uniq = dk.Alternate();
  int* wsorted = dw.Current();
  int* wuniq = dw.Alternate();
  if (given) e = cub::DeviceReduce::ReduceByKey(tmp, tb2, sorted, uniq, wsorted, wuniq, d_num, MinOp(), nkeys);
  else e = cub::DeviceSelect::Unique(tmp, tb2, sorted, uniq, d_num, nkeys);
  long long num = 0;
  unsigned long long last = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&num, d_num, sizeof(long long), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && num > 0) e = cudaMemcpy(&last, uniq + num - 1, sizeof(last), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  const long long E = num - ((num > 0 && last == kDropKey) ? 1 : 0);
  if (E > 0x7fffffffLL) return I2_ERR_OVERFLOW;
  int *nindex = nullptr, *nlist = nullptr, *w = nullptr;
  e = dev_alloc(&nindex, sizeof(int) * ((size_t)nodes + 1));
  if (e == cudaSuccess) e = dev_alloc(&nlist, sizeof(int) * ((size_t)E + 4));
  if (e == cudaSuccess && cw.mode) e = dev_alloc(&w, sizeof(int) * ((size_t)E + 4));
  if (e == cudaSuccess) {
    CutWeights c2 = cw;
    c2.given = wuniq;
    k_cut_csr<<<4096, 256>>>(uniq, E, nodes, c2, nindex, nlist, w);
    e = cudaDeviceSynchronize();
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    dev_free(nindex);
    dev_free(nlist);
    dev_free(w);
    return cuda_status(e);
  }
  return graph_adopt(nodes, (int)E, nindex, nlist, w, out);
}

// ---------------------------------------------------------------------------
// COO pairs -> keys.

__global__ void k_coo_keys(const int* __restrict__ src, const int* __restrict__ dst, const int* __restrict__ w,
                           long long m, int nodes, int sym, unsigned long long* keys, int* wk, int* bad) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int per = sym ? 2 : 1;
  for (long long k = tid; k < m; k += stride) {
    const int u = src[k], v = dst[k];
    if ((unsigned)u >= (unsigned)nodes || (unsigned)v >= (unsigned)nodes) {
      atomicOr(bad, 1);
      keys[per * k] = kDropKey;
      if (sym) keys[per * k + 1] = kDropKey;
      continue;
    }
    const bool loop = u == v;
    keys[per * k] = loop ? kDropKey : ((unsigned long long)u << 32) | (unsigned)v;
    if (sym) keys[per * k + 1] = loop ? kDropKey : ((unsigned long long)v << 32) | (unsigned)u;
    if (w) {
      wk[per * k] = w[k];
      if (sym) wk[per * k + 1] = w[k];
    }
  }
}

// ---------------------------------------------------------------------------
// Candidate pairs of ER and of the grid's long-range edges: key (lo << 32 | hi)
// or kDropKey, with the candidate's index as the value.

__global__ void k_er_candidates(uint64_t seed, int n, long long first, long long count, unsigned long long* keys,
                                unsigned long long* idx) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < count; k += stride) {
    const uint64_t j = (uint64_t)(first + k);
    const uint64_t u = h3(seed, kStreamErU, j) % (uint64_t)n;
    const uint64_t v = h3(seed, kStreamErV, j) % (uint64_t)n;
    const uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
    keys[k] = u == v ? kDropKey : ((lo << 32) | hi);
    idx[k] = j;
  }
}

__device__ __forceinline__ bool grid_kept(uint64_t seed, uint64_t drop, long long idx) {
  return h3(seed, kStreamGridDrop, (uint64_t)idx) >= drop;
}

__global__ void k_grid_extra_candidates(uint64_t seed, int side, uint64_t drop, long long count,
                                        unsigned long long* keys, unsigned long long* idx) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long V = (long long)side * side;
  const long long H = (long long)side * (side - 1);
  for (long long k = tid; k < count; k += stride) {
    const uint64_t j = (uint64_t)k;
    const long long u = (long long)(h3(seed, kStreamGridU, j) % (uint64_t)V);
    const long long v = (long long)(h3(seed, kStreamGridV, j) % (uint64_t)V);
    const long long lo = u < v ? u : v, hi = u < v ? v : u;
    bool ok = u != v;
    if (ok) {  // not a kept grid edge
      long long gi = -1;
      if (hi == lo + 1 && (lo % side) != side - 1) gi = (lo / side) * (side - 1) + (lo % side);
      else if (hi == lo + side) gi = H + lo;
      if (gi >= 0 && grid_kept(seed, drop, gi)) ok = false;
    }
    keys[k] = ok ? (((unsigned long long)lo << 32) | (unsigned long long)hi) : kDropKey;
    idx[k] = j;
  }
}

__global__ void k_grid_count(uint64_t seed, uint64_t drop, long long G, unsigned long long* kept) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned long long c = 0;
  for (long long i = tid; i < G; i += stride) c += grid_kept(seed, drop, i) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(kept, c);
}

__global__ void k_grid_keys(uint64_t seed, int side, uint64_t drop, long long G, unsigned long long* keys) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long H = (long long)side * (side - 1);
  for (long long i = tid; i < G; i += stride) {
    unsigned long long a = kDropKey, b = kDropKey;
    if (grid_kept(seed, drop, i)) {
      long long u, v;
      if (i < H) {
        u = (i / (side - 1)) * side + i % (side - 1);
        v = u + 1;
      } else {
        u = i - H;
        v = u + side;
      }
      a = ((unsigned long long)u << 32) | (unsigned long long)v;
      b = ((unsigned long long)v << 32) | (unsigned long long)u;
    }
    keys[2 * i] = a;
    keys[2 * i + 1] = b;
  }
}

// Both directions of `count` pair keys (lo << 32 | hi).
__global__ void k_both_directions(const unsigned long long* __restrict__ pairs, long long count,
                                  unsigned long long* out) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = tid; k < count; k += stride) {
    const unsigned long long p = pairs[k];
    out[2 * k] = p;
    out[2 * k + 1] = (p << 32) | (p >> 32);
  }
}

// The first `want` distinct valid candidate pairs in index order, written to
// out (device, want entries). Candidates come from make(count, keys, idx);
// their count starts at `start` and grows by a quarter (+64) until enough
// distinct pairs are found. Returns I2_OK, I2_ERR_ARG when the count has
// passed `limit` without enough of them, or a CUDA status.
template <class Make>
static int first_distinct(long long want, long long start, long long limit, Make make, unsigned long long* out) {
  long long C = start;
  for (;;) {
    Scratch sc;
    unsigned long long *k0, *k1, *i0, *i1;
    long long* d_num;
    cudaError_t e = sc.get(&k0, sizeof(unsigned long long) * C);
    if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * C);
    if (e == cudaSuccess) e = sc.get(&i0, sizeof(unsigned long long) * C);
    if (e == cudaSuccess) e = sc.get(&i1, sizeof(unsigned long long) * C);
    if (e == cudaSuccess) e = sc.get(&d_num, sizeof(long long));
    if (e != cudaSuccess) return cuda_status(e);
    make(C, k0, i0);
    size_t tb = 0, tb2 = 0;
    cub::DoubleBuffer<unsigned long long> dk(k0, k1), di(i0, i1);
    e = cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, di, C);
    if (e == cudaSuccess) e = cub::DeviceSelect::UniqueByKey(nullptr, tb2, k0, i0, k1, i1, d_num, C);
    void* tmp = nullptr;
    if (e == cudaSuccess) e = sc.get(&tmp, std::max(tb, tb2));
    // stable: equal pairs keep their index order, so the first of each run has the smallest index
    if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp, tb, dk, di, C);
    if (e != cudaSuccess) return cuda_status(e);
    unsigned long long *uk = dk.Alternate(), *ui = di.Alternate();
    e = cub::DeviceSelect::UniqueByKey(tmp, tb2, dk.Current(), di.Current(), uk, ui, d_num, C);
    long long U = 0;
    unsigned long long last = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&U, d_num, sizeof(long long), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && U > 0) e = cudaMemcpy(&last, uk + U - 1, sizeof(last), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    if (U > 0 && last == kDropKey) --U;
    if (U >= want || C > limit) {
      if (U < want) return I2_ERR_ARG;
      // survivors by index: sort (index, pair) and keep the first `want`
      cub::DoubleBuffer<unsigned long long> bi(ui, dk.Current()), bk(uk, di.Current());
      size_t tb3 = 0;
      e = cub::DeviceRadixSort::SortPairs(nullptr, tb3, bi, bk, U);
      void* tmp2 = nullptr;
      if (e == cudaSuccess) e = sc.get(&tmp2, tb3);
      if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairs(tmp2, tb3, bi, bk, U);
      if (e == cudaSuccess && want > 0)
        e = cudaMemcpy(out, bk.Current(), sizeof(unsigned long long) * want, cudaMemcpyDeviceToDevice);
      if (e == cudaSuccess) e = cudaDeviceSynchronize();
      return e == cudaSuccess ? I2_OK : cuda_status(e);
    }
    C = C + C / 4 + 64;  // the host generator's growth
  }
}

}  // namespace i2

using namespace i2;

// RMAT on n vertices: `scale` bits per endpoint, `samples` samples, endpoints
// at or above n rejected (dropped) after relabelling.
static int generate_rmat(long long n, int scale, long long samples, double a, double b, double c, uint64_t seed,
                         int weighted, i2_graph** out) {
  const long long nkeys = 2 * samples;
  Scratch sc;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  cudaError_t e = sc.get(&k0, sizeof(unsigned long long) * nkeys);
  if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * nkeys);
  if (e != cudaSuccess) return cuda_status(e);
  k_rmat_keys<<<4096, 256>>>(seed, scale, make_thresholds(a, b, c), make_perm(seed, scale), samples, (int)n, k0);
  return csr_from_keys(k0, k1, nullptr, nullptr, nkeys, (int)n, CutWeights{weighted ? 1 : 0, seed, nullptr}, out);
}

extern "C" int i2_graph_generate_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                                      int weighted, i2_graph** out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return I2_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  const long long n = 1LL << scale;
  if (n > 0x7fffffffLL) return I2_ERR_OVERFLOW;
  return generate_rmat(n, scale, (long long)edge_factor * n, a, b, c, seed, weighted, out);
}

extern "C" int i2_graph_generate_rmat_n(int n, int edge_factor, double a, double b, double c, uint64_t seed,
                                        int weighted, i2_graph** out) {
  if (!out || n < 2 || edge_factor < 1) return I2_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  int scale = 1;
  while ((1LL << scale) < n) ++scale;
  return generate_rmat(n, scale, (long long)edge_factor << scale, a, b, c, seed, weighted, out);
}

extern "C" int i2_graph_generate_er(int n, long long m, uint64_t seed, int weighted, i2_graph** out) {
  if (!out || n < 2 || m < 0) return I2_ERR_ARG;
  const long long maxm = (long long)n * (n - 1) / 2;
  if (m > maxm || 2 * m > 0x7fffffffLL) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  Scratch sc;
  unsigned long long *pairs = nullptr, *k0 = nullptr, *k1 = nullptr;
  cudaError_t e = sc.get(&pairs, sizeof(unsigned long long) * std::max(1LL, m));
  if (e != cudaSuccess) return cuda_status(e);
  // the host generator's candidate counts: m + m/16 + 64, growing by a quarter, until past 8 (m + 64)
  int st = first_distinct(m, m + m / 16 + 64, 8 * (m + 64),
                          [&](long long C, unsigned long long* keys, unsigned long long* idx) {
                            k_er_candidates<<<4096, 256>>>(seed, n, 0, C, keys, idx);
                          },
                          pairs);
  if (st) return st;
  e = sc.get(&k0, sizeof(unsigned long long) * std::max(1LL, 2 * m));
  if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * std::max(1LL, 2 * m));
  if (e != cudaSuccess) return cuda_status(e);
  k_both_directions<<<4096, 256>>>(pairs, m, k0);
  return csr_from_keys(k0, k1, nullptr, nullptr, 2 * m, n, CutWeights{weighted ? 1 : 0, seed, nullptr}, out);
}

extern "C" int i2_graph_generate_grid(int side, double remove_frac, double add_frac, uint64_t seed, int weighted,
                                      i2_graph** out) {
  if (!out || side < 2 || remove_frac < 0 || remove_frac >= 1 || add_frac < 0) return I2_ERR_ARG;
  const long long V = (long long)side * side;
  if (V > 0x7fffffffLL) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  const long long H = (long long)side * (side - 1);
  const long long G = 2 * H;
  const uint64_t drop = prob_to_u64(remove_frac);
  Scratch sc;
  unsigned long long* d_kept = nullptr;
  cudaError_t e = sc.get(&d_kept, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(d_kept, 0, sizeof(unsigned long long));
  if (e != cudaSuccess) return cuda_status(e);
  k_grid_count<<<4096, 256>>>(seed, drop, G, d_kept);
  unsigned long long kept = 0;
  e = cudaMemcpy(&kept, d_kept, sizeof(kept), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  const long long K = std::llround(add_frac * (double)kept);
  const long long nkeys = 2 * G + 2 * K;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  e = sc.get(&k0, sizeof(unsigned long long) * nkeys);
  if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * nkeys);
  if (e != cudaSuccess) return cuda_status(e);
  k_grid_keys<<<4096, 256>>>(seed, side, drop, G, k0);
  if (K > 0) {
    unsigned long long* extra = nullptr;
    e = sc.get(&extra, sizeof(unsigned long long) * K);
    if (e != cudaSuccess) return cuda_status(e);
    // the host draws candidates until K new pairs are found; a stream that
    // dries up within 64 (K + 64) candidates is refused
    int st = first_distinct(K, K + K / 8 + 64, 64 * (K + 64),
                            [&](long long C, unsigned long long* keys, unsigned long long* idx) {
                              k_grid_extra_candidates<<<4096, 256>>>(seed, side, drop, C, keys, idx);
                            },
                            extra);
    if (st) return st;
    k_both_directions<<<4096, 256>>>(extra, K, k0 + 2 * G);
  }
  return csr_from_keys(k0, k1, nullptr, nullptr, nkeys, (int)V, CutWeights{weighted ? 1 : 0, seed, nullptr}, out);
}

extern "C" int i2_graph_from_coo_device(int nodes, long long m, const int* src, const int* dst, const int* w,
                                        int symmetrize, i2_graph** out) {
  if (!out || nodes < 1 || m < 0 || (m > 0 && (!src || !dst))) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  const long long nkeys = (symmetrize ? 2 : 1) * m;
  if (nkeys > 0x7fffffffLL) return I2_ERR_OVERFLOW;
  if (m > 0 && (!device_range_ok(src, sizeof(int) * (size_t)m) || !device_range_ok(dst, sizeof(int) * (size_t)m) ||
                (w && !device_range_ok(w, sizeof(int) * (size_t)m))))
    return I2_ERR_ARG;
  Scratch sc;
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  int *w0 = nullptr, *w1 = nullptr, *bad = nullptr;
  const size_t nk = (size_t)std::max(1LL, nkeys);
  cudaError_t e = sc.get(&k0, sizeof(unsigned long long) * nk);
  if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * nk);
  if (e == cudaSuccess && w) e = sc.get(&w0, sizeof(int) * nk);
  if (e == cudaSuccess && w) e = sc.get(&w1, sizeof(int) * nk);
  if (e == cudaSuccess) e = sc.get(&bad, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(bad, 0, sizeof(int));
  if (e != cudaSuccess) return cuda_status(e);
  if (m > 0) k_coo_keys<<<4096, 256>>>(src, dst, w, m, nodes, symmetrize ? 1 : 0, k0, w0, bad);
  int hbad = 0;
  e = cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e);
  if (hbad) return I2_ERR_FORMAT;
  return csr_from_keys(k0, k1, w0, w1, nkeys, nodes, CutWeights{w ? 2 : 0, 0, nullptr}, out);
}

// ---------------------------------------------------------------------------
// Degree-ordered copy of a graph: vertex IDs renumbered by descending degree
// (ties by ascending ID), so that the few vertices most adjacency lists name
// sit together at the front of every per-vertex array. On RMAT the generator
// scatters its hubs over the whole ID range, and once dist[] outgrows L2 (2^25
// vertices and more) the neighbours' random dist reads and atomicMins miss;
// renumbered, the vertices that take most of those accesses fit in L2.

namespace i2 {
namespace {

__global__ void k_degree_ids(const int* __restrict__ nindex, int n, int* __restrict__ deg, int* __restrict__ ids) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    deg[v] = nindex[v + 1] - nindex[v];
    ids[v] = v;
  }
}

__global__ void k_invert(const int* __restrict__ perm, int n, int* __restrict__ inv) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) inv[perm[i]] = i;
}

// One warp per vertex (grid-stride): every CSR entry e of old vertex u becomes
// the key (inv[u] << 32 | inv[nlist[e]]) at position e, its weight beside it.
__global__ void k_relabel_keys(const int* __restrict__ nindex, const int* __restrict__ nlist,
                               const int* __restrict__ w, const int* __restrict__ inv, int n,
                               unsigned long long* __restrict__ keys, int* __restrict__ wk) {
  const int lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long u = warp; u < n; u += nwarps) {
    const unsigned long long hi = (unsigned long long)(unsigned)inv[u] << 32;
    const int beg = nindex[u], end = nindex[u + 1];
    for (int e = beg + lane; e < end; e += 32) {
      const int v = nlist[e];  // in range in every graph handle; dropped if not
      keys[e] = (unsigned)v < (unsigned)n ? (hi | (unsigned)inv[v]) : kDropKey;
      if (w) wk[e] = w[e];
    }
  }
}

}  // namespace

int degree_ordered_copy(const i2_graph* g, i2_graph** twin, int** inv_out) {
  *twin = nullptr;
  *inv_out = nullptr;
  int n = 0, E = 0;
  const int *nindex = nullptr, *nlist = nullptr, *w = nullptr;
  int st = graph_device_csr(g, &n, &E, &nindex, &nlist, &w);
  if (st) return st;
  Scratch sc;
  int *deg = nullptr, *ids = nullptr, *deg_sorted = nullptr, *perm = nullptr;
  void* tmp = nullptr;
  size_t tb = 0;
  cudaError_t e = sc.get(&deg, sizeof(int) * (size_t)n);
  if (e == cudaSuccess) e = sc.get(&ids, sizeof(int) * (size_t)n);
  if (e == cudaSuccess) e = sc.get(&deg_sorted, sizeof(int) * (size_t)n);
  if (e == cudaSuccess) e = sc.get(&perm, sizeof(int) * (size_t)n);
  if (e == cudaSuccess) e = cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, deg, deg_sorted, ids, perm, n);
  if (e == cudaSuccess) e = sc.get(&tmp, tb);
  if (e != cudaSuccess) return cuda_status(e);
  k_degree_ids<<<1024, 256>>>(nindex, n, deg, ids);
  // LSD radix sort is stable: equal degrees keep ascending IDs
  e = cub::DeviceRadixSort::SortPairsDescending(tmp, tb, deg, deg_sorted, ids, perm, n);
  int* inv = nullptr;
  if (e == cudaSuccess) e = dev_alloc(&inv, sizeof(int) * (size_t)n);
  if (e != cudaSuccess) return cuda_status(e);
  k_invert<<<1024, 256>>>(perm, n, inv);
  unsigned long long *k0 = nullptr, *k1 = nullptr;
  int *w0 = nullptr, *w1 = nullptr;
  const size_t nk = (size_t)(E > 0 ? E : 1);
  e = sc.get(&k0, sizeof(unsigned long long) * nk);
  if (e == cudaSuccess) e = sc.get(&k1, sizeof(unsigned long long) * nk);
  if (e == cudaSuccess && w) e = sc.get(&w0, sizeof(int) * nk);
  if (e == cudaSuccess && w) e = sc.get(&w1, sizeof(int) * nk);
  if (e == cudaSuccess) {
    k_relabel_keys<<<4096, 256>>>(nindex, nlist, w, inv, n, k0, w0);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    dev_free(inv);
    return cuda_status(e);
  }
  st = csr_from_keys(k0, k1, w0, w1, E, n, CutWeights{w ? 2 : 0, 0, nullptr}, twin);
  if (st) {
    dev_free(inv);
    return st;
  }
  *inv_out = inv;
  return I2_OK;
}

}  // namespace i2
