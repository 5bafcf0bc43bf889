// B200 relaxation engine: device graphs, traversal runs and the C ABI of
// include/i2b200.h for BFS, SSSP and CC.
//
// A traversal is: reset the control block, fill dist/labels and seed F_0
// (k_fill, k_seed), then one relax launch per iteration until the frontier is
// empty (the do-while of the reference's host drivers, e.g.
// BFS_CUDA_V_Data_Push_..._Warp_..._NonDup.cu:112-122). In the default loop
// mode (I2_LOOP_GRAPH) the whole sequence is one CUDA graph whose WHILE
// conditional node holds one cooperative relax launch that runs every
// iteration itself, its blocks meeting at a bounded barrier between
// iterations (relax_resident, resident.cu). I2_LOOP_RELAUNCH keeps one launch
// per iteration inside the graph: the fixed style's kernel, or the dispatch
// kernel whose blocks branch on the style picked for this iteration. Either
// way the last block of an iteration picks the next style and sets the loop
// condition on the device, so there is no host round trip per iteration.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include "../../include/i2b200.h"
#include "common.cuh"
#include "engine.h"
#include "host_graph.h"
#include "mlp.cuh"
#include "relax.cuh"
#include "iteration.cuh"

namespace i2 {

static_assert(sizeof(IterRec) == sizeof(i2_iter_record), "record layout");
static_assert((int)kNumVariants == (int)I2_NUM_VARIANTS, "variant count");

// ---------------------------------------------------------------------------
// Init kernels.

// dist[v] = INF (BFS/SSSP) or v (CC). For CC every vertex enters F_0.
template <int ALG>
__global__ void __launch_bounds__(kBlock) k_fill(Ctx c) {
  __shared__ Stage s;
  stage_init(s);
  Acc a;
  acc_init(a);
  __syncthreads();
  const int V = c.g.nodes;
  for (long long base = (long long)blockIdx.x * kBlock; base < V; base += (long long)gridDim.x * kBlock) {
    const int v = (int)base + threadIdx.x;
    const bool in = v < V;
    constexpr bool kAll = ALG == kCC || ALG == kMIS;  // every vertex starts in F_0
    const int deg = (kAll && in) ? c.g.nindex[v + 1] - c.g.nindex[v] : 0;
    // MIS: a vertex without neighbours is in the set at once
    if (in) c.dist[v] = ALG == kCC ? v : ALG == kMIS ? (deg == 0 ? kMisIn : kMisUndecided) : kInf;
    if (kAll) {
      const bool put = in && deg > 0;  // vertices without edges are already final
      const unsigned word = __ballot_sync(0xffffffffu, put);
      if ((threadIdx.x & 31) == 0 && word) c.bm[0][v >> 5] = word;
      if (put) {
        a.mindist = min(a.mindist, v);
        stage_entry(c, s, a, 0, v, deg);
      }
      stage_flush(c, s, 0);
    }
  }
  if (ALG == kCC || ALG == kMIS) {
    stage_flush(c, s, 0);
    acc_reduce(a, s);
    if (threadIdx.x == 0) {
      const Acc& r = s.red[0];
      Slot& sl = c.ctl->slot[0];
      if (r.maxdeg) atomicMax(&sl.maxdeg, r.maxdeg);
      if (r.mindist != kInf) atomicMin(&sl.mindist, r.mindist);
    }
  }
}

// One block: seed the sources (BFS/SSSP) and select the first variant.
template <int ALG>
__global__ void __launch_bounds__(kBlock) k_seed(Ctx c) {
  Ctl* ctl = c.ctl;
  if (ALG != kCC && ALG != kMIS) {
    const int ns = c.srcs ? ctl->nsrc : 1;
    for (int j = threadIdx.x; j < ns; j += blockDim.x) {
      const int v = c.srcs ? c.srcs[j] : ctl->src;
      const int deg = c.g.nindex[v + 1] - c.g.nindex[v];
      const unsigned bit = 1u << (v & 31);
      if (atomicOr(&c.bm[0][v >> 5], bit) & bit) continue;
      c.dist[v] = 0;
      atomicAdd((unsigned long long*)&ctl->visited, 1ull);
      Slot& sl = ctl->slot[0];
      atomicMin(&sl.mindist, 0);
      if (deg == 0) {
        atomicAnd(&c.bm[0][v >> 5], ~bit);  // nothing to propagate
        continue;
      }
      atomicMax(&sl.maxdeg, deg);
      const unsigned long long b = atomicAdd(&sl.packed, (1ull << 32) | (unsigned)deg);
      c.wl[0][slot_size(b)] = v;
      c.woff[0][slot_size(b)] = slot_edges(b);
      if (deg >= c.heavy) {
        const int t = heavy_tiles(deg);
        const unsigned long long hb = atomicAdd(&sl.hpacked, (1ull << 32) | (unsigned)t);
        c.hwl[0][slot_size(hb)] = v;
        c.htoff[0][slot_size(hb)] = slot_edges(hb);
      }
    }
  } else if (threadIdx.x == 0) {
    ctl->visited = c.g.nodes;
  }
  __threadfence();
  __syncthreads();
  select_next(c, 0, 0, true, -1);
}

// Per-run parameters, passed by value to k_reset so that queued runs never
// share a host buffer.
struct RunParams {
  int algo, mode, fixed_variant, allowed, src, nsrc, iter_cap, delta, hold, stall_ms, then_at, then_variant, hshift;
  bool operator!=(const RunParams& o) const { return std::memcmp(this, &o, sizeof(RunParams)) != 0; }
};

__global__ void k_reset(Ctl* ctl, RunParams p) {
  if (threadIdx.x != 0) return;
  unsigned* w = reinterpret_cast<unsigned*>(ctl);
  for (unsigned k = 0; k < sizeof(Ctl) / sizeof(unsigned); ++k) w[k] = 0u;
  for (int k = 0; k < 3; ++k) ctl->slot[k].mindist = kInf;
  ctl->tstart = ~0ull;
  ctl->iter_cap = p.iter_cap;
  ctl->mode = p.mode;
  ctl->fixed_variant = p.fixed_variant;
  ctl->variant = p.fixed_variant;
  ctl->allowed = p.allowed;
  ctl->src = p.src;
  ctl->nsrc = p.nsrc;
  ctl->algo = p.algo;
  ctl->delta = p.delta;
  ctl->hshift = p.hshift;
  ctl->then_at = p.then_at;
  ctl->then_variant = p.then_variant;
  ctl->hold = p.hold;
  ctl->stall_ns = (unsigned long long)p.stall_ms * 1000000ull;
  ctl->threshold = p.delta > 0 ? p.delta : kInf;  // sources start at 0
  ctl->pmin[0] = kInf;
  ctl->pmin[1] = kInf;
}

// ---------------------------------------------------------------------------
// Graph maintenance kernels.

// *best = the smallest vertex of degree maxdeg.
__global__ void k_hub(DGraph g, int maxdeg, int* best) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int b = INT_MAX;
  for (long long v = tid; v < g.nodes; v += stride)
    if (g.nindex[v + 1] - g.nindex[v] == maxdeg) {
      b = (int)v;
      break;  // later vertices of this thread are larger
    }
  for (int o = 16; o > 0; o >>= 1) b = min(b, __shfl_down_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0 && b != INT_MAX) atomicMin(best, b);
}

// Sets bit 8 of *bad when a weight is negative (SSSP needs weights >= 0).
__global__ void k_negative_weights(const int* w, long long n, int* bad) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int neg = 0;
  for (long long e = tid; e < n; e += stride) neg |= w[e] < 0;
  if (__any_sync(0xffffffffu, neg) && (threadIdx.x & 31) == 0) atomicOr(bad, 8);
}

__global__ void k_validate(DGraph g, int* bad) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long v = tid; v < g.nodes; v += stride)
    if (g.nindex[v + 1] < g.nindex[v]) atomicOr(bad, 1);
  for (long long e = tid; e < g.edges; e += stride)
    if ((unsigned)g.nlist[e] >= (unsigned)g.nodes) atomicOr(bad, 2);
  if (tid == 0 && (g.nindex[0] != 0 || g.nindex[g.nodes] != g.edges)) atomicOr(bad, 4);
}

struct DevStats {
  int maxdeg;
  int nheavy;
  int wmin;
  int unsorted;
  int asym;
  int pad;
  double sumsq;
  double wsum;
};

__global__ void k_degree_stats(DGraph g, int heavy, DevStats* st) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int mx = 0, nh = 0, uns = 0;
  double s2 = 0.0;
  for (long long v = tid; v < g.nodes; v += stride) {
    const int b = g.nindex[v], e = g.nindex[v + 1];
    const int d = e - b;
    mx = max(mx, d);
    nh += d >= heavy;
    s2 += (double)d * d;
  }
  int wmin = INT_MAX;
  double ws = 0.0;
  if (g.eweight)
    for (long long e = tid; e < g.edges; e += stride) {
      const int w = g.eweight[e];
      wmin = min(wmin, w);
      ws += (double)w;
    }
  atomicMax(&st->maxdeg, mx);
  atomicAdd(&st->wsum, ws);
  atomicAdd(&st->nheavy, nh);
  atomicMin(&st->wmin, wmin);
  if (uns) atomicOr(&st->unsorted, 1);
  atomicAdd(&st->sumsq, s2);
}

// Adjacency lists strictly increasing (sorted, no duplicates)? One thread per
// CSR entry, using the starting-point array for the entry's row.
__global__ void k_sorted(DGraph g, const int* __restrict__ sp, DevStats* st) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int uns = 0;
  for (long long e = 1 + tid; e < g.edges; e += stride)
    uns |= (sp[e] == sp[e - 1]) && (g.nlist[e] <= g.nlist[e - 1]);
  if (uns) atomicOr(&st->unsorted, 1);
}

// For every entry (u, v, w): is (v, u, w) present? One thread per entry,
// binary search in v's sorted adjacency.
__global__ void k_symmetry(DGraph g, const int* __restrict__ sp, DevStats* st) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  int asym = 0;
  for (long long k = tid; k < g.edges && !asym; k += stride) {
    const int u = sp[k];
    const int v = g.nlist[k];
    int lo = g.nindex[v], hi = g.nindex[v + 1] - 1, pos = -1;
    while (lo <= hi) {
      const int mid = lo + ((hi - lo) >> 1);  // lo + hi may exceed INT_MAX
      if ((unsigned)mid >= (unsigned)g.edges) {
        asym = 1;  // cannot happen on a validated CSR; refuse rather than read out of bounds
        break;
      }
      const int x = g.nlist[mid];
      if (x == u) { pos = mid; break; }
      if (x < u) lo = mid + 1; else hi = mid - 1;
    }
    if (pos < 0 || (g.eweight && g.eweight[pos] != g.eweight[k])) asym = 1;
  }
  if (asym) atomicOr(&st->asym, 1);
}

// sp[k] = row of CSR entry k; one warp per vertex, coalesced stores.
__global__ void k_build_sp(DGraph g, int* sp) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (long long v = warp; v < g.nodes; v += nwarps)
    for (long long k = g.nindex[v] + lane; k < g.nindex[v + 1]; k += 32) sp[k] = (int)v;
}

// Reference synthetic weights (include/sssp_vertex_cuda.h:127-137) on the device.
__global__ void k_synth_weights(DGraph g, int* w) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = tid; i < g.nodes; i += stride)
    for (int j = g.nindex[i]; j < g.nindex[i + 1]; ++j) {
      const int prod = (int)((unsigned)i * (unsigned)g.nlist[j]);
      int x = 1 + (prod % g.nodes);
      w[j] = x < 0 ? -x : x;
    }
}

// Reached vertices and the sum of their degrees (E_r).
__global__ void k_reached(DGraph g, const int* dist, unsigned long long* out) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned long long nv = 0, ne = 0;
  for (long long v = tid; v < g.nodes; v += stride)
    if (dist[v] != kInf) {
      nv++;
      ne += (unsigned long long)(g.nindex[v + 1] - g.nindex[v]);
    }
  for (int o = 16; o > 0; o >>= 1) {
    nv += __shfl_down_sync(0xffffffffu, nv, o);
    ne += __shfl_down_sync(0xffffffffu, ne, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], nv);
    atomicAdd(&out[1], ne);
  }
}

// Values of a traversal on the degree-ordered copy, back in original IDs:
// out[v] = copy[inv[v]] (coalesced inv read and write, gathered copy read).
__global__ void k_unpermute(const int* __restrict__ copy, const int* __restrict__ inv, int n,
                            int* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) out[v] = copy[inv[v]];
}

// CC on the degree-ordered copy labels each vertex with its component's
// smallest copy ID; the caller's labels are the smallest original IDs. First
// mn[r] = min { v : label of copy vertex inv[v] is r } (one atomicMin per
// distinct label in a warp, by its lowest lane, which holds the smallest v
// since a warp covers consecutive v; skipped when mn[r] is already smaller,
// as it soon is for the giant component), then out[v] = mn[label(inv[v])].
__global__ void k_cc_min_init(int* __restrict__ mn, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) mn[v] = INT_MAX;
}

__global__ void k_cc_min_original(const int* __restrict__ copy_label, const int* __restrict__ inv, int n,
                                  int* mn) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) {
    const int r = copy_label[inv[v]];
    const unsigned peers = __match_any_sync(__activemask(), r);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1 && v < *(volatile int*)&mn[r]) atomicMin(&mn[r], v);
  }
}

__global__ void k_cc_labels(const int* __restrict__ copy_label, const int* __restrict__ inv,
                            const int* __restrict__ mn, int n, int* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += stride) out[v] = mn[copy_label[inv[v]]];
}

// ---------------------------------------------------------------------------
// Kernel tables.

typedef void (*KernelFn)(Ctx);

template <int ALG>
static KernelFn relax_fn(int v) {
  switch (v) {
    case kVPThread: return relax_push<ALG, kVPThread>;
    case kVPWarp: return relax_push<ALG, kVPWarp>;
    case kVPCta: return relax_edge_balanced<ALG>;
    case kVPBlock: return relax_push<ALG, kVPBlock>;
    case kPullFrontier: return relax_pull<ALG, true>;
    case kPullTopo: return relax_pull<ALG, false>;
    case kEdgeTopo: return relax_edge_topo<ALG>;
    case kPushTopo: return relax_push_topo<ALG>;
    case kUnionFind:
      if constexpr (ALG == kCC) return relax_union<ALG>;
      return nullptr;
  }
  return nullptr;
}

// The selectors' per-iteration kernel; `wide`: the form compiled for the fixed
// styles' resident blocks per SM (graphs of kWideSelectorNodes vertices or more).
static KernelFn dispatch_kernel(int algo, bool wide) {
  if (algo == kBFS) return wide ? relax_dispatch<kBFS, I2_EB_MIN_BLOCKS> : relax_dispatch<kBFS>;
  if (algo == kSSSP) return wide ? relax_dispatch<kSSSP, I2_EB_MIN_BLOCKS> : relax_dispatch<kSSSP>;
  return wide ? relax_dispatch<kCC, I2_EB_MIN_BLOCKS> : relax_dispatch<kCC>;  // MIS never dispatches
}

KernelFn relax_kernel(int algo, int v, bool near_far) {
  if (near_far && algo == kSSSP && v == kVPCta) return relax_near_far;
  if (algo == kBFS) return relax_fn<kBFS>(v);
  if (algo == kSSSP) return relax_fn<kSSSP>(v);
  if (algo == kCC) return relax_fn<kCC>(v);
  return relax_mis;  // one style
}

static KernelFn fill_kernel(int algo) {
  if (algo == kBFS) return k_fill<kBFS>;
  if (algo == kSSSP) return k_fill<kSSSP>;
  if (algo == kCC) return k_fill<kCC>;
  return k_fill<kMIS>;
}
static KernelFn seed_kernel(int algo) {
  if (algo == kBFS) return k_seed<kBFS>;
  if (algo == kSSSP) return k_seed<kSSSP>;
  if (algo == kCC) return k_seed<kCC>;
  return k_seed<kMIS>;
}

// ---------------------------------------------------------------------------
// Device state helpers.

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return I2_OK;
  if (e == cudaErrorMemoryAllocation) return I2_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return I2_ERR_NO_DEVICE;
  return I2_ERR_CUDA;
}

#define I2_CK(call)                         \
  do {                                      \
    cudaError_t e_ = (call);                \
    if (e_ != cudaSuccess) {                \
      cudaGetLastError();                   \
      return cuda_status(e_);               \
    }                                       \
  } while (0)

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

// Preferred shared-memory carveout (percent of the unified L1/shared storage)
// for the relax kernels; -1 leaves the choice to the driver. A large carveout
// costs L1 capacity, which the adjacency reads use.
static int g_carveout = -1;

int grid_for(KernelFn fn, int max_per_sm) {
  cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout, g_carveout);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, (const void*)fn, kBlock, 0);
  per = std::max(1, std::min(per, max_per_sm));
  return per * sm_count();
}

// Per-device selector parameters.
static std::mutex g_mlp_mu;
static float* g_mlp_dev[64] = {nullptr};

const float* mlp_device_params() {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_mlp_mu);
  return (dev >= 0 && dev < 64) ? g_mlp_dev[dev] : nullptr;
}

int mlp_install(const float* params, int count) {
  if (!params || count != kParams) return I2_ERR_ARG;
  int dev = 0;
  I2_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return I2_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_mlp_mu);
  if (!g_mlp_dev[dev]) I2_CK(cudaMalloc(&g_mlp_dev[dev], sizeof(float) * kParams));
  I2_CK(cudaMemcpy(g_mlp_dev[dev], params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  return I2_OK;
}

}  // namespace i2

using namespace i2;

// ---------------------------------------------------------------------------
// Graph handle.

struct ExecKey {
  int algo, mode, variant, multi, near_far, resident;
  bool operator<(const ExecKey& o) const {
    if (algo != o.algo) return algo < o.algo;
    if (mode != o.mode) return mode < o.mode;
    if (variant != o.variant) return variant < o.variant;
    if (multi != o.multi) return multi < o.multi;
    if (near_far != o.near_far) return near_far < o.near_far;
    return resident < o.resident;
  }
};

struct ExecEntry {
  cudaGraphExec_t ex = nullptr;
  cudaGraphNode_t reset = nullptr;
  RunParams last{};
  Ctx ctx{};
};

struct i2_graph {
  DGraph g{};
  GStats gs{};
  int device = 0;
  bool owns = false;
  int* d_nindex = nullptr;
  int* d_nlist = nullptr;
  int* d_eweight = nullptr;
  bool owns_weights = false;
  int* d_sp = nullptr;
  int heavy = 4096;
  int blocks_per_sm = 8;  // cap; the occupancy of each kernel decides below it
  // workspace
  bool ws_ready = false;
  int* dist = nullptr;
  int* wl[3] = {nullptr, nullptr, nullptr};
  unsigned* woff[3] = {nullptr, nullptr, nullptr};
  int* hwl[3] = {nullptr, nullptr, nullptr};
  unsigned* htoff[3] = {nullptr, nullptr, nullptr};
  unsigned* bm[3] = {nullptr, nullptr, nullptr};
  unsigned* fbm = nullptr;  // far-pile bitmap, allocated after bm[2]
  unsigned long long* hist = nullptr;  // near/far distance histograms, after fbm
  int* pile[2] = {nullptr, nullptr};
  int bm_words = 0;
  bool resident_ok = true;  // cleared if the device refuses the cooperative loop node
  Ctl* ctl = nullptr;
  IterRec* recs = nullptr;
  int rec_cap = 0;
  int* srcs = nullptr;
  int srcs_cap = 0;
  unsigned long long* reach = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, ev3 = nullptr;
  Ctl* h_ctl = nullptr;  // pinned
  std::map<ExecKey, ExecEntry> execs;
  std::vector<cudaGraph_t> graphs;
  int last_iters = 0;
  // sweep scratch
  int* snap_dist = nullptr;
  unsigned* snap_bm = nullptr;
  int* snap_wl = nullptr;
  int* snap_hwl = nullptr;
  // degree-ordered copy (i2_graph_reorder): BFS and SSSP run on it, their
  // sources mapped by inv and their results gathered back to original IDs
  i2_graph* twin = nullptr;
  int* d_inv = nullptr;         // original ID -> copy's ID (device)
  std::vector<int> h_inv;       // the same on the host, to map sources
  bool last_on_twin = false;    // the last traversal ran on the copy (records)
};

namespace i2 {

// ---------------------------------------------------------------------------
// Device memory pool and pinned control blocks.

namespace {
struct DevPool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t s = nullptr;  // allocations and frees are ordered on it
};
std::mutex g_pool_mu;
DevPool g_pools[64];
std::mutex g_ctl_mu;
std::vector<Ctl*> g_ctl_free;  // pinned host control blocks of freed graphs
}  // namespace

static DevPool* dev_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_pool_mu);
  DevPool& p = g_pools[dev];
  if (!p.pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaStream_t s = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    unsigned long long keep = ~0ull;  // never hand reserved memory back on its own
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      cudaMemPoolDestroy(pool);
      return nullptr;
    }
    p.pool = pool;
    p.s = s;
  }
  return &p;
}

cudaError_t dev_alloc_bytes(void** ptr, size_t bytes) {
  *ptr = nullptr;
  DevPool* p = dev_pool();
  if (!p) return cudaErrorInitializationError;
  cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes, p->pool, p->s);
  if (e == cudaErrorMemoryAllocation) {
    // Reserved but unused blocks may be too fragmented to serve the request:
    // hand them back and try once more.
    cudaGetLastError();
    cudaStreamSynchronize(p->s);
    cudaMemPoolTrimTo(p->pool, 0);
    e = cudaMallocFromPoolAsync(ptr, bytes, p->pool, p->s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->s);  // usable by every stream from here
  if (e != cudaSuccess) *ptr = nullptr;
  return e;
}

void dev_free(void* ptr) {
  if (!ptr) return;
  DevPool* p = dev_pool();
  if (!p) return;
  cudaDeviceSynchronize();
  cudaFreeAsync(ptr, p->s);
}

static int trim_pool() {
  DevPool* p = dev_pool();
  if (!p) return I2_ERR_NO_DEVICE;
  I2_CK(cudaStreamSynchronize(p->s));
  I2_CK(cudaMemPoolTrimTo(p->pool, 0));
  return I2_OK;
}

static cudaError_t ctl_host_get(Ctl** out) {
  {
    std::lock_guard<std::mutex> lk(g_ctl_mu);
    if (!g_ctl_free.empty()) {
      *out = g_ctl_free.back();
      g_ctl_free.pop_back();
      return cudaSuccess;
    }
  }
  return cudaMallocHost(out, sizeof(Ctl));
}

static void ctl_host_put(Ctl* c) {
  if (!c) return;
  std::lock_guard<std::mutex> lk(g_ctl_mu);
  g_ctl_free.push_back(c);
}

static void drop_execs(i2_graph* g) {
  for (auto& kv : g->execs) cudaGraphExecDestroy(kv.second.ex);
  g->execs.clear();
}

static void free_graph_state(i2_graph* g) {
  drop_execs(g);
  for (auto gr : g->graphs) cudaGraphDestroy(gr);
  g->graphs.clear();
  dev_free(g->dist);
  for (int k = 0; k < 3; ++k) {
    dev_free(g->wl[k]);
    dev_free(g->woff[k]);
    dev_free(g->hwl[k]);
    dev_free(g->htoff[k]);
  }
  dev_free(g->bm[0]);
  dev_free(g->pile[0]);
  dev_free(g->pile[1]);
  dev_free(g->ctl);
  dev_free(g->recs);
  dev_free(g->srcs);
  dev_free(g->reach);
  dev_free(g->snap_dist);
  dev_free(g->snap_bm);
  dev_free(g->snap_wl);
  dev_free(g->snap_hwl);
  if (g->h_ctl) ctl_host_put(g->h_ctl);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  if (g->ev2) cudaEventDestroy(g->ev2);
  if (g->ev3) cudaEventDestroy(g->ev3);
  if (g->stream) cudaStreamDestroy(g->stream);
  dev_free(g->d_sp);
  if (g->twin) i2_graph_free(g->twin);
  g->twin = nullptr;
  dev_free(g->d_inv);
  g->d_inv = nullptr;
  if (g->owns) {
    dev_free(g->d_nindex);
    dev_free(g->d_nlist);
  }
  if (g->owns || g->owns_weights) dev_free(g->d_eweight);
}

static int compute_stats(i2_graph* g) {
  DevStats* st = nullptr;
  I2_CK(dev_alloc(&st, sizeof(DevStats)));
  DevStats h{};
  h.wmin = INT_MAX;
  cudaMemcpy(st, &h, sizeof(h), cudaMemcpyHostToDevice);
  const int grid = 4 * sm_count();
  k_degree_stats<<<grid, 256, 0, g->stream>>>(g->g, g->heavy, st);
  cudaStreamSynchronize(g->stream);
  cudaMemcpy(&h, st, sizeof(h), cudaMemcpyDeviceToHost);
  cudaError_t e = cudaGetLastError();
  dev_free(st);
  if (e != cudaSuccess) return cuda_status(e);
  GStats& s = g->gs;
  s.nodes = g->g.nodes;
  s.edges = g->g.edges;
  s.maxdeg = h.maxdeg;
  s.nheavy = h.nheavy;
  s.wmin = g->g.eweight ? (h.wmin == INT_MAX ? 1 : h.wmin) : 1;
  s.symmetric = -1;  // decided on first need (ensure_symmetry)
  const double mean = (double)g->g.edges / (double)g->g.nodes;
  const double var = std::max(0.0, h.sumsq / (double)g->g.nodes - mean * mean);
  s.avgdeg = (float)mean;
  s.degcv = mean > 0 ? (float)(std::sqrt(var) / mean) : 0.f;
  s.wmean = (g->g.eweight && g->g.edges > 0) ? (float)(h.wsum / (double)g->g.edges) : 1.f;
  return I2_OK;
}

static int finish_setup(i2_graph* g) {
  I2_CK(cudaGetDevice(&g->device));
  I2_CK(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
  I2_CK(cudaEventCreate(&g->ev0));
  I2_CK(cudaEventCreate(&g->ev1));
  I2_CK(cudaEventCreate(&g->ev2));
  I2_CK(cudaEventCreate(&g->ev3));
  I2_CK(ctl_host_get(&g->h_ctl));
  g->g.vec_ok = ((((uintptr_t)g->g.nlist) & 15) == 0 && (((uintptr_t)g->g.eweight) & 15) == 0) ? 1 : 0;
  return compute_stats(g);
}

// Words of the bitmap block: 4 bitmaps, then (8-byte aligned) the two
// distance histograms of the budgeted near/far ordering.
static size_t hist_offset_words(const i2_graph* g) { return (4ull * g->bm_words + 1) & ~1ull; }
static size_t bm_block_words(const i2_graph* g) { return hist_offset_words(g) + 2ull * 2 * kHistBins; }

static int ensure_workspace(i2_graph* g) {
  if (g->ws_ready) return I2_OK;
  const long long V = g->g.nodes;
  g->bm_words = (int)((V + 31) / 32);
  I2_CK(dev_alloc(&g->dist, sizeof(int) * V));
  for (int k = 0; k < 3; ++k) {
    I2_CK(dev_alloc(&g->wl[k], sizeof(int) * V));
    I2_CK(dev_alloc(&g->woff[k], sizeof(unsigned) * V));
    I2_CK(dev_alloc(&g->hwl[k], sizeof(int) * std::max(1, g->gs.nheavy)));
    I2_CK(dev_alloc(&g->htoff[k], sizeof(unsigned) * std::max(1, g->gs.nheavy)));
  }
  // one block: the three frontier bitmaps, the far-pile bitmap and the
  // near/far distance histograms (cleared together before every run)
  unsigned* bm = nullptr;
  I2_CK(dev_alloc(&bm, sizeof(unsigned) * bm_block_words(g)));
  for (int k = 0; k < 3; ++k) g->bm[k] = bm + (size_t)k * g->bm_words;
  g->fbm = bm + 3ull * g->bm_words;
  g->hist = reinterpret_cast<unsigned long long*>(bm + hist_offset_words(g));
  I2_CK(dev_alloc(&g->ctl, sizeof(Ctl)));
  g->rec_cap = (int)std::min<long long>(V + 2, 1 << 16);
  I2_CK(dev_alloc(&g->recs, sizeof(IterRec) * g->rec_cap));
  I2_CK(dev_alloc(&g->reach, sizeof(unsigned long long) * 2));
  g->ws_ready = true;
  return I2_OK;
}

static size_t pile_capacity(const i2_graph* g) { return (size_t)g->g.nodes + 1; }

static int ensure_piles(i2_graph* g) {
  if (g->pile[0]) return I2_OK;
  // each pile: nodes + 1 vertices, then their degrees (a full pile sends
  // vertices to the next frontier instead)
  for (int k = 0; k < 2; ++k) I2_CK(dev_alloc(&g->pile[k], sizeof(int) * 2 * pile_capacity(g)));
  drop_execs(g);  // graphs bake the context
  return I2_OK;
}

static int ensure_sp(i2_graph* g) {
  if (g->d_sp) return I2_OK;
  I2_CK(dev_alloc(&g->d_sp, sizeof(int) * ((size_t)g->g.edges + 4)));
  k_build_sp<<<8 * sm_count(), 256, 0, g->stream>>>(g->g, g->d_sp);
  I2_CK(cudaStreamSynchronize(g->stream));
  g->g.sp = g->d_sp;
  return I2_OK;
}

// Pull variants read a vertex's out-list as its in-list, so they need every
// (u, v, w) to have a (v, u, w) partner. Checked once, on first need.
static int ensure_symmetry(i2_graph* g) {
  if (g->gs.symmetric >= 0) return I2_OK;
  int st = ensure_sp(g);
  if (st) return st;
  DevStats* d = nullptr;
  I2_CK(dev_alloc(&d, sizeof(DevStats)));
  DevStats h{};
  cudaMemcpy(d, &h, sizeof(h), cudaMemcpyHostToDevice);
  const int grid = 8 * sm_count();
  k_sorted<<<grid, 256, 0, g->stream>>>(g->g, g->d_sp, d);
  cudaStreamSynchronize(g->stream);
  cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  if (!h.unsorted) {
    k_symmetry<<<grid, 256, 0, g->stream>>>(g->g, g->d_sp, d);
    cudaStreamSynchronize(g->stream);
    cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
  }
  cudaError_t e = cudaGetLastError();
  dev_free(d);
  if (e != cudaSuccess) return cuda_status(e);
  g->gs.symmetric = (!h.unsorted && !h.asym) ? 1 : 0;
  drop_execs(g);  // graphs bake the statistics into their arguments
  return I2_OK;
}

// Styles applicable to this graph and algorithm: pull and union-find read a
// vertex's out-list as its in-list (symmetric graphs only), the edge sweeps
// need sp[], and union-find computes CC labels only.
// Smallest graph (vertices) on which the selectors' union-find CC runs as
// union-find's own kernel (run_traversal).
constexpr long long kUnionFindKernelNodes = 1LL << 22;

// Whether the selectors run in the form compiled for more resident blocks.
static bool wide_selector(const i2_graph* g) { return (long long)g->g.nodes >= kWideSelectorNodes; }

static int allowed_mask(const i2_graph* g, int algo) {
  int m = 0;
  for (int v = 0; v < kNumVariants; ++v) m |= 1 << v;
  if (g->gs.symmetric != 1) m &= ~((1 << kPullFrontier) | (1 << kPullTopo) | (1 << kUnionFind));
  if (!g->d_sp) m &= ~(1 << kEdgeTopo);
  if (algo != I2_CC) m &= ~(1 << kUnionFind);
  return m;
}

static Ctx make_ctx(const i2_graph* g) {
  Ctx c{};
  c.g = g->g;
  c.gs = g->gs;
  c.dist = g->dist;
  for (int k = 0; k < 3; ++k) {
    c.wl[k] = g->wl[k];
    c.woff[k] = g->woff[k];
    c.hwl[k] = g->hwl[k];
    c.htoff[k] = g->htoff[k];
    c.bm[k] = g->bm[k];
  }
  c.ctl = g->ctl;
  c.recs = g->recs;
  c.rec_cap = g->rec_cap;
  c.heavy = g->heavy;
  c.bm_words = g->bm_words;
  c.pile_cap = (unsigned)std::min<size_t>(pile_capacity(g), 0xffffffffu);
  for (int k = 0; k < 2; ++k) {
    c.pile[k] = g->pile[k];
    c.pdeg[k] = g->pile[k] ? g->pile[k] + pile_capacity(g) : nullptr;
  }
  c.fbm = g->fbm;
  c.hist = g->hist;
  c.mlp = mlp_device_params();
  c.srcs = nullptr;
  return c;
}

// Default edge budget of the near/far ordering per SM (I2_SSSP_BUDGET_AUTO):
// about 7 warp tiles for each resident warp of the edge-balanced kernel.
// RMAT-22 SSSP (ms, device-timed): plain 2.57; budget 1M 2.95, 2M 2.57,
// 4M 2.38, 8M 2.60, 16M 2.97 edges.
constexpr int kBudgetEdgesPerSM = 28672;

// Near/far ordering applies to SSSP with the fixed edge-balanced push only
// (the style that implements the split launches). Returns the ordering's
// Ctl::delta: > 0 a fixed threshold step, < 0 minus an edge budget, 0 off.
// A fixed step relaxes up to 2.2x fewer edges on RMAT graphs, but the step
// that wins moves with the graph. The edge budget instead keeps each near
// frontier at about B edges: enough to fill the GPU, few enough that
// distances settle before their vertices relax.
// Smallest graph (CSR entries) on which the selectors' SSSP takes the budgeted
// ordering (skewed degrees only; see run_traversal).
constexpr long long kBudgetRuleEdges = 1LL << 26;

static int pick_order(const i2_graph* g, int algo, int mode, int variant, int step, int budget) {
  if (algo != I2_SSSP || mode != 0 || variant != kVPCta) return 0;
  if (step > 0) return step;
  if (budget == I2_SSSP_BUDGET_AUTO) {
    // Twice the budget on graphs of 2^30 CSR entries or more. RMAT-26 on its
    // degree-ordered copy, per traversal: 35.9 ms at the base budget (4.2 M
    // edges), 34.6 at 6 M, 34.1 at 8.4 M, 34.2 at 10 M, 35.7 at 12 M; on
    // RMAT-22 (2^27 entries) the base budget is the fastest.
    int b = std::max(1 << 16, sm_count() * kBudgetEdgesPerSM);
    if ((long long)g->g.edges >= (1LL << 30)) b *= 2;
    return -b;
  }
  if (budget > 0) return -budget;
  return 0;
}

// Histogram bin width of the edge budget: the largest power of two not above
// the smallest weight, the step by which distances grow per hop. (On RMAT-22
// with weights in [1, 255] most distances from the hub are below 32: the
// minimum over many paths takes the light edges, so bins sized by the mean
// weight put the whole budget quantile into the first bin.)
static int budget_shift(const i2_graph* g) {
  const int wm = g->gs.wmin > 1 ? g->gs.wmin : 1;
  int s = 0;
  while ((2LL << s) <= wm) ++s;  // floor(log2(wmin))
  return s;
}

static RunParams make_params(const i2_graph* g, int algo, int mode, int variant, int src, int nsrc, int cap,
                             int delta = 0) {
  RunParams p{};
  p.algo = algo;
  p.mode = mode;
  p.fixed_variant = variant < 0 ? 0 : variant;
  p.allowed = allowed_mask(g, algo);
  p.src = src;
  p.nsrc = nsrc;
  p.delta = delta;
  p.hshift = budget_shift(g);
  // Test hook: withhold the first barrier release of a resident traversal,
  // so that every block's bounded wait runs out (I2_STALL_MS bounds it).
  const char* hold = std::getenv("I2_TEST_HOLD_BARRIER");
  p.hold = (hold && hold[0] == '1') ? 1 : 0;
  const char* stall = std::getenv("I2_STALL_MS");
  p.stall_ms = stall ? std::max(1, std::atoi(stall)) : 10000;
  // a split launch moves at least one pile entry into a frontier, or learns
  // the pile's exact minimum for the next one
  p.iter_cap = cap > 0 ? cap : (int)std::min<long long>((long long)g->g.nodes * (delta != 0 ? 3 : 1) + 2, INT_MAX);
  return p;
}

static int add_kernel_node(cudaGraph_t gr, cudaGraphNode_t* node, const cudaGraphNode_t* deps, int ndeps,
                           KernelFn fn, int grid, Ctx* ctx) {
  cudaKernelNodeParams p{};
  p.func = (void*)fn;
  p.gridDim = dim3(grid);
  p.blockDim = dim3(kBlock);
  p.sharedMemBytes = 0;
  void* args[1] = {ctx};
  p.kernelParams = args;
  p.extra = nullptr;
  I2_CK(cudaGraphAddKernelNode(node, gr, deps, ndeps, &p));
  return I2_OK;
}

static int build_exec(i2_graph* g, int algo, int mode, int variant, bool multi, bool resident, const RunParams& rp,
                      ExecEntry** out) {
  ExecKey key{algo, mode, mode == 0 ? variant : -1, multi ? 1 : 0, rp.delta != 0 ? 1 : 0, resident ? 1 : 0};
  auto it = g->execs.find(key);
  if (it != g->execs.end()) {
    *out = &it->second;
    return I2_OK;
  }
  cudaGraph_t gr;
  I2_CK(cudaGraphCreate(&gr, 0));
  g->graphs.push_back(gr);
  cudaGraphConditionalHandle loop_h;
  I2_CK(cudaGraphConditionalHandleCreate(&loop_h, gr, 1, cudaGraphCondAssignDefault));
  Ctx c = make_ctx(g);
  c.srcs = multi ? g->srcs : nullptr;
  c.loop_h = (unsigned long long)loop_h;
  c.use_loop = 1;
  // bitmaps <- 0
  cudaGraphNode_t n_ms, n_reset, n_fill, n_seed, n_loop;
  cudaMemsetParams ms{};
  ms.dst = g->bm[0];
  ms.value = 0;
  ms.elementSize = 4;
  ms.width = bm_block_words(g);  // frontier and far-pile bitmaps, histograms
  ms.height = 1;
  ms.pitch = 0;
  I2_CK(cudaGraphAddMemsetNode(&n_ms, gr, nullptr, 0, &ms));
  // control block <- run parameters
  {
    cudaKernelNodeParams kp{};
    Ctl* ctl = g->ctl;
    RunParams p = rp;
    void* args[2] = {&ctl, &p};
    kp.func = (void*)k_reset;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    I2_CK(cudaGraphAddKernelNode(&n_reset, gr, &n_ms, 1, &kp));
  }
  int st = add_kernel_node(gr, &n_fill, &n_reset, 1, fill_kernel(algo), grid_for(fill_kernel(algo), 8), &c);
  if (st) return st;
  st = add_kernel_node(gr, &n_seed, &n_fill, 1, seed_kernel(algo), 1, &c);
  if (st) return st;
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = loop_h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  I2_CK(cudaGraphAddNode(&n_loop, gr, &n_seed, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // The loop body is one kernel. Resident: a cooperative launch that runs
  // every iteration itself (the loop then runs once). Otherwise one launch per
  // iteration: the fixed style's kernel, or the dispatch kernel whose blocks
  // branch on the style the previous iteration selected.
  {
    cudaGraphNode_t n;
    KernelFn fn = resident ? resident_kernel(algo, mode == 0 ? variant : -1, rp.delta != 0, wide_selector(g))
                  : mode == 0 ? relax_kernel(algo, variant, rp.delta != 0)
                              : dispatch_kernel(algo, wide_selector(g));
    st = add_kernel_node(body, &n, nullptr, 0, fn, grid_for(fn, g->blocks_per_sm), &c);
    if (st) return st;
    if (resident) {
      cudaKernelNodeAttrValue av{};
      av.cooperative = 1;
      I2_CK(cudaGraphKernelNodeSetAttribute(n, cudaKernelNodeAttributeCooperative, &av));
    }
  }
  ExecEntry e;
  I2_CK(cudaGraphInstantiate(&e.ex, gr, 0));
  e.reset = n_reset;
  e.last = rp;
  e.ctx = c;
  auto ins = g->execs.emplace(key, e);
  *out = &ins.first->second;
  return I2_OK;
}

// Launch the traversal graph with this run's parameters. Changing the reset
// node's arguments affects only launches made after the change.
static int launch_exec(i2_graph* g, ExecEntry* e, const RunParams& rp, cudaStream_t s) {
  if (e->last != rp) {
    cudaKernelNodeParams kp{};
    Ctl* ctl = g->ctl;
    RunParams p = rp;
    void* args[2] = {&ctl, &p};
    kp.func = (void*)k_reset;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    I2_CK(cudaGraphExecKernelNodeSetParams(e->ex, e->reset, &kp));
    e->last = rp;
  }
  I2_CK(cudaGraphLaunch(e->ex, s));
  return I2_OK;
}

// Reset the bitmaps and the control block on the stream (host-driven paths).
static int prepare_run(i2_graph* g, cudaStream_t s, const RunParams& rp) {
  I2_CK(cudaMemsetAsync(g->bm[0], 0, sizeof(unsigned) * bm_block_words(g), s));
  k_reset<<<1, 32, 0, s>>>(g->ctl, rp);
  I2_CK(cudaGetLastError());
  return I2_OK;
}

// Host-driven loop (one control-block read per iteration, like the reference's
// do-while). Each relax launch is bracketed by CUDA events on the launching
// stream; their sum is returned in *relax_ms.
static int run_host_loop(i2_graph* g, cudaStream_t s, int algo, bool multi, double* relax_ms) {
  Ctx c = make_ctx(g);
  c.srcs = multi ? g->srcs : nullptr;
  KernelFn ff = fill_kernel(algo);
  ff<<<grid_for(ff, 8), kBlock, 0, s>>>(c);
  seed_kernel(algo)<<<1, kBlock, 0, s>>>(c);
  Ctl* h = g->h_ctl;
  double total = 0.0;
  for (;;) {
    I2_CK(cudaMemcpyAsync(h, g->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    I2_CK(cudaStreamSynchronize(s));
    // the last launch's decision: another frontier, a near/far split, the
    // compress launch of union-find, or the end (including the iteration cap)
    if (!h->go || (h->status & kStatusIterCap)) break;
    KernelFn fn = relax_kernel(algo, h->variant, h->delta != 0);
    I2_CK(cudaEventRecord(g->ev2, s));
    fn<<<grid_for(fn, g->blocks_per_sm), kBlock, 0, s>>>(c);
    I2_CK(cudaGetLastError());
    I2_CK(cudaEventRecord(g->ev3, s));
    I2_CK(cudaEventSynchronize(g->ev3));
    float ms = 0.f;
    I2_CK(cudaEventElapsedTime(&ms, g->ev2, g->ev3));
    total += ms;
  }
  *relax_ms = total;
  return I2_OK;
}

static int fill_report(i2_graph* g, cudaStream_t s, int algo, i2_report* rep, double host_relax_ms) {
  I2_CK(cudaMemcpyAsync(g->h_ctl, g->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
  I2_CK(cudaMemsetAsync(g->reach, 0, sizeof(unsigned long long) * 2, s));
  k_reached<<<4 * sm_count(), 256, 0, s>>>(g->g, g->dist, g->reach);
  unsigned long long r[2] = {0, 0};
  I2_CK(cudaMemcpyAsync(r, g->reach, sizeof(r), cudaMemcpyDeviceToHost, s));
  I2_CK(cudaStreamSynchronize(s));
  const Ctl* h = g->h_ctl;
  g->last_iters = h->iter;
  if (rep) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    rep->seconds = ms * 1e-3;
    rep->relax_seconds = host_relax_ms >= 0.0 ? host_relax_ms * 1e-3 : h->relax_ns * 1e-9;
    rep->iterations = h->iter;
    for (int k = 0; k < 16; ++k) rep->variant_hist[k] = h->hist[k];
    rep->reached_vertices = (long long)r[0];
    rep->reached_edges = (long long)r[1];
  }
  if (h->status & kStatusStall) return I2_ERR_STALL;
  if (h->status & kStatusIterCap) return I2_ERR_ITER_CAP;
  (void)algo;
  return I2_OK;
}

// BFS, SSSP or (symmetric graphs) CC of a graph that has a degree-ordered
// copy: the traversal runs on the copy (same options, on the caller's stream
// or the graph's), from the mapped sources, and a gather puts its values into
// this graph's result buffer in original IDs. Levels and distances do not
// depend on the numbering, so the result is the one the original CSR gives;
// CC labels are mapped to each component's smallest original ID. The
// report's seconds are the copy's (init and iterations) plus the mapping's.
static int run_on_twin(i2_graph* g, int algo, int src, const int* srcs_host, int nsrc, const i2_opts* opts,
                       i2_report* rep) {
  std::vector<int> mapped;
  if (srcs_host) {
    if (nsrc < 1) return I2_ERR_ARG;
    mapped.resize(nsrc);
    for (int j = 0; j < nsrc; ++j) {
      if (srcs_host[j] < 0 || srcs_host[j] >= g->g.nodes) return I2_ERR_ARG;
      mapped[j] = g->h_inv[srcs_host[j]];
    }
  } else if (src < 0 || src >= g->g.nodes) {
    return I2_ERR_ARG;
  }
  int st = ensure_workspace(g);
  if (st) return st;
  i2_opts o{};
  if (opts) o = *opts;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;
  o.stream = (void*)s;
  st = run_traversal(g->twin, algo, srcs_host ? 0 : g->h_inv[src], srcs_host ? mapped.data() : nullptr, nsrc, &o,
                     rep);
  if (st && st != I2_ERR_ITER_CAP) return st;
  g->last_on_twin = true;
  g->last_iters = g->twin->last_iters;
  const int n = g->g.nodes;
  if (rep) I2_CK(cudaEventRecord(g->ev2, s));
  const int grid = (int)std::min<long long>(4LL * sm_count(), (n + 255) / 256);
  if (algo == I2_CC) {
    int* mn = g->wl[0];  // free while the original CSR is not traversed
    k_cc_min_init<<<grid, 256, 0, s>>>(mn, n);
    k_cc_min_original<<<grid, 256, 0, s>>>(g->twin->dist, g->d_inv, n, mn);
    k_cc_labels<<<grid, 256, 0, s>>>(g->twin->dist, g->d_inv, mn, n, g->dist);
  } else {
    k_unpermute<<<grid, 256, 0, s>>>(g->twin->dist, g->d_inv, n, g->dist);
  }
  I2_CK(cudaGetLastError());
  if (rep) {  // the copy's traversal time (its report) plus the mapping
    I2_CK(cudaEventRecord(g->ev3, s));
    I2_CK(cudaEventSynchronize(g->ev3));
    float ms = 0.f;
    I2_CK(cudaEventElapsedTime(&ms, g->ev2, g->ev3));
    rep->seconds += ms * 1e-3;
  }
  return st;
}

int run_traversal(i2_graph* g, int algo, int src, const int* srcs_host, int nsrc, const i2_opts* opts,
                  i2_report* rep) {
  if (!g) return I2_ERR_ARG;
  if (algo < I2_BFS || algo > I2_MIS) return I2_ERR_ARG;
  I2_CK(cudaSetDevice(g->device));
  if (g->twin && (algo == I2_BFS || algo == I2_SSSP)) return run_on_twin(g, algo, src, srcs_host, nsrc, opts, rep);
  if (g->twin && algo == I2_CC) {
    // A component's smallest original ID follows from the copy's labels only
    // where components are the same vertex sets in both (symmetric edges);
    // the copy's adjacency is sorted, so its check decides set symmetry.
    int st = ensure_symmetry(g->twin);
    if (st) return st;
    if (g->twin->gs.symmetric == 1) return run_on_twin(g, algo, 0, nullptr, 0, opts, rep);
  }
  g->last_on_twin = false;
  i2_opts o{};
  if (opts) o = *opts;
  if (o.loop_mode < I2_LOOP_GRAPH || o.loop_mode > I2_LOOP_RELAUNCH) return I2_ERR_ARG;
  const bool sourced = algo == I2_BFS || algo == I2_SSSP;
  if (sourced && !srcs_host && (src < 0 || src >= g->g.nodes)) return I2_ERR_ARG;
  if (algo == I2_SSSP) {
    if (!g->g.eweight) return I2_ERR_ARG;
    if (g->gs.wmin < 0) return I2_ERR_UNSUPPORTED;
  }
  int st = ensure_workspace(g);
  if (st) return st;
  if (algo == I2_MIS) {  // one style; the set is defined on undirected graphs
    st = ensure_symmetry(g);
    if (st) return st;
    if (g->gs.symmetric != 1) return I2_ERR_UNSUPPORTED;
    o.variant = kVPWarp;
    o.then_at = 0;
    o.sssp_delta = 0;
    o.sssp_budget = 0;
  }
  int mode = 0, variant = o.variant;
  if (variant == I2_AUTO_HEURISTIC) mode = 1;
  else if (variant == I2_AUTO_LEARNED) mode = 2;
  else if (variant < 0 || variant >= kNumVariants) return I2_ERR_ARG;
  if (o.then_at < 0) return I2_ERR_ARG;
  if (o.then_at > 0) {  // a fixed switch of style: per-iteration dispatch
    if (mode != 0 || o.then_variant < 0 || o.then_variant >= kNumVariants) return I2_ERR_ARG;
    mode = 3;
  }
  // SSSP on a graph of skewed degrees (coefficient of variation above 1) with
  // 2^26 CSR entries or more, from one source: both selectors run the
  // edge-balanced push in the budgeted near/far ordering for the whole
  // traversal (the per-iteration styles cannot take part in its moves and
  // trims). Measured against plain frontier-driven relaxation: 1.13x faster on
  // RMAT-22 and 1.31x on RMAT-26; 5-28% slower on ER, grid and RMAT graphs of
  // up to 2^21 vertices and 2^25 entries, which keep the per-iteration rule.
  // CC on a symmetric graph of 2^22 vertices or more where union-find pays:
  // both selectors take it before the first iteration, so it runs as
  // union-find's own kernel (grid 4096²: 1.37-1.47 ms against 1.79-1.89 in the
  // selectors' kernel at 4 blocks per SM). On smaller graphs the selectors'
  // kernel, with its 64 registers, measured faster (ER 2^20: 0.25 against
  // 0.33 ms; grid 2^18: 0.14 against 0.22-0.28).
  if (algo == I2_CC && (mode == 1 || mode == 2) && (long long)g->g.nodes >= kUnionFindKernelNodes) {
    st = ensure_symmetry(g);
    if (st) return st;
    if (((allowed_mask(g, algo) >> kUnionFind) & 1) && union_find_pays(g->g.nodes, g->gs.avgdeg)) {
      mode = 0;
      variant = kUnionFind;
    }
  }
  if (algo == I2_SSSP && (mode == 1 || mode == 2) && !srcs_host && o.sssp_delta <= 0 &&
      (long long)g->g.edges >= kBudgetRuleEdges && g->gs.degcv > 1.f) {
    mode = 0;
    variant = kVPCta;
    if (o.sssp_budget <= 0) o.sssp_budget = I2_SSSP_BUDGET_AUTO;
  }
  if (mode != 0 || variant == kEdgeTopo) {
    st = ensure_sp(g);
    if (st) return st;
  }
  if (mode != 0 || variant == kPullFrontier || variant == kPullTopo || variant == kUnionFind) {
    st = ensure_symmetry(g);
    if (st) return st;
  }
  if ((mode == 0 || mode == 3) && !((allowed_mask(g, algo) >> variant) & 1)) return I2_ERR_UNSUPPORTED;
  if (mode == 3 && !((allowed_mask(g, algo) >> o.then_variant) & 1)) return I2_ERR_UNSUPPORTED;
  cudaStream_t s = o.stream ? (cudaStream_t)o.stream : g->stream;
  const bool multi = srcs_host != nullptr;
  if (multi) {
    if (nsrc < 1) return I2_ERR_ARG;
    for (int j = 0; j < nsrc; ++j)
      if (srcs_host[j] < 0 || srcs_host[j] >= g->g.nodes) return I2_ERR_ARG;
    if (g->srcs_cap < nsrc) {
      dev_free(g->srcs);
      g->srcs = nullptr;
      I2_CK(dev_alloc(&g->srcs, sizeof(int) * nsrc));
      g->srcs_cap = nsrc;
      // graphs bake the source pointer: rebuild them
      drop_execs(g);
    }
    I2_CK(cudaMemcpyAsync(g->srcs, srcs_host, sizeof(int) * nsrc, cudaMemcpyHostToDevice, s));
  }
  const int delta = pick_order(g, algo, mode, variant, o.sssp_delta, o.sssp_budget);
  if (delta != 0) {
    st = ensure_piles(g);
    if (st) return st;
  }
  RunParams rp = make_params(g, algo, mode, variant, src, nsrc, o.iter_cap, delta);
  if (mode == 3) {
    rp.then_at = o.then_at;
    rp.then_variant = o.then_variant;
  }
  ExecEntry* ex = nullptr;
  const bool graph_loop = o.loop_mode == I2_LOOP_GRAPH || o.loop_mode == I2_LOOP_RELAUNCH;
  if (graph_loop) {
    // Resident traversal where the device takes the cooperative node; graphs
    // with one launch per iteration otherwise.
    const bool resident = o.loop_mode == I2_LOOP_GRAPH && g->resident_ok;
    st = build_exec(g, algo, mode, variant, multi, resident, rp, &ex);
    if (st && resident) {
      cudaGetLastError();
      g->resident_ok = false;
      st = build_exec(g, algo, mode, variant, multi, false, rp, &ex);
    }
    if (st) return st;
  }
  double host_relax_ms = -1.0;
  if (rep) I2_CK(cudaEventRecord(g->ev0, s));
  if (graph_loop) {
    st = launch_exec(g, ex, rp, s);
    if (st) return st;
  } else {
    st = prepare_run(g, s, rp);
    if (st) return st;
    st = run_host_loop(g, s, algo, multi, &host_relax_ms);
    if (st) return st;
  }
  if (rep) I2_CK(cudaEventRecord(g->ev1, s));
  I2_CK(cudaGetLastError());
  // Without a report the call stays asynchronous on the stream.
  if (!rep && graph_loop) return I2_OK;
  return fill_report(g, s, algo, rep, host_relax_ms);
}

int graph_adopt(int nodes, int edges, int* d_nindex, int* d_nlist, int* d_eweight, i2_graph** out) {
  i2_graph* g = new i2_graph();
  g->owns = true;
  g->d_nindex = d_nindex;
  g->d_nlist = d_nlist;
  g->d_eweight = d_eweight;
  g->g.nodes = nodes;
  g->g.edges = edges;
  g->g.nindex = d_nindex;
  g->g.nlist = d_nlist;
  g->g.eweight = d_eweight;
  int st = finish_setup(g);
  if (st) {
    free_graph_state(g);
    delete g;
    return st;
  }
  *out = g;
  return I2_OK;
}

int graph_copy_result(i2_graph* g, int* host_out, const i2_opts* opts) {
  cudaStream_t s = (opts && opts->stream) ? (cudaStream_t)opts->stream : g->stream;
  I2_CK(cudaMemcpyAsync(host_out, g->dist, sizeof(int) * (size_t)g->g.nodes, cudaMemcpyDeviceToHost, s));
  I2_CK(cudaStreamSynchronize(s));
  return I2_OK;
}

// Per-iteration sweep: along the trajectory of `follow` (a variant, or the
// heuristic when negative), save the state before each launch, time every
// allowed variant from that state (best of `reps`), restore, and advance.
static int sweep(i2_graph* g, int algo, int src, int follow, int reps, i2_iter_record* recs, float* times, int cap,
                 int* nout) {
  I2_CK(cudaSetDevice(g->device));
  int st = ensure_workspace(g);
  if (st) return st;
  st = ensure_symmetry(g);
  if (st) return st;
  const long long V = g->g.nodes;
  if (!g->snap_dist) {
    I2_CK(dev_alloc(&g->snap_dist, sizeof(int) * V));
    I2_CK(dev_alloc(&g->snap_bm, sizeof(unsigned) * 3ull * g->bm_words));
  }
  cudaStream_t s = g->stream;
  const int mode = follow == I2_AUTO_LEARNED ? 2 : (follow < 0 ? 1 : 0);
  st = prepare_run(g, s, make_params(g, algo, mode, follow < 0 ? 0 : follow, src, 1, 0));
  if (st) return st;
  Ctx c = make_ctx(g);
  KernelFn ff = fill_kernel(algo);
  ff<<<grid_for(ff, 8), kBlock, 0, s>>>(c);
  seed_kernel(algo)<<<1, kBlock, 0, s>>>(c);
  const int allowed = allowed_mask(g, algo);
  Ctl snap;
  int it = 0;
  // Styles are timed through the dispatch kernel, the one the selectors run.
  KernelFn dk = dispatch_kernel(algo, wide_selector(g));
  const int dgrid = grid_for(dk, g->blocks_per_sm);
  while (it < cap) {
    I2_CK(cudaMemcpyAsync(g->h_ctl, g->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    I2_CK(cudaStreamSynchronize(s));
    snap = *g->h_ctl;
    if (!snap.go || (snap.status & kStatusIterCap)) break;
    if (snap.uf_phase) {  // the trajectory took union-find: its compress launch is not a choice
      dk<<<dgrid, kBlock, 0, s>>>(c);
      I2_CK(cudaGetLastError());
      continue;
    }
    I2_CK(cudaMemcpyAsync(g->snap_dist, g->dist, sizeof(int) * V, cudaMemcpyDeviceToDevice, s));
    I2_CK(cudaMemcpyAsync(g->snap_bm, g->bm[0], sizeof(unsigned) * 3ull * g->bm_words, cudaMemcpyDeviceToDevice, s));
    for (int v = 0; v < kNumVariants; ++v) {
      float best = -1.f;
      if ((allowed >> v) & 1) {
        for (int r = 0; r < std::max(1, reps); ++r) {
          *g->h_ctl = snap;
          g->h_ctl->variant = v;
          I2_CK(cudaMemcpyAsync(g->ctl, g->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, s));
          I2_CK(cudaMemcpyAsync(g->dist, g->snap_dist, sizeof(int) * V, cudaMemcpyDeviceToDevice, s));
          I2_CK(cudaMemcpyAsync(g->bm[0], g->snap_bm, sizeof(unsigned) * 3ull * g->bm_words, cudaMemcpyDeviceToDevice, s));
          I2_CK(cudaEventRecord(g->ev0, s));
          dk<<<dgrid, kBlock, 0, s>>>(c);
          if (v == kUnionFind) {  // its later launches belong to it
            dk<<<dgrid, kBlock, 0, s>>>(c);
            dk<<<dgrid, kBlock, 0, s>>>(c);
          }
          I2_CK(cudaEventRecord(g->ev1, s));
          I2_CK(cudaEventSynchronize(g->ev1));
          float ms = 0.f;
          I2_CK(cudaEventElapsedTime(&ms, g->ev0, g->ev1));
          // The launches' own device time (their iteration records), without the
          // launch latency that the resident traversal does not pay.
          const int nrec = v == kUnionFind ? 3 : 1;
          if (snap.iter + nrec <= g->rec_cap) {
            IterRec r[3];
            I2_CK(cudaMemcpy(r, g->recs + snap.iter, sizeof(IterRec) * nrec, cudaMemcpyDeviceToHost));
            ms = 0.f;
            for (int j = 0; j < nrec; ++j) ms += (float)r[j].t_ns * 1e-6f;
          }
          if (best < 0.f || ms < best) best = ms;
        }
        best *= 1e6f;  // ns
      }
      times[(size_t)it * kNumVariants + v] = best;
    }
    *g->h_ctl = snap;
    I2_CK(cudaMemcpyAsync(g->ctl, g->h_ctl, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    I2_CK(cudaMemcpyAsync(g->dist, g->snap_dist, sizeof(int) * V, cudaMemcpyDeviceToDevice, s));
    I2_CK(cudaMemcpyAsync(g->bm[0], g->snap_bm, sizeof(unsigned) * 3ull * g->bm_words, cudaMemcpyDeviceToDevice, s));
    dk<<<dgrid, kBlock, 0, s>>>(c);
    I2_CK(cudaGetLastError());
    if (snap.iter < g->rec_cap)
      I2_CK(cudaMemcpyAsync(&recs[it], g->recs + snap.iter, sizeof(IterRec), cudaMemcpyDeviceToHost, s));
    ++it;
  }
  I2_CK(cudaStreamSynchronize(s));
  *nout = it;
  g->last_iters = it;
  return I2_OK;
}

// True when [p, p + bytes) lies inside one device (or managed) allocation of
// the current context. Host pointers, pinned or not, are refused: a kernel
// given one would fault or read the wrong memory. So is device memory of
// another GPU: kernels launched on the current device would read it through a
// peer mapping, or fault where there is none.
typedef int (*MemGetAddressRangeFn)(unsigned long long*, size_t*, unsigned long long);

int graph_device_csr(const i2_graph* g, int* nodes, int* edges, const int** nindex, const int** nlist,
                     const int** eweight) {
  if (!g) return I2_ERR_ARG;
  *nodes = g->g.nodes;
  *edges = g->g.edges;
  *nindex = g->g.nindex;
  *nlist = g->g.nlist;
  *eweight = g->g.eweight;
  return I2_OK;
}

bool device_range_ok(const void* p, size_t bytes) {
  if (bytes == 0) return true;
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return false;
  if (a.type == cudaMemoryTypeDevice) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || a.device != cur) {
      cudaGetLastError();
      return false;
    }
  }
  static MemGetAddressRangeFn range_fn = nullptr;
  static bool looked = false;
  if (!looked) {
    looked = true;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      range_fn = (MemGetAddressRangeFn)fn;
    cudaGetLastError();
  }
  if (!range_fn) return true;  // type check only
  unsigned long long base = 0;
  size_t size = 0;
  if (range_fn(&base, &size, (unsigned long long)(uintptr_t)p) != 0) return false;
  return (unsigned long long)(uintptr_t)p + bytes <= base + size;
}

}  // namespace i2

// ---------------------------------------------------------------------------
// C ABI.

extern "C" {

const char* i2_status_string(int status) {
  switch (status) {
    case I2_OK: return "ok";
    case I2_ERR_ARG: return "invalid argument";
    case I2_ERR_IO: return "file i/o error";
    case I2_ERR_FORMAT: return "malformed graph";
    case I2_ERR_NOMEM: return "out of memory";
    case I2_ERR_CUDA: return "cuda error";
    case I2_ERR_NO_DEVICE: return "no cuda device";
    case I2_ERR_UNSUPPORTED: return "variant not supported on this graph";
    case I2_ERR_ITER_CAP: return "iteration cap reached";
    case I2_ERR_OVERFLOW: return "int32 limit exceeded";
    case I2_ERR_CAPACITY: return "graph exceeds the fixed scratch of i2_run_noalloc";
    case I2_ERR_STALL: return "a resident traversal's barrier wait ran out of time";
  }
  return "unknown status";
}

const char* i2_variant_name(int v) {
  static const char* names[] = {"vp_thread", "vp_warp", "vp_cta", "vp_block",
                                "pull_frontier", "pull_topo", "edge_topo", "push_topo", "union_find"};
  if (v == I2_AUTO_HEURISTIC) return "auto_heuristic";
  if (v == I2_AUTO_LEARNED) return "auto_learned";
  if (v < 0 || v >= kNumVariants) return "invalid";
  return names[v];
}

int i2_version(void) { return 100; }

int i2_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

static int upload_common(i2_graph* g) {
  int st = finish_setup(g);
  if (st) {
    free_graph_state(g);
    delete g;
  }
  return st;
}

// The shape of the CSR is checked on the host; its entries (monotone nindex,
// nlist in range) on the device right after the copy, before any other kernel
// reads them: a host pass over nlist costs about as much as copying it. The
// adjacency and the weights go over two streams (two copy engines).
int i2_graph_upload(const i2_eclgraph* h, i2_graph** out) {
  if (!h || !out) return I2_ERR_ARG;
  *out = nullptr;
  if (h->nodes < 1 || h->edges < 0) return I2_ERR_FORMAT;
  if (!h->nindex || (h->edges > 0 && !h->nlist)) return I2_ERR_ARG;
  if (h->nindex[0] != 0 || h->nindex[h->nodes] != h->edges) return I2_ERR_FORMAT;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  i2_graph* g = new i2_graph();
  g->owns = true;
  const size_t nn = (size_t)h->nodes + 1, ne = (size_t)h->edges + 4;
  cudaStream_t s1 = nullptr, s2 = nullptr;
  int* bad = nullptr;
  int hbad = 0;
  cudaError_t e = dev_alloc(&g->d_nindex, sizeof(int) * nn);
  if (e == cudaSuccess) e = dev_alloc(&g->d_nlist, sizeof(int) * ne);
  if (e == cudaSuccess && h->eweight) e = dev_alloc(&g->d_eweight, sizeof(int) * ne);
  if (e == cudaSuccess) e = dev_alloc(&bad, sizeof(int));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s1, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), s1);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->d_nindex, h->nindex, sizeof(int) * nn, cudaMemcpyHostToDevice, s1);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(g->d_nlist, h->nlist, sizeof(int) * h->edges, cudaMemcpyHostToDevice, s1);
  if (e == cudaSuccess && h->eweight)
    e = cudaMemcpyAsync(g->d_eweight, h->eweight, sizeof(int) * h->edges, cudaMemcpyHostToDevice, s2);
  g->g.nodes = h->nodes;
  g->g.edges = h->edges;
  g->g.nindex = g->d_nindex;
  g->g.nlist = g->d_nlist;
  g->g.eweight = g->d_eweight;
  if (e == cudaSuccess) {
    k_validate<<<4 * sm_count(), 256, 0, s1>>>(g->g, bad);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s1);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s1);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s2);
  if (s1) cudaStreamDestroy(s1);
  if (s2) cudaStreamDestroy(s2);
  dev_free(bad);
  if (e != cudaSuccess || hbad) {
    cudaGetLastError();
    free_graph_state(g);
    delete g;
    return e != cudaSuccess ? cuda_status(e) : I2_ERR_FORMAT;
  }
  int st = upload_common(g);
  if (st) return st;
  *out = g;
  return I2_OK;
}

int i2_graph_hub(i2_graph* g, int* v) {
  if (!g || !v) return I2_ERR_ARG;
  I2_CK(cudaSetDevice(g->device));
  int* d = nullptr;
  I2_CK(dev_alloc(&d, sizeof(int)));
  int h = INT_MAX;
  cudaError_t e = cudaMemcpyAsync(d, &h, sizeof(int), cudaMemcpyHostToDevice, g->stream);
  if (e == cudaSuccess) {
    k_hub<<<4 * sm_count(), 256, 0, g->stream>>>(g->g, g->gs.maxdeg, d);
    e = cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, g->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
  dev_free(d);
  if (e != cudaSuccess) return cuda_status(e);
  *v = h == INT_MAX ? 0 : h;
  return I2_OK;
}

int i2_graph_sp(i2_graph* g, const int** sp_dev, int* sp_host) {
  if (!g || (!sp_dev && !sp_host)) return I2_ERR_ARG;
  I2_CK(cudaSetDevice(g->device));
  int st = ensure_sp(g);
  if (st) return st;
  if (sp_dev) *sp_dev = g->d_sp;
  if (sp_host && g->g.edges > 0)
    I2_CK(cudaMemcpy(sp_host, g->d_sp, sizeof(int) * (size_t)g->g.edges, cudaMemcpyDeviceToHost));
  return I2_OK;
}

int i2_graph_wrap_device(const i2_eclgraph* d, i2_graph** out) {
  if (!d || !out || d->nodes < 1 || d->edges < 0 || !d->nindex || (d->edges > 0 && !d->nlist)) return I2_ERR_ARG;
  *out = nullptr;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  if (!device_range_ok(d->nindex, sizeof(int) * ((size_t)d->nodes + 1)) ||
      !device_range_ok(d->nlist, sizeof(int) * (size_t)d->edges) ||
      (d->eweight && !device_range_ok(d->eweight, sizeof(int) * (size_t)d->edges)))
    return I2_ERR_ARG;
  i2_graph* g = new i2_graph();
  g->owns = false;
  g->d_nindex = d->nindex;
  g->d_nlist = d->nlist;
  g->d_eweight = d->eweight;
  g->g.nodes = d->nodes;
  g->g.edges = d->edges;
  g->g.nindex = d->nindex;
  g->g.nlist = d->nlist;
  g->g.eweight = d->eweight;
  // Validate before any kernel indexes through the arrays.
  int* bad = nullptr;
  int hbad = 0;
  cudaError_t e = dev_alloc(&bad, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(bad, 0, sizeof(int));
  if (e == cudaSuccess) {
    k_validate<<<4 * sm_count(), 256>>>(g->g, bad);
    e = cudaMemcpy(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost);
  }
  dev_free(bad);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete g;
    return cuda_status(e);
  }
  if (hbad) {
    delete g;
    return I2_ERR_FORMAT;
  }
  int st = upload_common(g);
  if (st) return st;
  *out = g;
  return I2_OK;
}

int i2_graph_size(const i2_graph* g, int* nodes, int* edges) {
  if (!g || !nodes || !edges) return I2_ERR_ARG;
  *nodes = g->g.nodes;
  *edges = g->g.edges;
  return I2_OK;
}

int i2_graph_degree(const i2_graph* g, int v, int* deg) {
  if (!g || !deg || v < 0 || v >= g->g.nodes) return I2_ERR_ARG;
  int pair[2];
  I2_CK(cudaMemcpy(pair, g->g.nindex + v, sizeof(pair), cudaMemcpyDeviceToHost));
  *deg = pair[1] - pair[0];
  return I2_OK;
}

int i2_graph_info_get(const i2_graph* g, i2_graph_info* out) {
  if (!g || !out) return I2_ERR_ARG;
  if (g->gs.symmetric < 0) {
    cudaSetDevice(g->device);
    const int st = ensure_symmetry(const_cast<i2_graph*>(g));
    if (st) return st;
  }
  out->nodes = g->gs.nodes;
  out->edges = g->gs.edges;
  out->maxdeg = g->gs.maxdeg;
  out->nheavy = g->gs.nheavy;
  out->wmin = g->gs.wmin;
  out->symmetric = g->gs.symmetric;
  out->has_weights = g->g.eweight != nullptr;
  out->avgdeg = g->gs.avgdeg;
  out->degcv = g->gs.degcv;
  return I2_OK;
}

int i2_graph_download(const i2_graph* g, i2_eclgraph* out) {
  if (!g || !out) return I2_ERR_ARG;
  int st = i2_alloc_eclgraph(g->g.nodes, g->g.edges, g->g.eweight ? 1 : 0, out);
  if (st) return st;
  cudaError_t e = cudaMemcpy(out->nindex, g->g.nindex, sizeof(int) * ((size_t)g->g.nodes + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(out->nlist, g->g.nlist, sizeof(int) * (size_t)g->g.edges, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && g->g.eweight)
    e = cudaMemcpy(out->eweight, g->g.eweight, sizeof(int) * (size_t)g->g.edges, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaGetLastError();
    i2_free_eclgraph(out);
    return cuda_status(e);
  }
  return I2_OK;
}

int i2_graph_tune(i2_graph* g, int heavy_threshold, int blocks_per_sm, int smem_carveout) {
  if (!g || heavy_threshold < 0 || blocks_per_sm < 0 || blocks_per_sm > 32) return I2_ERR_ARG;
  if (smem_carveout < -1 || smem_carveout > 100) return I2_ERR_ARG;
  g_carveout = smem_carveout;
  I2_CK(cudaSetDevice(g->device));
  if (g->stream) I2_CK(cudaStreamSynchronize(g->stream));
  drop_execs(g);
  if (blocks_per_sm) g->blocks_per_sm = blocks_per_sm;
  if (heavy_threshold && heavy_threshold != g->heavy) {
    g->heavy = std::max(32, heavy_threshold);
    // the heavy lists are sized by the number of heavy vertices
    for (int k = 0; k < 3; ++k) {
      dev_free(g->hwl[k]);
      dev_free(g->htoff[k]);
      g->hwl[k] = nullptr;
      g->htoff[k] = nullptr;
    }
    int st = compute_stats(g);
    if (st) return st;
    if (g->ws_ready)
      for (int k = 0; k < 3; ++k) {
        I2_CK(dev_alloc(&g->hwl[k], sizeof(int) * std::max(1, g->gs.nheavy)));
        I2_CK(dev_alloc(&g->htoff[k], sizeof(unsigned) * std::max(1, g->gs.nheavy)));
      }
  }
  if (g->twin) return i2_graph_tune(g->twin, heavy_threshold, blocks_per_sm, smem_carveout);
  return I2_OK;
}

int i2_graph_synth_weights(i2_graph* g) {
  if (!g) return I2_ERR_ARG;
  if (g->g.eweight) return I2_OK;
  I2_CK(cudaSetDevice(g->device));
  int* w = nullptr;
  I2_CK(dev_alloc(&w, sizeof(int) * ((size_t)g->g.edges + 4)));
  k_synth_weights<<<8 * sm_count(), 256, 0, g->stream>>>(g->g, w);
  I2_CK(cudaStreamSynchronize(g->stream));
  g->d_eweight = w;
  g->owns_weights = true;
  g->g.eweight = w;
  g->g.vec_ok = ((((uintptr_t)g->g.nlist) & 15) == 0 && (((uintptr_t)w) & 15) == 0) ? 1 : 0;
  drop_execs(g);
  const int st = compute_stats(g);
  if (st || !g->twin) return st;
  // the weights are a function of the original IDs: renumber again
  return i2_graph_reorder(g, I2_ORDER_DEGREE);
}

int i2_graph_free(i2_graph* g) {
  if (!g) return I2_ERR_ARG;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  free_graph_state(g);
  delete g;
  return I2_OK;
}

int i2_graph_reorder(i2_graph* g, int order) {
  if (!g || (order != I2_ORDER_NONE && order != I2_ORDER_DEGREE)) return I2_ERR_ARG;
  I2_CK(cudaSetDevice(g->device));
  if (g->stream) I2_CK(cudaStreamSynchronize(g->stream));
  if (g->twin) {
    i2_graph_free(g->twin);
    g->twin = nullptr;
    dev_free(g->d_inv);
    g->d_inv = nullptr;
    g->h_inv.clear();
    g->h_inv.shrink_to_fit();
    g->last_on_twin = false;
  }
  // nothing to renumber without edges: traversals stay on the original
  if (order == I2_ORDER_NONE || g->g.edges == 0) return I2_OK;
  i2_graph* twin = nullptr;
  int* inv = nullptr;
  int st = degree_ordered_copy(g, &twin, &inv);
  if (st) return st;
  std::vector<int> h(g->g.nodes);
  const cudaError_t e = cudaMemcpy(h.data(), inv, sizeof(int) * h.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    i2_graph_free(twin);
    dev_free(inv);
    return cuda_status(e);
  }
  // the copy launches like the original (settings of i2_graph_tune; the
  // heavy lists are sized for the threshold by the tune call)
  st = i2_graph_tune(twin, g->heavy, g->blocks_per_sm, g_carveout);
  if (st) {
    i2_graph_free(twin);
    dev_free(inv);
    return st;
  }
  g->twin = twin;
  g->d_inv = inv;
  g->h_inv.swap(h);
  return I2_OK;
}

int i2_trim_device_memory(void) {
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  return trim_pool();
}

static int run_host_out(i2_graph* g, int algo, int src, int* out, const i2_opts* opts, i2_report* rep) {
  if (!out) return I2_ERR_ARG;
  int st = run_traversal(g, algo, src, nullptr, 0, opts, rep);
  if (st && st != I2_ERR_ITER_CAP) return st;
  cudaStream_t s = (opts && opts->stream) ? (cudaStream_t)opts->stream : g->stream;
  I2_CK(cudaMemcpyAsync(out, g->dist, sizeof(int) * (size_t)g->g.nodes, cudaMemcpyDeviceToHost, s));
  I2_CK(cudaStreamSynchronize(s));
  return st;
}

int i2_bfs(i2_graph* g, int src, int* dist, const i2_opts* opts, i2_report* rep) {
  return run_host_out(g, I2_BFS, src, dist, opts, rep);
}
int i2_sssp(i2_graph* g, int src, int* dist, const i2_opts* opts, i2_report* rep) {
  return run_host_out(g, I2_SSSP, src, dist, opts, rep);
}
int i2_cc(i2_graph* g, int* label, const i2_opts* opts, i2_report* rep) {
  return run_host_out(g, I2_CC, 0, label, opts, rep);
}

int i2_mis(i2_graph* g, int* status, const i2_opts* opts, i2_report* rep) {
  return run_host_out(g, I2_MIS, 0, status, opts, rep);
}

int i2_run_device(i2_graph* g, int algo, int src, int* out_dev, const i2_opts* opts, i2_report* rep) {
  int st = run_traversal(g, algo, (algo == I2_CC || algo == I2_MIS) ? 0 : src, nullptr, 0, opts, rep);
  if (st && st != I2_ERR_ITER_CAP) return st;
  if (out_dev) {
    cudaStream_t s = (opts && opts->stream) ? (cudaStream_t)opts->stream : g->stream;
    I2_CK(cudaMemcpyAsync(out_dev, g->dist, sizeof(int) * (size_t)g->g.nodes, cudaMemcpyDeviceToDevice, s));
  }
  return st;
}

int i2_get_records(const i2_graph* g, i2_iter_record* out, int cap, int* n) {
  if (!g || !out || !n || cap < 0) return I2_ERR_ARG;
  if (g->last_on_twin && g->twin) return i2_get_records(g->twin, out, cap, n);
  if (!g->ws_ready) {
    *n = 0;
    return I2_OK;
  }
  const int m = std::min(std::min(g->last_iters, g->rec_cap), cap);
  if (m > 0) I2_CK(cudaMemcpy(out, g->recs, sizeof(IterRec) * m, cudaMemcpyDeviceToHost));
  *n = m;
  return I2_OK;
}

int i2_sweep(i2_graph* g, int algo, int src, int follow, int reps, i2_iter_record* recs, float* times, int cap,
             int* n) {
  if (!g || !recs || !times || !n || cap < 1 || algo < I2_BFS || algo > I2_CC) return I2_ERR_ARG;
  if (follow >= kNumVariants || follow < I2_AUTO_LEARNED) return I2_ERR_ARG;
  if (algo != I2_CC && (src < 0 || src >= g->g.nodes)) return I2_ERR_ARG;
  if (algo == I2_SSSP && !g->g.eweight) return I2_ERR_ARG;
  if (follow >= 0) {
    int st = ensure_symmetry(g);
    if (st) return st;
    if (!((allowed_mask(g, algo) >> follow) & 1)) return I2_ERR_UNSUPPORTED;
  }
  return sweep(g, algo, src, follow, reps, recs, times, cap, n);
}

int i2_mlp_param_count(void) { return kParams; }

int i2_mlp_set_params(const float* params, int count) { return mlp_install(params, count); }

}  // extern "C"

// ---------------------------------------------------------------------------
// Traversal that allocates nothing.
//
// Some callers cannot allocate device memory at the moment they run a query:
// their process's device memory is already held by another allocator (for
// example a framework's caching allocator that reserved the GPU), their query
// loop cannot afford cudaMalloc/cudaFree, which synchronise the device, or
// their query must not be able to fail with out-of-memory. i2_run_noalloc
// serves them: the caller passes the CSR arrays and the output array (all in
// device memory), and every piece of scratch the traversal needs (frontier
// lists, their edge offsets, the frontier bitmaps and the control block) lives
// in one fixed-size device array defined in this file. That array is part of
// the library image: every GPU that loads the library holds it (about 3 MB)
// until the process exits. Graphs above kNoAllocMaxNodes vertices are refused.

namespace i2 {

constexpr int kNoAllocMaxNodes = 1 << 17;  // 131072 vertices
constexpr int kNoAllocWords = kNoAllocMaxNodes / 32;

// Layout of the scratch array (offsets in bytes, each 256-byte aligned).
constexpr size_t kNoAllocAlign(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNaWl = 0;
constexpr size_t kNaWoff = kNaWl + kNoAllocAlign(3ull * kNoAllocMaxNodes * sizeof(int));
constexpr size_t kNaBm = kNaWoff + kNoAllocAlign(3ull * kNoAllocMaxNodes * sizeof(unsigned));
constexpr size_t kNaHeavy = kNaBm + kNoAllocAlign(3ull * kNoAllocWords * sizeof(unsigned));
constexpr size_t kNaCtl = kNaHeavy + 256;
constexpr size_t kNaBad = kNaCtl + kNoAllocAlign(sizeof(Ctl));
constexpr size_t kNoAllocBytes = kNaBad + 256;

}  // namespace i2

// The scratch itself. In host code this name is only a host-side stand-in:
// its device address is obtained with cudaGetSymbolAddress (per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[i2::kNoAllocBytes];

namespace i2 {

static std::mutex g_noalloc_mu;
static unsigned char* g_noalloc_dev[64] = {nullptr};

// Device address of the scratch on the current device; looked up on the first
// call per device.
static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  I2_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return I2_ERR_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_dev[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return cuda_status(e);
    }
    g_noalloc_dev[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_dev[dev];
  return I2_OK;
}

}  // namespace i2

extern "C" int i2_run_noalloc(int algo, const i2_eclgraph* dev, int src, int* dist_dev, void* stream,
                              int* iterations) {
  using namespace i2;
  if (algo < I2_BFS || algo > I2_CC || !dev || !dist_dev) return I2_ERR_ARG;
  if (dev->nodes < 1 || dev->edges < 0 || !dev->nindex || (dev->edges > 0 && !dev->nlist)) return I2_ERR_ARG;
  if (dev->nodes > kNoAllocMaxNodes) return I2_ERR_CAPACITY;
  if (algo != I2_CC && (src < 0 || src >= dev->nodes)) return I2_ERR_ARG;
  if (algo == I2_SSSP && !dev->eweight) return I2_ERR_ARG;
  if (i2_device_count() < 1) return I2_ERR_NO_DEVICE;
  const int* w = algo == I2_SSSP ? dev->eweight : nullptr;
  if (!device_range_ok(dev->nindex, sizeof(int) * ((size_t)dev->nodes + 1)) ||
      !device_range_ok(dev->nlist, sizeof(int) * (size_t)dev->edges) ||
      (w && !device_range_ok(w, sizeof(int) * (size_t)dev->edges)) ||
      !device_range_ok(dist_dev, sizeof(int) * (size_t)dev->nodes))
    return I2_ERR_ARG;
  unsigned char* base = nullptr;
  int st = noalloc_scratch(&base);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  Ctl* ctl = reinterpret_cast<Ctl*>(base + kNaCtl);
  int* bad = reinterpret_cast<int*>(base + kNaBad);

  Ctx c{};
  c.g.nodes = dev->nodes;
  c.g.edges = dev->edges;
  c.g.nindex = dev->nindex;
  c.g.nlist = dev->nlist;
  c.g.eweight = w;
  c.g.sp = nullptr;
  c.g.vec_ok = ((((uintptr_t)dev->nlist) & 15) == 0 && (((uintptr_t)w) & 15) == 0) ? 1 : 0;
  c.gs.nodes = dev->nodes;
  c.gs.edges = dev->edges;
  c.gs.wmin = 1;
  c.gs.avgdeg = (float)dev->edges / (float)dev->nodes;
  c.dist = dist_dev;
  for (int k = 0; k < 3; ++k) {
    c.wl[k] = reinterpret_cast<int*>(base + kNaWl) + (size_t)k * kNoAllocMaxNodes;
    c.woff[k] = reinterpret_cast<unsigned*>(base + kNaWoff) + (size_t)k * kNoAllocMaxNodes;
    c.bm[k] = reinterpret_cast<unsigned*>(base + kNaBm) + (size_t)k * kNoAllocWords;
    // the heavy lists stay empty: the threshold is above every degree
    c.hwl[k] = reinterpret_cast<int*>(base + kNaHeavy);
    c.htoff[k] = reinterpret_cast<unsigned*>(base + kNaHeavy + 128);
  }
  c.ctl = ctl;
  c.recs = nullptr;
  c.rec_cap = 0;
  c.heavy = INT_MAX;
  c.bm_words = (dev->nodes + 31) / 32;
  c.mlp = nullptr;
  c.srcs = nullptr;
  c.use_loop = 0;

  // Reject malformed arrays before any traversal kernel indexes through them.
  int hbad = 0;
  I2_CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
  k_validate<<<4 * sm_count(), 256, 0, s>>>(c.g, bad);
  // negative weights: refused like the allocating entry points refuse them
  if (w) k_negative_weights<<<4 * sm_count(), 256, 0, s>>>(w, dev->edges, bad);
  I2_CK(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  I2_CK(cudaStreamSynchronize(s));
  if (hbad & 7) return I2_ERR_FORMAT;
  if (hbad & 8) return I2_ERR_UNSUPPORTED;

  // The scratch keeps the previous call's contents: the bitmaps must start at
  // zero (k_reset rewrites the control block, k_fill the output).
  RunParams rp{};
  rp.algo = algo;
  rp.mode = 0;
  rp.fixed_variant = kVPCta;
  rp.allowed = 1 << kVPCta;
  rp.src = algo == I2_CC ? 0 : src;
  rp.nsrc = 1;
  rp.iter_cap = dev->nodes + 2;
  I2_CK(cudaMemsetAsync(c.bm[0], 0, sizeof(unsigned) * 3ull * kNoAllocWords, s));
  k_reset<<<1, 32, 0, s>>>(ctl, rp);
  KernelFn ff = fill_kernel(algo);
  ff<<<grid_for(ff, 8), kBlock, 0, s>>>(c);
  seed_kernel(algo)<<<1, kBlock, 0, s>>>(c);
  KernelFn fn = relax_kernel(algo, kVPCta, false);
  const int grid = grid_for(fn, 8);
  Ctl h;
  for (;;) {
    I2_CK(cudaMemcpyAsync(&h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    I2_CK(cudaStreamSynchronize(s));
    if (slot_size(h.slot[h.iter % 3].packed) == 0 || (h.status & kStatusIterCap)) break;
    fn<<<grid, kBlock, 0, s>>>(c);
    I2_CK(cudaGetLastError());
  }
  if (iterations) *iterations = h.iter;
  return (h.status & kStatusIterCap) ? I2_ERR_ITER_CAP : I2_OK;
}
