// Relaxation kernels of the B200 engine: one persistent, grid-stride kernel per
// (algorithm, variant). Each launch performs exactly one iteration of the
// frontier contract described in common.cuh.
//
// Reference styles these variants re-create (file names under codes/cuda/):
//   kVPThread  ~ *_V_Data_Push_*_Thread_*   (e.g. BFS ..._Atomic_Thread_..._NonDup.cu)
//   kVPWarp    ~ *_V_Data_Push_*_Warp_*     (BFS_CUDA_V_Data_Push_..._Warp_..._NonDup.cu:62-84)
//   kVPBlock   ~ *_V_Data_Push_*_Block_*    (BFS_CUDA_V_Data_Push_..._Block_..._Dup.cu:62-83)
//   kVPCta     ~ *_E_Data_Push_*            (SSSP_CUDA_E_Data_Push_..._NonDup.cu:63-82): one thread per
//                                           frontier edge, the edges split evenly over the grid
//   kPullFrontier / kPullTopo ~ *_V_{Data,Topo}_Pull_* (BFS ..._V_Topo_Pull_..._Warp_...cu:57-79,
//                                           CC_CUDA_V_Topo_Pull_..._Warp_...cu:59-78)
//   kEdgeTopo  ~ *_E_Topo_Push_*            (BFS_CUDA_E_Topo_Push_..._Thread_...cu:57-72)
//   kPushTopo  ~ *_V_Topo_Push_*            (BFS_CUDA_V_Topo_Push_..._Thread_...cu:56-79)
// The B200 versions differ in mechanism, not in fixed point:
//  * frontier appends are staged per block in shared memory and published with
//    one packed 64-bit atomic per flush, which also yields each entry's offset
//    in the frontier's edge space (the reference appends with one atomicAdd per
//    vertex, BFS_..._Warp_..._NonDup.cu:78);
//  * duplicates are filtered by a frontier bitmap (the reference uses a time[]
//    stamp array, :77);
//  * each thread issues the dist[] loads of several neighbours before any of
//    their atomicMin operations, so that several misses are in flight per thread;
//  * adjacency is read with 128-bit loads where aligned, and the frontier's
//    heavy vertices are cut into tiles that any block may take.
#pragma once
#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>
#include <cooperative_groups/scan.h>
#include <cub/block/block_scan.cuh>
#include <type_traits>
#include "common.cuh"

namespace i2 {

namespace cg = cooperative_groups;

constexpr int kScanItems = kQueue / kBlock;                 // staged entries per thread in a flush
// Edges per lane of the edge-balanced tile, and the resident blocks per SM its
// kernels are compiled for (which bounds their registers: 6 -> 40 per thread).
// Measured on RMAT-22 and a 2048^2 grid (ms, SSSP / BFS / CC on RMAT):
// 2 edges at 6 blocks 2.65 / 1.12 / 2.21 (default), 4 at 5 blocks 2.80 / 1.14
// / 2.23, 3 at 5 2.78 / 1.14 / 2.30, 1 at 8 3.11 / 1.24 / 2.39; 2 at 7 or 8
// blocks and 4 at 6 spill and run 1.2-2x slower.
#ifndef I2_EB_EDGES
#define I2_EB_EDGES 2
#endif
constexpr int kEdgesPerThread = I2_EB_EDGES;                // edge-balanced variant
constexpr int kTileEdges = kBlock * kEdgesPerThread;        // edges per edge-balanced tile

typedef cub::BlockScan<int, kBlock> BlockScanT;

// Loads of the graph's adjacency (nlist, eweight, sp): each entry is read
// about once per iteration, so it is loaded with an evict-first policy, which
// keeps the randomly accessed, L2-sized arrays (values, bitmaps, frontier
// lists, nindex) resident in L2 instead of the streamed lines. On RMAT-22 this
// measured 3-7% faster for BFS, SSSP and CC than the read-only path.
// I2_STREAM_LOADS: 0 read-only path without a hint, 1 evict-first (default),
// 2 explicit L2 policies: adjacency evict-first, not allocated in L1 (measured
// within 1% of 1 on RMAT-22 BFS, SSSP and CC and on a 2048² grid).
#ifndef I2_STREAM_LOADS
#define I2_STREAM_LOADS 1
#endif
#if I2_STREAM_LOADS == 2
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long pol;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ int ld_adj(const int* p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(l2_evict_first()));
  return v;
}
__device__ __forceinline__ int4 ld_adj(const int4* p) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.b32 {%0, %1, %2, %3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p), "l"(l2_evict_first()));
  return v;
}
#else
template <typename T>
__device__ __forceinline__ T ld_adj(const T* p) {
#if I2_STREAM_LOADS
  return __ldcs(p);
#else
  return __ldg(p);
#endif
}
#endif

// Frontier statistics of one thread's pushes; kept in registers and reduced
// once per block at the end of the launch.
struct Acc {
  int maxdeg;
  int mindist;
  int visited;
  int fmin;  // smallest value put on a far pile
};

__device__ __forceinline__ void acc_init(Acc& a) {
  a.maxdeg = 0;
  a.mindist = kInf;
  a.visited = 0;
  a.fmin = kInf;
}

// Per-block staging of pushes into the next frontier.
struct Stage {
  int q[kQueue];    // vertices
  int qd[kQueue];   // their degrees
  int hq[kHQueue];  // heavy vertices
  int ht[kHQueue];  // their tile counts
  int n;
  int hn;
  unsigned long long base;
  unsigned long long hbase;
  int chunk;
  int last;
  int j0;
  int m;
  Acc red[kBlock / kWarp];
  typename BlockScanT::TempStorage scan;
};

__device__ __forceinline__ void stage_init(Stage& s) {
  if (threadIdx.x == 0) {
    s.n = 0;
    s.hn = 0;
    s.last = 0;
  }
}

__device__ __forceinline__ int heavy_tiles(int deg) { return (deg + kHeavyTile - 1) / kHeavyTile; }

// Block-wide reduction of the per-thread statistics into s.red[0] (thread 0).
// S is any shared struct with `Acc red[kBlock / kWarp]` and `int last`.
template <typename S>
__device__ __forceinline__ void acc_reduce(Acc a, S& s) {
  for (int o = 16; o > 0; o >>= 1) {
    a.maxdeg = max(a.maxdeg, __shfl_down_sync(0xffffffffu, a.maxdeg, o));
    a.mindist = min(a.mindist, __shfl_down_sync(0xffffffffu, a.mindist, o));
    a.visited += __shfl_down_sync(0xffffffffu, a.visited, o);
    a.fmin = min(a.fmin, __shfl_down_sync(0xffffffffu, a.fmin, o));
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) s.red[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      s.red[0].maxdeg = max(s.red[0].maxdeg, s.red[w].maxdeg);
      s.red[0].mindist = min(s.red[0].mindist, s.red[w].mindist);
      s.red[0].visited += s.red[w].visited;
      s.red[0].fmin = min(s.red[0].fmin, s.red[w].fmin);
    }
  }
}

// Append (v, deg) or (v, tiles) to a list without the staging queue: used only
// when a round produces more pushes than the shared queue holds. The threads
// that overflow together share one packed atomic.
__device__ __forceinline__ void direct_append(unsigned long long* packed, int* list, unsigned* off, int v, int w) {
  cg::coalesced_group g = cg::coalesced_threads();
  const int pre = cg::exclusive_scan(g, w);
  const int tot = cg::reduce(g, w, cg::plus<int>());
  unsigned long long base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(packed, ((unsigned long long)g.size() << 32) | (unsigned)tot);
  base = g.shfl(base, 0);
  const int pos = (int)(base >> 32) + (int)g.thread_rank();
  list[pos] = v;
  off[pos] = (unsigned)(base & 0xffffffffu) + (unsigned)pre;
}

// Append v (degree deg) to far pile p; the threads that append together share
// one atomic. False when the pile is full (the size counter may then pass the
// capacity: readers clamp it).
__device__ __forceinline__ bool pile_append(const Ctx& c, int p, int v, int deg) {
  cg::coalesced_group g = cg::coalesced_threads();
  unsigned base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(&c.ctl->psize[p], (unsigned)g.size());
  base = g.shfl(base, 0);
  const unsigned pos = base + g.thread_rank();
  if (pos >= c.pile_cap || pos < base) return false;
  c.pile[p][pos] = v;
  c.pdeg[p][pos] = deg;
  return true;
}

// Per-block distance histograms of the budgeted near/far ordering (shared
// memory; h null when off): h[0..kHistBins) for the next frontier (every near
// push adds the vertex's degree to the bin of its value, (val - fbase) >> shift
// clamped to the bins), h[kHistBins..) for the far pile (every new pile entry,
// relative to pbase). The block adds its bins to the device histograms once
// per launch.
struct Hists {
  unsigned* h;
  int fbase;
  int pbase;
  int shift;
};

__device__ __forceinline__ int hist_bin(int val, int base, int shift) {
  const long long off = ((long long)val - (long long)base) >> shift;
  return (int)(off < 0 ? 0 : (off >= kHistBins ? kHistBins - 1 : off));
}

__device__ __forceinline__ void hist_near(const Hists& hs, int val, int deg) {
  atomicAdd(&hs.h[hist_bin(val, hs.fbase, hs.shift)], (unsigned)deg);
}

__device__ __forceinline__ void hist_far(const Hists& hs, int val, int deg) {
  atomicAdd(&hs.h[kHistBins + hist_bin(val, hs.pbase, hs.shift)], (unsigned)deg);
}

// Defer v (new value val, at or above the threshold) to the current far pile.
// The pile's bitmap keeps one live entry per vertex: a vertex already on the
// pile only lowers the pile's minimum. Vertices without edges are never
// deferred. With a warp stage the entry is staged (published by warp_flush
// with one atomic per flush); without one it is appended at once. False when
// the pile is full: the caller then pushes v into the next frontier, which is
// always valid. With the edge budget (hs) new entries are histogrammed.
struct WarpStage;
__device__ __forceinline__ bool stage_far(const Ctx& c, WarpStage* ws, int v, int deg);

__device__ __forceinline__ bool defer_vertex(const Ctx& c, Acc& a, int v, int val, WarpStage* ws = nullptr,
                                             const Hists* hs = nullptr) {
  const unsigned bit = 1u << (v & 31);
  unsigned* w = &c.fbm[v >> 5];
  if (*(volatile unsigned*)w & bit) {
    a.fmin = min(a.fmin, val);
    return true;
  }
  if (atomicOr(w, bit) & bit) {
    a.fmin = min(a.fmin, val);
    return true;
  }
  const int deg = c.g.nindex[v + 1] - c.g.nindex[v];
  if (deg == 0) {
    atomicAnd(w, ~bit);
    return true;
  }
  if (ws ? !stage_far(c, ws, v, deg) : !pile_append(c, c.ctl->pcur, v, deg)) {
    atomicAnd(w, ~bit);
    return false;
  }
  a.fmin = min(a.fmin, val);
  if (hs) hist_far(*hs, val, deg);
  return true;
}

// A near push of v supersedes v's pile entry, if any (its bit is cleared, so
// the entry is dropped when the pile is next read). Needed where the
// threshold may fall (the edge budget): there a pile entry cannot be told
// stale from its value alone.
__device__ __forceinline__ void unpile(const Ctx& c, int v) {
  const unsigned bit = 1u << (v & 31);
  unsigned* w = &c.fbm[v >> 5];
  if (*(volatile unsigned*)w & bit) atomicAnd(w, ~bit);
}

// Record vertex v (degree deg >= 1) in the next frontier. The bitmap bit is
// already set, and the frontier minimum already updated, by the caller.
__device__ __forceinline__ void stage_entry(const Ctx& c, Stage& s, Acc& a, int nxt, int v, int deg) {
  a.maxdeg = max(a.maxdeg, deg);
  int p = atomicAdd(&s.n, 1);
  if (p < kQueue) {
    s.q[p] = v;
    s.qd[p] = deg;
  } else {
    direct_append(&c.ctl->slot[nxt].packed, c.wl[nxt], c.woff[nxt], v, deg);
  }
  if (deg >= c.heavy) {
    const int t = heavy_tiles(deg);
    p = atomicAdd(&s.hn, 1);
    if (p < kHQueue) {
      s.hq[p] = v;
      s.ht[p] = t;
    } else {
      direct_append(&c.ctl->slot[nxt].hpacked, c.hwl[nxt], c.htoff[nxt], v, t);
    }
  }
}

// Push after a successful atomicMin (old > val). The frontier minimum is
// lowered on every improvement, including repeat improvements of a vertex that
// is already in the next frontier, so it is a true lower bound of the values
// the next iteration reads. A plain read of the bitmap word skips the atomic
// for vertices already pushed in this launch (bits of the next frontier are
// only set during the launch, so a set bit that is read is never stale).
// Vertices without edges leave the frontier at once.
__device__ __forceinline__ void push_vertex(const Ctx& c, Stage& s, Acc& a, int nxt, int v, int val, int old) {
  if (old == kInf) a.visited++;
  a.mindist = min(a.mindist, val);
  const unsigned bit = 1u << (v & 31);
  unsigned* w = &c.bm[nxt][v >> 5];
  if (*(volatile unsigned*)w & bit) return;
  if (atomicOr(w, bit) & bit) return;
  const int deg = c.g.nindex[v + 1] - c.g.nindex[v];
  if (deg == 0) {
    atomicAnd(w, ~bit);
    return;
  }
  stage_entry(c, s, a, nxt, v, deg);
}

// Exclusive scan of up to kHQueue ints in shared memory by warp 0.
__device__ __forceinline__ int warp_scan_heavy(Stage& s, int hn) {
  constexpr int kPer = kHQueue / kWarp;
  const int lane = threadIdx.x & 31;
  int loc[kPer];
  int sum = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int j = lane * kPer + i;
    loc[i] = sum;
    sum += j < hn ? s.ht[j] : 0;
  }
  int incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int excl = incl - sum;
  const int tot = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int j = lane * kPer + i;
    if (j < hn) s.ht[j] = excl + loc[i];
  }
  return tot;
}

// Publish the staged pushes of this block (block-uniform call): one packed
// atomic reserves positions and edge offsets for all staged entries.
__device__ __forceinline__ void stage_flush(const Ctx& c, Stage& s, int nxt) {
  __syncthreads();
  const int n = min(s.n, kQueue);
  const int hn = min(s.hn, kHQueue);
  __syncthreads();  // every thread has read the counters before anyone changes them
  if (n == 0 && hn == 0) return;
  const int t = threadIdx.x;
  int d[kScanItems];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const int j = t * kScanItems + i;
    d[i] = j < n ? s.qd[j] : 0;
  }
  int tot = 0;
  BlockScanT(s.scan).ExclusiveSum(d, d, tot);
  if (hn && t < 32) {
    const int htot = warp_scan_heavy(s, hn);
    if (t == 0) s.hbase = atomicAdd(&c.ctl->slot[nxt].hpacked, ((unsigned long long)hn << 32) | (unsigned)htot);
  }
  if (t == 0) {
    if (n) s.base = atomicAdd(&c.ctl->slot[nxt].packed, ((unsigned long long)n << 32) | (unsigned)tot);
    s.n = 0;
    s.hn = 0;
  }
  __syncthreads();
  if (n) {
    const int b = (int)(s.base >> 32);
    const unsigned eb = (unsigned)(s.base & 0xffffffffu);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
      const int j = t * kScanItems + i;
      if (j < n) {
        c.wl[nxt][b + j] = s.q[j];
        c.woff[nxt][b + j] = eb + (unsigned)d[i];
      }
    }
  }
  if (hn) {
    const int b = (int)(s.hbase >> 32);
    const unsigned tb = (unsigned)(s.hbase & 0xffffffffu);
    for (int j = t; j < hn; j += blockDim.x) {
      c.hwl[nxt][b + j] = s.hq[j];
      c.htoff[nxt][b + j] = tb + (unsigned)s.ht[j];
    }
  }
  __syncthreads();
}

// Relax up to R candidate edges of this thread. All dist[] loads are issued
// before any atomicMin. A value read before another thread lowered it is only
// larger, which can cost an unneeded atomic but never skips an improvement.
template <int ALG, int R>
__device__ __forceinline__ void relax_batch(const Ctx& c, Stage& s, Acc& a, int nxt, const int* du, const int* nv,
                                            const int* wv, const bool* ok) {
  int cand[R], cur[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    cand[r] = ok[r] ? Op<ALG>::cand(du[r], wv[r]) : kInf;
    cur[r] = ok[r] ? c.dist[nv[r]] : kInf;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (cand[r] < cur[r]) {
      const int old = atomicMin(&c.dist[nv[r]], cand[r]);
      if (cand[r] < old) push_vertex(c, s, a, nxt, nv[r], cand[r], old);
    }
  }
}

// Relax CSR entries [lo, hi) of one source with value du. The calling group has
// gsize threads and this thread is `lane` in it. Aligned 16-byte units of nlist
// (and eweight) are read with one 128-bit load; a unit that would reach past
// the end of the arrays is read element by element.
template <int ALG>
__device__ __forceinline__ void relax_range(const Ctx& c, Stage& s, Acc& a, int nxt, int du, int lo, int hi, int lane,
                                            int gsize) {
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  const int dus[4] = {du, du, du, du};
  if (c.g.vec_ok && hi - lo >= 8) {
    // 64-bit index arithmetic: edges may come within a few units of INT_MAX
    const long long q0 = lo >> 2;
    const long long q1 = ((long long)hi + 3) >> 2;
    for (long long q = q0 + lane; q < q1; q += gsize) {
      const long long k0 = q << 2;
      int nv[4], wv[4] = {0, 0, 0, 0};
      bool ok[4];
      if (k0 + 3 < c.g.edges) {
        const int4 x = ld_adj(reinterpret_cast<const int4*>(nl + k0));
        nv[0] = x.x; nv[1] = x.y; nv[2] = x.z; nv[3] = x.w;
        if (Op<ALG>::kWeighted) {
          const int4 y = ld_adj(reinterpret_cast<const int4*>(ew + k0));
          wv[0] = y.x; wv[1] = y.y; wv[2] = y.z; wv[3] = y.w;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) ok[r] = k0 + r >= lo && k0 + r < hi;
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const long long k = k0 + r;
          ok[r] = k >= lo && k < hi;
          nv[r] = ok[r] ? nl[k] : 0;
          if (Op<ALG>::kWeighted) wv[r] = ok[r] ? ew[k] : 0;
        }
      }
      relax_batch<ALG, 4>(c, s, a, nxt, dus, nv, wv, ok);
    }
  } else {
    for (long long k0 = lo + (long long)lane * 4; k0 < hi; k0 += (long long)gsize * 4) {
      int nv[4], wv[4] = {0, 0, 0, 0};
      bool ok[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const long long k = k0 + r;
        ok[r] = k < hi;
        nv[r] = ok[r] ? ld_adj(nl + k) : 0;
        if (Op<ALG>::kWeighted) wv[r] = ok[r] ? ld_adj(ew + k) : 0;
      }
      relax_batch<ALG, 4>(c, s, a, nxt, dus, nv, wv, ok);
    }
  }
}

// Last j in [0, n) with off[j] <= x (off[0] == 0 <= x).
__device__ __forceinline__ int owner_search(const unsigned* off, int n, unsigned x) {
  int lo = 0, hi = n;
  while (hi - lo > 1) {
    const int mid = lo + ((hi - lo) >> 1);
    if (off[mid] <= x) lo = mid; else hi = mid;
  }
  return lo;
}

// Warp-cooperative version for global arrays (warp 0 calls it; every lane gets
// the result): each round probes 32 evenly spaced positions, so the range
// shrinks 32-fold per round of parallel loads instead of 2-fold per dependent load.
__device__ __forceinline__ int owner_search_warp(const unsigned* off, int n, unsigned x) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = n;  // off[lo] <= x, answer in [lo, hi)
  while (hi - lo > 32) {
    const long long span = hi - lo;
    const int p = lo + (int)((span * lane) / 32);
    const unsigned ballot = __ballot_sync(0xffffffffu, off[p] <= x);
    const int last = 31 - __clz(ballot);  // lane 0 always qualifies (p == lo)
    const int nlo = lo + (int)((span * last) / 32);
    const int nhi = last == 31 ? hi : lo + (int)((span * (last + 1)) / 32);
    lo = nlo;
    hi = nhi;
  }
  const int p = lo + lane;
  const unsigned ballot = __ballot_sync(0xffffffffu, p < hi && off[p] <= x);
  return lo + 31 - __clz(ballot);
}

// Flush only when the staging queue is at least half full (block-uniform).
__device__ __forceinline__ void stage_flush_if_half(const Ctx& c, Stage& s, int nxt) {
  __syncthreads();
  const bool full = s.n >= kQueue / 2 || s.hn >= kHQueue / 2;
  __syncthreads();
  if (full) stage_flush(c, s, nxt);
}

// Contiguous share [lo, hi) of [0, total) for this block among `nb` blocks.
__device__ __forceinline__ void block_share(unsigned total, int nb, unsigned* lo, unsigned* hi) {
  *lo = (unsigned)(((unsigned long long)total * blockIdx.x) / nb);
  *hi = (unsigned)(((unsigned long long)total * (blockIdx.x + 1)) / nb);
}

// Heavy frontier vertices: their adjacency is cut into tiles of kHeavyTile
// entries. Each block takes a contiguous share of the tile sequence, finds the
// vertex of its first tile once, and walks forward.
template <int ALG>
__device__ void heavy_path(const Ctx& c, Stage& s, Acc& a, int cur, int nxt, int active) {
  const unsigned long long hp = c.ctl->slot[cur].hpacked;
  const int nh = slot_size(hp);
  const unsigned ntiles = slot_edges(hp);
  if (ntiles == 0) return;
  unsigned t0, t1;
  block_share(ntiles, active, &t0, &t1);
  if (t0 >= t1) return;  // uniform
  const unsigned* toff = c.htoff[cur];
  if (threadIdx.x < 32) {
    const int j = owner_search_warp(toff, nh, t0);
    if (threadIdx.x == 0) s.j0 = j;
  }
  __syncthreads();
  int j = s.j0;
  for (unsigned t = t0; t < t1; ++t) {
    while (j + 1 < nh && toff[j + 1] <= t) ++j;
    const int u = c.hwl[cur][j];
    const int du = c.dist[u];
    const int beg = c.g.nindex[u];
    const int end = c.g.nindex[u + 1];
    const int lo = beg + (int)(t - toff[j]) * kHeavyTile;
    const int hi = min(end, lo + kHeavyTile);
    if (Op<ALG>::valid(du)) relax_range<ALG>(c, s, a, nxt, du, lo, hi, threadIdx.x, blockDim.x);
    stage_flush_if_half(c, s, nxt);
  }
}

// Clear the bitmap of F_{i-1} (slot old): by entries when it is small, by
// words otherwise. Spread over the launch's `active` blocks.
__device__ __forceinline__ void clear_old(const Ctx& c, int old, int active) {
  const int n = slot_size(c.ctl->slot[old].packed);
  unsigned* bm = c.bm[old];
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)active * blockDim.x;
  if ((long long)n * 4 > c.bm_words) {
    for (long long w = tid; w < c.bm_words; w += stride) bm[w] = 0u;
  } else {
    const int* wl = c.wl[old];
    for (long long j = tid; j < n; j += stride) bm[wl[j] >> 5] = 0u;
  }
}

static __device__ void finish_iteration(const Ctx& c, int i, int cur, int nxt, int old);

// Blocks of a launch that take part in it. Blocks at or above this index
// return at once, so a small frontier does not pay for the whole grid; the
// clearing of F_{i-1} is work too. Full sweeps pass `need` = gridDim.x.
__device__ __forceinline__ int active_blocks(const Ctx& c, int old, long long need) {
  const int n_old = slot_size(c.ctl->slot[old].packed);
  const long long clear = ((long long)n_old * 4 > c.bm_words) ? ((long long)c.bm_words + 8191) / 8192
                                                                : ((long long)n_old + 2047) / 2048;
  long long a = need > clear ? need : clear;
  if (a < 1) a = 1;
  if (a > gridDim.x) a = gridDim.x;
  return (int)a;
}

// Common epilogue: publish block statistics and let the last block finish the
// iteration. Every block of the launch, active or not, counts into `done`, so
// the iteration advances only after every block has read its state.
template <typename S>
__device__ __forceinline__ bool block_epilogue(const Ctx& c, S& s, const Acc& a, int i, int cur, int nxt, int old,
                                               int /*active*/) {
  acc_reduce(a, s);
  if (threadIdx.x == 0) {
    const Acc& r = s.red[0];
    Slot& sl = c.ctl->slot[nxt];
    if (r.maxdeg) atomicMax(&sl.maxdeg, r.maxdeg);
    if (r.mindist != kInf) atomicMin(&sl.mindist, r.mindist);
    if (r.visited) atomicAdd((unsigned long long*)&c.ctl->visited, (unsigned long long)r.visited);
    // far pushes of a relax or trim launch go onto pile pcur, a move's onto the other
    if (r.fmin != kInf) atomicMin(&c.ctl->pmin[c.ctl->split == 1 ? 1 - c.ctl->pcur : c.ctl->pcur], r.fmin);
    __threadfence();
    const unsigned t = atomicAdd(&c.ctl->done, 1u);
    s.last = (t == gridDim.x - 1);
  }
  __syncthreads();
  const bool last = s.last;
  if (last) {
    __threadfence();
    finish_iteration(c, i, cur, nxt, old);
  }
  return last;  // this block finished the iteration
}

// The launch's start time is taken by block 0, which the scheduler dispatches
// first; the last block reads it after every block has finished.
// Epilogue of a block with no work in this launch.
template <typename S>
__device__ __forceinline__ bool idle_epilogue(const Ctx& c, S& s, int i, int cur, int nxt, int old) {
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(&c.ctl->done, 1u);
    s.last = (t == gridDim.x - 1);
  }
  __syncthreads();
  const bool last = s.last;
  if (last) {
    __threadfence();
    finish_iteration(c, i, cur, nxt, old);
  }
  return last;  // this block finished the iteration
}

__device__ __forceinline__ void block_prologue(const Ctx& c) {
  if (blockIdx.x == 0 && threadIdx.x == 0) c.ctl->tstart = globaltimer();
}

// ---------------------------------------------------------------------------
// Data-driven push, vertex granularity: thread, warp or block per frontier
// vertex. Heavy vertices are skipped here and taken by the heavy path.

template <int ALG, int VAR>
__device__ __forceinline__ bool body_push(const Ctx& c, Stage& s) {
  block_prologue(c);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int n = slot_size(c.ctl->slot[cur].packed);
  const int per = VAR == kVPThread ? kBlock : (VAR == kVPWarp ? kBlock / kWarp : 1);
  const int active = active_blocks(c, old, ((long long)n + per - 1) / per + slot_edges(c.ctl->slot[cur].hpacked));
  if (blockIdx.x >= active) {
    return idle_epilogue(c, s, i, cur, nxt, old);
  }
  stage_init(s);
  Acc a;
  acc_init(a);
  clear_old(c, old, active);
  __syncthreads();
  const int* wl = c.wl[cur];

  for (;;) {
    if (threadIdx.x == 0) s.chunk = atomicAdd(&c.ctl->chunk, per);
    __syncthreads();
    const int base = s.chunk;
    if (base >= n) break;  // uniform
    if (VAR == kVPThread) {
      const int idx = base + threadIdx.x;
      if (idx < n) {
        const int u = wl[idx];
        const int beg = c.g.nindex[u], end = c.g.nindex[u + 1];
        const int du = c.dist[u];
        if (end - beg < c.heavy && Op<ALG>::valid(du)) relax_range<ALG>(c, s, a, nxt, du, beg, end, 0, 1);
      }
    } else if (VAR == kVPWarp) {
      const int idx = base + threadIdx.x / kWarp;
      if (idx < n) {
        const int u = wl[idx];
        const int beg = c.g.nindex[u], end = c.g.nindex[u + 1];
        const int du = c.dist[u];
        if (end - beg < c.heavy && Op<ALG>::valid(du))
          relax_range<ALG>(c, s, a, nxt, du, beg, end, threadIdx.x % kWarp, kWarp);
      }
    } else {
      const int u = wl[base];
      const int beg = c.g.nindex[u], end = c.g.nindex[u + 1];
      const int du = c.dist[u];
      if (end - beg < c.heavy && Op<ALG>::valid(du))
        relax_range<ALG>(c, s, a, nxt, du, beg, end, threadIdx.x, blockDim.x);
    }
    stage_flush_if_half(c, s, nxt);
  }
  heavy_path<ALG>(c, s, a, cur, nxt, active);
  stage_flush(c, s, nxt);
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Edge-balanced push: the frontier's edges [0, edges) are split into one
// contiguous share per warp of the grid (equal edges, hence equal work). A warp
// finds the frontier entry holding its first edge once (warp-cooperative
// search) and walks its share in warp tiles of kWarpTile edges: it loads the
// entries overlapping the tile into its own slice of shared memory, and each
// lane relaxes kEdgesPerThread consecutive edges. Warps never wait for each
// other: each stages its pushes in its own queue and publishes them with a
// warp scan and one packed atomic. No vertex is too big or too small: work is
// split by edges, as in the reference's edge-centric codes.
constexpr int kWarpTile = kWarp * kEdgesPerThread;  // edges per warp tile
// Warp staging capacity (overflow appends directly); a warp flushes once it
// holds half of it, and a tile pushes at most kWarpTile entries. 192 rather
// than 256: the 5 KB less shared memory per block is L1 for the random value
// and bitmap reads (RMAT-22 SSSP 4% faster; 128 loses on grids).
#ifndef I2_WARP_QUEUE
#define I2_WARP_QUEUE 192
#endif
constexpr int kWarpQueue = I2_WARP_QUEUE;
static_assert(kWarpQueue % kWarp == 0 && kWarpQueue / 2 + kWarpTile <= kWarpQueue,
              "a tile's pushes must fit after a half-full queue");
constexpr int kWarpsPerBlock = kBlock / kWarp;

struct WarpStage {
  unsigned off[kWarpTile + kWarp];
  int beg[kWarpTile];
  int du[kWarpTile];
  int q[kWarpQueue];
  int qd[kWarpQueue];
  int n;
};

// Stage a push into the warp's queue (heavy entries go straight to their list).
__device__ __forceinline__ void warp_stage_entry(const Ctx& c, WarpStage& ws, Acc& a, int nxt, int v, int deg) {
  a.maxdeg = max(a.maxdeg, deg);
  const int p = atomicAdd(&ws.n, 1);
  if (p < kWarpQueue) {
    ws.q[p] = v;
    ws.qd[p] = deg;
  } else {
    direct_append(&c.ctl->slot[nxt].packed, c.wl[nxt], c.woff[nxt], v, deg);
  }
  if (deg >= c.heavy) direct_append(&c.ctl->slot[nxt].hpacked, c.hwl[nxt], c.htoff[nxt], v, heavy_tiles(deg));
}

// Stage a far-pile entry of the near/far ordering: kept in the warp's queue
// as ~v (negative) beside its degree, and published by warp_flush<true>.
// Without room in the queue it is appended at once.
__device__ __forceinline__ bool stage_far(const Ctx& c, WarpStage* ws, int v, int deg) {
  const int p = atomicAdd(&ws->n, 1);
  if (p < kWarpQueue) {
    ws->q[p] = ~v;
    ws->qd[p] = deg;
    return true;
  }
  return pile_append(c, c.ctl->pcur, v, deg);
}

template <bool DEFER>
__device__ __forceinline__ void warp_push_vertex(const Ctx& c, WarpStage& ws, Acc& a, int nxt, int v, int val,
                                                 int old, int thr, const Hists& hs) {
  if (old == kInf) a.visited++;
  if (DEFER && val >= thr && defer_vertex(c, a, v, val, &ws, hs.h ? &hs : nullptr)) return;
  if (DEFER && hs.h) unpile(c, v);
  a.mindist = min(a.mindist, val);
  const unsigned bit = 1u << (v & 31);
  unsigned* w = &c.bm[nxt][v >> 5];
  if (*(volatile unsigned*)w & bit) return;
  if (atomicOr(w, bit) & bit) return;
  const int deg = c.g.nindex[v + 1] - c.g.nindex[v];
  if (deg == 0) {
    atomicAnd(w, ~bit);
    return;
  }
  if (DEFER && hs.h) hist_near(hs, val, deg);
  warp_stage_entry(c, ws, a, nxt, v, deg);
}

// Publish the warp's staged entries (warp-uniform call): one packed atomic
// reserves positions and edge offsets in the next frontier for all of them.
// DEFER: the queue also holds far-pile entries (negative, ~v); they go onto
// the current pile with one more atomic, and the frontier entries are
// compacted. Far entries that find the pile full join the next frontier.
template <bool DEFER = false>
__device__ __forceinline__ void warp_flush(const Ctx& c, WarpStage& ws, int nxt) {
  constexpr int kPer = kWarpQueue / kWarp;
  __syncwarp();
  const int n = min(ws.n, kWarpQueue);
  __syncwarp();
  if (n == 0) return;
  const int lane = threadIdx.x & 31;
  if constexpr (DEFER) {
    int nf = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int j = lane * kPer + i;
      nf += (j < n && ws.q[j] < 0) ? 1 : 0;
    }
    int fincl = nf;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, fincl, o);
      if (lane >= o) fincl += y;
    }
    const int ftot = __shfl_sync(0xffffffffu, fincl, 31);
    if (ftot) {
      const int p = c.ctl->pcur;
      unsigned pb = 0;
      if (lane == 0) pb = atomicAdd(&c.ctl->psize[p], (unsigned)ftot);
      pb = __shfl_sync(0xffffffffu, pb, 0);
      unsigned k = pb + (unsigned)(fincl - nf);
      for (int i = 0; i < kPer; ++i) {
        const int j = lane * kPer + i;
        if (j < n && ws.q[j] < 0) {
          const int v = ~ws.q[j];
          if (k < c.pile_cap && k >= pb) {
            c.pile[p][k] = v;
            c.pdeg[p][k] = ws.qd[j];
          } else {  // pile full: the vertex joins the next frontier instead
            const unsigned bit = 1u << (v & 31);
            atomicAnd(&c.fbm[v >> 5], ~bit);
            if (!(atomicOr(&c.bm[nxt][v >> 5], bit) & bit)) {
              ws.q[j] = v;
              if (ws.qd[j] >= c.heavy)
                direct_append(&c.ctl->slot[nxt].hpacked, c.hwl[nxt], c.htoff[nxt], v, heavy_tiles(ws.qd[j]));
            }
          }
          ++k;
        }
      }
      __syncwarp();
    }
  }
  if constexpr (!DEFER) {
    int d[kPer];
    int sum = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int j = lane * kPer + i;
      d[i] = sum;
      sum += j < n ? ws.qd[j] : 0;
    }
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    const int excl = incl - sum;
    const int tot = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 0) {
      base = atomicAdd(&c.ctl->slot[nxt].packed, ((unsigned long long)n << 32) | (unsigned)tot);
      ws.n = 0;
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    const int b = (int)(base >> 32);
    const unsigned eb = (unsigned)(base & 0xffffffffu);
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int j = lane * kPer + i;
      if (j < n) {
        c.wl[nxt][b + j] = ws.q[j];
        c.woff[nxt][b + j] = eb + (unsigned)(excl + d[i]);
      }
    }
    __syncwarp();
    return;
  }
  // frontier entries: count and degree prefix in one 64-bit scan
  unsigned long long d[kPer];
  unsigned long long sum = 0;
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int j = lane * kPer + i;
    d[i] = sum;
    if (j < n && ws.q[j] >= 0) sum += (1ull << 32) | (unsigned)ws.qd[j];
  }
  unsigned long long incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const unsigned long long excl = incl - sum;
  const unsigned long long tot = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 0) {
    if (tot) base = atomicAdd(&c.ctl->slot[nxt].packed, tot);
    ws.n = 0;
  }
  base = __shfl_sync(0xffffffffu, base, 0);
  const int b = (int)(base >> 32);
  const unsigned eb = (unsigned)(base & 0xffffffffu);
#pragma unroll
  for (int i = 0; i < kPer; ++i) {
    const int j = lane * kPer + i;
    if (j < n && ws.q[j] >= 0) {
      const unsigned long long x = excl + d[i];
      c.wl[nxt][b + (int)(x >> 32)] = ws.q[j];
      c.woff[nxt][b + (int)(x >> 32)] = eb + (unsigned)(x & 0xffffffffu);
    }
  }
  __syncwarp();
}

template <int ALG, bool DEFER>
__device__ __forceinline__ void warp_relax_batch(const Ctx& c, WarpStage& ws, Acc& a, int nxt, const int* du,
                                                 const int* nv, const int* wv, const bool* ok, int thr,
                                                 const Hists& hs) {
  int cand[kEdgesPerThread], cur[kEdgesPerThread];
#pragma unroll
  for (int r = 0; r < kEdgesPerThread; ++r) {
    cand[r] = ok[r] ? Op<ALG>::cand(du[r], wv[r]) : kInf;
    cur[r] = ok[r] ? c.dist[nv[r]] : kInf;
  }
#pragma unroll
  for (int r = 0; r < kEdgesPerThread; ++r) {
    if (cand[r] < cur[r]) {
      const int old = atomicMin(&c.dist[nv[r]], cand[r]);
      if (cand[r] < old) warp_push_vertex<DEFER>(c, ws, a, nxt, nv[r], cand[r], old, thr, hs);
    }
  }
}

struct EpiStage {
  Acc red[kBlock / kWarp];
  int last;
};

#ifndef I2_EB_MIN_BLOCKS
#define I2_EB_MIN_BLOCKS 6
#endif
// Resident blocks per SM that the selectors' kernels (every style in one
// kernel) are compiled for: 4 leaves them 64 registers, where 6 (the fixed
// styles' 40) spilled 160-224 bytes per thread. Held-out RMAT/ER/grid graphs
// of 2^18 and 2^20 vertices, geomean time against 6: BFS 0.90, SSSP 0.97-0.98,
// CC 0.97-0.98 for both selectors (5 blocks: 0.93-0.98); grid 4096² BFS 0.92.
// On RMAT-26 the heuristic BFS took 1.21x as long at 4 blocks (its pull
// iterations over 2^26 vertices need the warps), so graphs of
// kWideSelectorNodes vertices or more get the selector kernel compiled for the
// fixed styles' I2_EB_MIN_BLOCKS.
#ifndef I2_SEL_MIN_BLOCKS
#define I2_SEL_MIN_BLOCKS 4
#endif

struct EBShared {
  EpiStage s;
  WarpStage wss[kWarpsPerBlock];
};

// Near/far ordering: the per-block distance histogram of the edge budget.
static_assert(kHistBins == kBlock, "one histogram bin per thread");
struct EBSharedFar : EBShared {
  unsigned hist[2 * kHistBins];  // next frontier, far pile
};

template <bool DEFER>
using EBSharedT = typename std::conditional<DEFER, EBSharedFar, EBShared>::type;

// Budgeted near/far ordering, start of a launch (block-uniform): clear the
// block's histograms. End of a launch: add them to the device histograms.
__device__ __forceinline__ void block_hist_begin(unsigned* h) {
  h[threadIdx.x] = 0u;
  h[kHistBins + threadIdx.x] = 0u;
  __syncthreads();
}

__device__ __forceinline__ void block_hist_end(const unsigned* h, unsigned long long* dst) {
  __syncthreads();
  const unsigned x = h[threadIdx.x], y = h[kHistBins + threadIdx.x];
  if (x) atomicAdd(&dst[threadIdx.x], (unsigned long long)x);
  if (y) atomicAdd(&dst[kHistBins + threadIdx.x], (unsigned long long)y);
}

// Launches of the SSSP near/far ordering other than relaxations (Ctl::split):
//  1 move: F_i is empty, the pile is not, and the threshold has just risen
//    from T0 to T. Each live pile entry with a distance below T moves into
//    F_{i+1}; one at or above T moves onto the other pile. Fixed step: an entry
//    whose distance is below T0 was lowered after it was deferred by a push
//    that put it into a frontier (values only fall and the threshold only
//    rises), so it has been relaxed with that distance and is dropped. Edge
//    budget: an entry is live while its fbm bit is set (a near push clears it)
//    and dead entries are dropped; the first copy of a vertex that moves clears
//    the bit, so it moves once; the kept entries are histogrammed anew (base T)
//    for the next move.
//  3 trim (edge budget): F_i carries more than twice the budget and the
//    threshold has just fallen to T; entries below T move into F_{i+1}, the
//    others onto the pile (nothing is relaxed).
// The loop is block-uniform: a block appends the entries it keeps with one
// atomic per pass (a single pile counter takes every block's appends).
__device__ __forceinline__ bool body_split(const Ctx& c, EBSharedFar& sh, int i, int cur, int nxt, int old) {
  __shared__ int s_keep[kWarpsPerBlock];
  __shared__ unsigned s_kbase;
  EpiStage& s = sh.s;
  Ctl* ctl = c.ctl;
  const int mode = ctl->split;
  const bool budget = ctl->delta < 0;
  const int p = ctl->pcur;
  const unsigned long long P = ctl->slot[cur].packed;
  // F_i's entries first (a trim's input, or what an early move carries), then
  // the pile's (a move)
  const unsigned nf = (unsigned)slot_size(P);
  const unsigned n = nf + (mode == 1 ? min(ctl->psize[p], c.pile_cap) : 0u);
  const int T = ctl->threshold, T0 = ctl->prev_threshold;
  const Hists hs = budget ? Hists{sh.hist, ctl->hbase, ctl->pbase, ctl->hshift} : Hists{};
  const int active = active_blocks(c, old, ((long long)n + kBlock - 1) / kBlock);
  if (blockIdx.x >= active) {
    return idle_epilogue(c, s, i, cur, nxt, old);
  }
  if (threadIdx.x == 0) s.last = 0;
  Acc a;
  acc_init(a);
  if (budget) block_hist_begin(sh.hist);
  clear_old(c, old, active);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  WarpStage& ws = sh.wss[wid];
  if (lane == 0) ws.n = 0;
  __syncwarp();
  const int* pv = c.pile[p];
  const int* pd = c.pdeg[p];
  // kR entries per thread and pass (L2-coherent loads: other blocks wrote
  // these arrays in earlier iterations). kR = 4 measured no faster on RMAT-22
  // moves and slower on trims (fewer blocks share a small frontier).
  constexpr int kR = 1;
  const unsigned stride = (unsigned)active * kBlock * kR;
  for (unsigned base = blockIdx.x * kBlock * kR; base < n; base += stride) {
    int v[kR], d[kR], deg[kR];
    unsigned fw[kR];
    bool in[kR], front[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      const unsigned j = base + (unsigned)r * kBlock + threadIdx.x;
      in[r] = j < n;
      front[r] = j < nf;
      v[r] = in[r] ? (front[r] ? __ldcg(&c.wl[cur][j]) : __ldcg(&pv[j - nf])) : 0;
      deg[r] = 0;
      if (in[r]) {
        if (front[r]) {
          const unsigned w1 = j + 1 < nf ? __ldcg(&c.woff[cur][j + 1]) : slot_edges(P);
          deg[r] = (int)(w1 - __ldcg(&c.woff[cur][j]));
        } else {
          deg[r] = __ldcg(&pd[j - nf]);
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      fw[r] = in[r] && !front[r] ? __ldcg(&c.fbm[v[r] >> 5]) : 0u;
      d[r] = in[r] ? __ldcg(&c.dist[v[r]]) : 0;
    }
    bool keep[kR];
    int nkeep = 0;
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      keep[r] = false;
      if (!in[r]) continue;
      const unsigned bit = 1u << (v[r] & 31);
      if (front[r]) {  // a frontier entry: below T it stays near, else it goes onto the pile
        if (d[r] >= T && defer_vertex(c, a, v[r], d[r], &ws, budget ? &hs : nullptr)) {
          // on the pile
        } else if (!(atomicOr(&c.bm[nxt][v[r] >> 5], bit) & bit)) {
          a.mindist = min(a.mindist, d[r]);
          if (budget) hist_near(hs, d[r], deg[r]);
          warp_stage_entry(c, ws, a, nxt, v[r], deg[r]);
        }
      } else if (budget) {  // a pile entry (move), live while its fbm bit is set
        if (fw[r] & bit) {
          if (d[r] < T) {
            if ((atomicAnd(&c.fbm[v[r] >> 5], ~bit) & bit) && !(atomicOr(&c.bm[nxt][v[r] >> 5], bit) & bit)) {
              a.mindist = min(a.mindist, d[r]);
              hist_near(hs, d[r], deg[r]);
              warp_stage_entry(c, ws, a, nxt, v[r], deg[r]);
            }
          } else {
            keep[r] = true;
            a.fmin = min(a.fmin, d[r]);
            hist_far(hs, d[r], deg[r]);
          }
        }
      } else if (d[r] < T) {  // fixed step
        atomicAnd(&c.fbm[v[r] >> 5], ~bit);
        if (d[r] >= T0) {
          atomicOr(&c.bm[nxt][v[r] >> 5], bit);
          a.mindist = min(a.mindist, d[r]);
          warp_stage_entry(c, ws, a, nxt, v[r], deg[r]);
        }
      } else {
        keep[r] = true;
        a.fmin = min(a.fmin, d[r]);
      }
      nkeep += keep[r] ? 1 : 0;
    }
    if (mode == 1) {  // kept entries onto the other pile: one atomic per block pass
      int incl = nkeep;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      if (lane == 31) s_keep[wid] = incl;
      __syncthreads();
      if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kWarpsPerBlock; ++w) {
          const int x = s_keep[w];
          s_keep[w] = t;
          t += x;
        }
        s_kbase = t ? atomicAdd(&ctl->psize[1 - p], (unsigned)t) : 0u;
      }
      __syncthreads();
      unsigned pos = s_kbase + (unsigned)s_keep[wid] + (unsigned)(incl - nkeep);
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        if (keep[r]) {
          if (pos < c.pile_cap) {  // kept entries <= pile entries <= capacity
            c.pile[1 - p][pos] = v[r];
            c.pdeg[1 - p][pos] = deg[r];
          }
          ++pos;
        }
      }
      __syncthreads();  // s_keep and s_kbase are rewritten by the next pass
    }
    __syncwarp();
    if (ws.n >= kWarpQueue - kR * kWarp) warp_flush<true>(c, ws, nxt);
  }
  warp_flush<true>(c, ws, nxt);
  if (budget) block_hist_end(sh.hist, c.hist);
  __syncthreads();
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// DEFER: SSSP near/far ordering (pushes at or above the threshold go onto the
// far pile, and split launches refill the frontier from it).
template <int ALG, bool DEFER = false>
__device__ __forceinline__ bool body_edge_balanced(const Ctx& c, EBSharedT<DEFER>& sh) {
  static_assert(!DEFER || ALG == kSSSP, "near/far ordering is for SSSP");
  EpiStage& s = sh.s;
  block_prologue(c);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  if constexpr (DEFER) {
    if (c.ctl->split) return body_split(c, sh, i, cur, nxt, old);
  }
  const int thr = DEFER ? c.ctl->threshold : kInf;
  Hists hs{};
  if constexpr (DEFER) {
    if (c.ctl->delta < 0) hs = Hists{sh.hist, c.ctl->hbase, c.ctl->pbase, c.ctl->hshift};
  }
  const unsigned long long P = c.ctl->slot[cur].packed;
  const int n = slot_size(P);
  const unsigned total = slot_edges(P);
  const int active = active_blocks(c, old, ((long long)total + kWarpTile * kWarpsPerBlock - 1) /
                                              (kWarpTile * kWarpsPerBlock));
  if (blockIdx.x >= active) {
    return idle_epilogue(c, s, i, cur, nxt, old);
  }
  if (threadIdx.x == 0) s.last = 0;
  Acc a;
  acc_init(a);
  if (DEFER && hs.h) block_hist_begin(hs.h);
  clear_old(c, old, active);
  const int lane = threadIdx.x & 31;
  WarpStage& ws = sh.wss[threadIdx.x >> 5];
  if (lane == 0) ws.n = 0;
  __syncwarp();
  const int* wl = c.wl[cur];
  const unsigned* woff = c.woff[cur];
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  // Only as many warps as there are warp tiles take part, so a small frontier
  // is not spread over (and searched by) every warp of the grid.
  const unsigned long long gw = (unsigned long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const unsigned long long need = ((unsigned long long)total + kWarpTile - 1) / kWarpTile;
  const unsigned long long nw = need < (unsigned long long)active * kWarpsPerBlock
                                    ? (need > 0 ? need : 1)
                                    : (unsigned long long)active * kWarpsPerBlock;
  const unsigned W0 = gw < nw ? (unsigned)((total * gw) / nw) : 0u;
  const unsigned W1 = gw < nw ? (unsigned)((total * (gw + 1)) / nw) : 0u;
  if (W0 < W1) {
    int j = owner_search_warp(woff, n, W0);  // entry holding edge W0
    for (unsigned e0 = W0; e0 < W1; e0 += kWarpTile) {
      const unsigned e1 = min(W1, e0 + kWarpTile);
      // offsets of the entries from j on, 32 at a time, until one reaches e1;
      // each batch's vertex ids are loaded with its offsets, and the adjacency
      // start and value of the entries inside the tile right after
      int m = 0;
      for (;;) {
        const int jj = j + m + lane;
        const bool in = jj < n;
        const unsigned w = in ? woff[jj] : total;
        const int v = in ? wl[jj] : 0;
        ws.off[m + lane] = w;
        const int below = __popc(__ballot_sync(0xffffffffu, w < e1));
        if (lane < below) {  // offsets ascend: the entries below e1 are a prefix
          ws.beg[m + lane] = c.g.nindex[v];
          ws.du[m + lane] = c.dist[v];
        }
        m += below;
        if (below < kWarp) break;
      }
      __syncwarp();
      const unsigned x0 = e0 + (unsigned)lane * kEdgesPerThread;
      int du[kEdgesPerThread], nv[kEdgesPerThread], wv[kEdgesPerThread];
      bool ok[kEdgesPerThread];
      int o = x0 < e1 ? owner_search(ws.off, m, x0) : 0;
#pragma unroll
      for (int r = 0; r < kEdgesPerThread; ++r) {
        const unsigned x = x0 + r;
        ok[r] = x < e1;
        nv[r] = 0;
        wv[r] = 0;
        du[r] = kInf;
        if (ok[r]) {
          while (x >= ws.off[o + 1]) ++o;
          const int e = ws.beg[o] + (int)(x - ws.off[o]);
          nv[r] = ld_adj(nl + e);
          if (Op<ALG>::kWeighted) wv[r] = ld_adj(ew + e);
          du[r] = ws.du[o];
          ok[r] = Op<ALG>::valid(du[r]);
        }
      }
      warp_relax_batch<ALG, DEFER>(c, ws, a, nxt, du, nv, wv, ok, thr, hs);
      // the next tile starts at e1: its first entry is the last one with offset <= e1
      j += (ws.off[m] == e1) ? m : m - 1;
      __syncwarp();
      if (ws.n >= kWarpQueue / 2) warp_flush<DEFER>(c, ws, nxt);
    }
  }
  warp_flush<DEFER>(c, ws, nxt);
  if (DEFER && hs.h) block_hist_end(hs.h, c.hist);
  __syncthreads();
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Bitmap-gated topology sweep: thread per vertex, light vertices only; heavy
// frontier vertices take the shared heavy path.
template <int ALG>
__device__ __forceinline__ bool body_push_topo(const Ctx& c, Stage& s) {
  block_prologue(c);
  stage_init(s);
  Acc a;
  acc_init(a);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int active = gridDim.x;  // topology sweeps use the whole grid
  clear_old(c, old, active);
  __syncthreads();
  const unsigned* bmc = c.bm[cur];
  const int V = c.g.nodes;
  for (long long base = (long long)blockIdx.x * kBlock; base < V; base += (long long)gridDim.x * kBlock) {
    const int v = (int)base + threadIdx.x;
    if (v < V && ((bmc[v >> 5] >> (v & 31)) & 1u)) {
      const int beg = c.g.nindex[v];
      const int end = c.g.nindex[v + 1];
      const int du = c.dist[v];
      if (end - beg < c.heavy && Op<ALG>::valid(du)) relax_range<ALG>(c, s, a, nxt, du, beg, end, 0, 1);
    }
    stage_flush_if_half(c, s, nxt);
  }
  heavy_path<ALG>(c, s, a, cur, nxt, active);
  stage_flush(c, s, nxt);
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Edge-centric sweep over all CSR entries, gated by the source's frontier bit.
template <int ALG>
__device__ __forceinline__ bool body_edge_topo(const Ctx& c, Stage& s) {
  block_prologue(c);
  stage_init(s);
  Acc a;
  acc_init(a);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int active = gridDim.x;  // topology sweeps use the whole grid
  clear_old(c, old, active);
  __syncthreads();
  const unsigned* bmc = c.bm[cur];
  const int E = c.g.edges;
  const long long units = ((long long)E + 3) >> 2;
  const int* __restrict__ sp = c.g.sp;
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  for (long long base = (long long)blockIdx.x * kBlock; base < units; base += (long long)gridDim.x * kBlock) {
    const long long q = base + threadIdx.x;
    if (q < units) {
      const long long k0 = q << 2;
      int su[4], nv[4], wv[4] = {0, 0, 0, 0}, du[4];
      bool ok[4];
      if (c.g.vec_ok && k0 + 3 < E) {
        const int4 x = ld_adj(reinterpret_cast<const int4*>(sp + k0));
        su[0] = x.x; su[1] = x.y; su[2] = x.z; su[3] = x.w;
        const int4 y = ld_adj(reinterpret_cast<const int4*>(nl + k0));
        nv[0] = y.x; nv[1] = y.y; nv[2] = y.z; nv[3] = y.w;
        if (Op<ALG>::kWeighted) {
          const int4 z = ld_adj(reinterpret_cast<const int4*>(ew + k0));
          wv[0] = z.x; wv[1] = z.y; wv[2] = z.z; wv[3] = z.w;
        }
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const long long k = k0 + r;
          su[r] = (k < E) ? sp[k] : -1;
          nv[r] = (k < E) ? nl[k] : 0;
          if (Op<ALG>::kWeighted) wv[r] = (k < E) ? ew[k] : 0;
        }
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int u = su[r];
        ok[r] = u >= 0 && ((bmc[u >> 5] >> (u & 31)) & 1u);
        du[r] = ok[r] ? c.dist[u] : kInf;
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) ok[r] = ok[r] && Op<ALG>::valid(du[r]);
      relax_batch<ALG, 4>(c, s, a, nxt, du, nv, wv, ok);
    }
    stage_flush_if_half(c, s, nxt);
  }
  stage_flush(c, s, nxt);
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Pull variants (symmetric graphs only). Thread per destination vertex; a warp
// covers 32 consecutive vertices, i.e. exactly one bitmap word, so the next
// frontier's bitmap is written with one plain store per warp. dist[v] is only
// written by v's own thread, so no atomics are needed on it.
template <int ALG, bool FRONTIER>
__device__ __forceinline__ bool body_pull(const Ctx& c, Stage& s) {
  block_prologue(c);
  stage_init(s);
  Acc a;
  acc_init(a);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int active = gridDim.x;  // every vertex is visited
  clear_old(c, old, active);
  __syncthreads();
  const unsigned* bmc = c.bm[cur];
  const int V = c.g.nodes;
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  const int fmin = c.ctl->slot[cur].mindist;
  // Smallest candidate any frontier vertex can produce.
  const int bound = FRONTIER ? (fmin == kInf ? kInf : Op<ALG>::cand(fmin, c.gs.wmin)) : INT_MIN;
  for (long long base = (long long)blockIdx.x * kBlock; base < V; base += (long long)gridDim.x * kBlock) {
    const int v = (int)base + threadIdx.x;
    bool improved = false;
    int best = kInf, dv = kInf, deg = 0;
    if (v < V) {
      dv = c.dist[v];
      best = dv;
      if (!FRONTIER || dv > bound) {
        const int beg = c.g.nindex[v];
        const int end = c.g.nindex[v + 1];
        deg = end - beg;
        for (int k = beg; k < end; ++k) {
          const int u = ld_adj(nl + k);
          if (FRONTIER && !((bmc[u >> 5] >> (u & 31)) & 1u)) continue;
          const int du = c.dist[u];
          if (!Op<ALG>::valid(du)) continue;
          const int cd = Op<ALG>::cand(du, Op<ALG>::kWeighted ? ld_adj(ew + k) : 0);
          if (cd < best) {
            best = cd;
            if (FRONTIER && best == bound) break;
          }
        }
        if (best < dv) {
          c.dist[v] = best;
          improved = true;
        }
      }
    }
    // A warp covers one whole bitmap word; lane 0's vertex lies in it.
    const unsigned word = __ballot_sync(0xffffffffu, improved);
    if ((threadIdx.x & 31) == 0 && word) c.bm[nxt][v >> 5] = word;
    if (improved) {
      if (dv == kInf) a.visited++;
      a.mindist = min(a.mindist, best);
      stage_entry(c, s, a, nxt, v, deg);
    }
    stage_flush_if_half(c, s, nxt);
  }
  stage_flush(c, s, nxt);
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Kernels: one per (algorithm, style) for fixed-style runs, and one dispatch
// kernel per algorithm for the selectors, whose blocks branch on the style
// chosen at the end of the previous iteration (one kernel node per iteration
// instead of a conditional SWITCH node).

// ---------------------------------------------------------------------------
// Union-find CC (kUnionFind; CC on symmetric graphs only). The labels are read
// as parent pointers: every label is a vertex of the same component with an ID
// no larger than the vertex's own (true of the initial labels and of every
// label propagation writes), so following labels ends at a vertex that is its
// own label, a root. The hook launch links, for every edge, the roots of its
// two ends, always the larger root below the smaller one with a compare-and-
// swap on the larger (which succeeds only while it is still a root). The
// smallest ID of a component is therefore never linked and ends as the root of
// the whole component; the compress launch sets every label to its root. The
// result is the minimum-ID labelling that label propagation converges to,
// reached from any propagation state in two launches.

// Root of x. With HALVE, each step also points the visited vertex at its
// grandparent (path halving): any ancestor is a valid label, and a vertex that
// is not a root never becomes one again, so these plain writes cannot undo a
// link. The loads may be served from this SM's L1 and so be stale: a stale
// parent is still an ancestor (links are never undone), and a vertex wrongly
// seen as a root only makes the linking compare-and-swap fail and return its
// true parent, from which the search continues (parents only decrease, so it
// ends). Cached loads matter: almost every find ends at a component's root,
// and reading that one entry from L2 every time serialises on it.
template <bool HALVE>
__device__ __forceinline__ int uf_find(int* p, int x) {
  for (;;) {
    const int px = p[x];
    if (px == x) return x;
    const int ppx = p[px];
    if (HALVE && ppx != px) p[x] = ppx;
    x = ppx;
  }
}

__device__ __forceinline__ void uf_union(int* p, int a, int b) {
  int ra = uf_find<true>(p, a), rb = uf_find<true>(p, b);
  while (ra != rb) {
    if (ra < rb) {
      const int t = ra;
      ra = rb;
      rb = t;
    }
    const int seen = atomicCAS(&p[ra], ra, rb);  // link the larger root below the smaller
    if (seen == ra) return;
    ra = uf_find<true>(p, seen);  // ra was linked meanwhile: continue from its root
    rb = uf_find<true>(p, rb);
  }
}

// Neighbours each vertex is linked with before the largest tree is sampled.
constexpr int kAfforestLinks = 2;
constexpr int kAfforestSamples = 1024;

// Root of x with coherent loads (the sampling after the first hook launch).
__device__ __forceinline__ int uf_find_fresh(int* p, int x) {
  for (;;) {
    const int px = *(volatile int*)&p[x];
    if (px == x) return x;
    x = px;
  }
}

// Boyer-Moore majority pairs (candidate, count) merge like single votes: a
// majority element of the union survives the merge of the parts' pairs.
__device__ __forceinline__ void vote_merge(int& cand, int& cnt, int c2, int n2) {
  if (c2 == cand) cnt += n2;
  else if (n2 > cnt) { cand = c2; cnt = n2 - cnt; }
  else cnt -= n2;
}

// Called by the whole last block of the first hook launch (kBlock threads):
// the roots of kAfforestSamples vertices spread over the graph, and the root
// held by a majority of them (Boyer-Moore vote, per thread, then merged across
// lanes and warps), taken as the largest tree. Any root would keep the result
// correct; the vote only decides how many vertices the second hook launch can
// skip. Registers and 64 bytes of shared memory: this runs in the epilogue of
// every relax kernel, whose shared-memory size sets the L1 left to it.
__device__ __forceinline__ void uf_sample_giant(const Ctx& c) {
  __shared__ int wc[kBlock / kWarp], wn[kBlock / kWarp];
  const int V = c.g.nodes;
  int cand = -1, cnt = 0;
  for (int k = threadIdx.x; k < kAfforestSamples; k += blockDim.x)
    vote_merge(cand, cnt, V > 0 ? uf_find_fresh(c.dist, (int)((unsigned)mis_priority(k) % (unsigned)V)) : 0, 1);
  for (int o = 16; o > 0; o >>= 1) {
    const int c2 = __shfl_down_sync(0xffffffffu, cand, o);
    const int n2 = __shfl_down_sync(0xffffffffu, cnt, o);
    vote_merge(cand, cnt, c2, n2);
  }
  if ((threadIdx.x & 31) == 0) {
    wc[threadIdx.x >> 5] = cand;
    wn[threadIdx.x >> 5] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) vote_merge(cand, cnt, wc[w], wn[w]);
    c.ctl->uf_giant = cand;
  }
  __syncthreads();
}

// Three launches (Ctl::uf_phase): (0) link every vertex with its first
// kAfforestLinks neighbours, after which the last block samples the largest
// tree; (1) link the remaining neighbours of every vertex whose root is not
// that tree's (an edge from a skipped vertex to a vertex outside the tree is
// linked from the other end, and an edge inside the tree changes nothing);
// (2) set every label to its root. Links put the larger root below the
// smaller one whatever the order, so the roots are the components' minimum
// IDs, as in a single pass over all edges (sampling scheme of Sutton et al.,
// "Optimizing parallel graph connectivity computation via subgraph sampling",
// IPDPS 2018). On graphs with a giant component the second launch skips most
// edges.
template <int ALG>
__device__ __forceinline__ bool body_union(const Ctx& c, Stage& s) {
  block_prologue(c);
  stage_init(s);
  Acc a;
  acc_init(a);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int active = gridDim.x;
  clear_old(c, old, active);
  int* p = c.dist;
  const int V = c.g.nodes;
  const int* __restrict__ nl = c.g.nlist;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int phase = c.ctl->uf_phase;
  if (phase == 0) {
    for (long long v = tid; v < V; v += stride) {
      const int b = c.g.nindex[v];
      const int e = min(c.g.nindex[v + 1], b + kAfforestLinks);
      for (int j = b; j < e; ++j) {
        const int u = ld_adj(nl + j);
        if (u != (int)v) uf_union(p, (int)v, u);
      }
    }
  } else if (phase == 1) {
    const int giant = c.ctl->uf_giant;
    for (long long v = tid; v < V; v += stride) {
      const int b = c.g.nindex[v] + kAfforestLinks;
      const int e = c.g.nindex[v + 1];
      if (b >= e || uf_find<true>(p, (int)v) == giant) continue;
      for (int j = b; j < e; ++j) {
        const int u = ld_adj(nl + j);
        if (u != (int)v) uf_union(p, (int)v, u);
      }
    }
  } else {
    // compress: read-only finds (a halving write could replace a finished
    // label with an intermediate ancestor), each thread writing its own labels
    for (long long v = tid; v < V; v += stride) {
      const int r = uf_find<false>(p, (int)v);
      if (r != (int)v) p[v] = r;
    }
  }
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Maximal independent set (kMIS; one style). A warp per frontier vertex v
// still undecided: its lanes scan v's neighbours for ones that outrank v. If one
// of them is in the set, v is out; if none is undecided (all out, or there are
// none), v is in; otherwise v waits. A vertex that decides pushes its undecided
// neighbours into the next frontier, so a waiting vertex is examined again as
// soon as a neighbour that outranks it decides. Decisions depend only on
// outranking vertices, whose decisions are final, so the set is the greedy one
// in decreasing rank whatever the order of the updates.
__device__ __forceinline__ bool body_mis(const Ctx& c, EBShared& sh) {
  EpiStage& s = sh.s;
  block_prologue(c);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  const int n = slot_size(c.ctl->slot[cur].packed);
  const int active = active_blocks(c, old, ((long long)n + kWarpsPerBlock - 1) / kWarpsPerBlock);
  if (blockIdx.x >= active) return idle_epilogue(c, s, i, cur, nxt, old);
  if (threadIdx.x == 0) s.last = 0;
  Acc a;
  acc_init(a);
  clear_old(c, old, active);
  const int lane = threadIdx.x & 31;
  WarpStage& ws = sh.wss[threadIdx.x >> 5];
  if (lane == 0) ws.n = 0;
  __syncwarp();
  const int* wl = c.wl[cur];
  volatile int* st = c.dist;
  const int* __restrict__ nl = c.g.nlist;
  const long long stride = (long long)active * kWarpsPerBlock;
  for (long long k = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); k < n; k += stride) {
    const int v = wl[k];
    if (st[v] != kMisUndecided) continue;  // warp-uniform
    const int pv = mis_priority(v);
    const int b = c.g.nindex[v], e = c.g.nindex[v + 1];
    bool in_set = false, waiting = false;
    for (int base = b; base < e; base += kWarp) {
      const int j = base + lane;
      if (j < e) {
        const int u = ld_adj(nl + j);
        if (u != v && mis_outranks(u, mis_priority(u), v, pv)) {
          const int su = st[u];
          in_set |= su == kMisIn;
          waiting |= su == kMisUndecided;
        }
      }
      if (__any_sync(0xffffffffu, in_set)) break;  // v is out whatever the rest holds
    }
    const bool out = __any_sync(0xffffffffu, in_set);
    const bool wait = !out && __any_sync(0xffffffffu, waiting);
    if (wait) continue;
    if (lane == 0) st[v] = out ? kMisOut : kMisIn;
    a.visited += lane == 0;
    for (int base = b; base < e; base += kWarp) {
      const int j = base + lane;
      if (j < e) {
        const int u = ld_adj(nl + j);
        if (u != v && st[u] == kMisUndecided) {
          const unsigned bit = 1u << (u & 31);
          unsigned* w = &c.bm[nxt][u >> 5];
          if (!(*(volatile unsigned*)w & bit) && !(atomicOr(w, bit) & bit))
            warp_stage_entry(c, ws, a, nxt, u, c.g.nindex[u + 1] - c.g.nindex[u]);
        }
      }
      __syncwarp();
      if (ws.n >= kWarpQueue / 2) warp_flush(c, ws, nxt);
    }
  }
  warp_flush(c, ws, nxt);
  __syncthreads();
  return block_epilogue(c, s, a, i, cur, nxt, old, active);
}

// ---------------------------------------------------------------------------
// Kernel wrappers.
template <int ALG, int VAR>
__global__ void __launch_bounds__(kBlock) relax_push(Ctx c) {
  __shared__ Stage s;
  body_push<ALG, VAR>(c, s);
}

template <int ALG>
__global__ void __launch_bounds__(kBlock, I2_EB_MIN_BLOCKS) relax_edge_balanced(Ctx c) {
  __shared__ EBShared sh;
  body_edge_balanced<ALG>(c, sh);
}

static __global__ void __launch_bounds__(kBlock, I2_EB_MIN_BLOCKS) relax_mis(Ctx c) {
  __shared__ EBShared sh;
  body_mis(c, sh);
}

// Edge-balanced SSSP push with near/far ordering (Ctl::delta != 0).
static __global__ void __launch_bounds__(kBlock, I2_EB_MIN_BLOCKS) relax_near_far(Ctx c) {
  __shared__ EBSharedFar sh;
  body_edge_balanced<kSSSP, true>(c, sh);
}

template <int ALG>
__global__ void __launch_bounds__(kBlock) relax_push_topo(Ctx c) {
  __shared__ Stage s;
  body_push_topo<ALG>(c, s);
}

template <int ALG>
__global__ void __launch_bounds__(kBlock) relax_edge_topo(Ctx c) {
  __shared__ Stage s;
  body_edge_topo<ALG>(c, s);
}

template <int ALG>
__global__ void __launch_bounds__(kBlock) relax_union(Ctx c) {
  __shared__ Stage s;
  body_union<ALG>(c, s);
}

template <int ALG, bool FRONTIER>
__global__ void __launch_bounds__(kBlock) relax_pull(Ctx c) {
  __shared__ Stage s;
  body_pull<ALG, FRONTIER>(c, s);
}

template <bool DEFER = false>
union AnyShared {
  Stage st;
  EBSharedT<DEFER> eb;
};

// ---------------------------------------------------------------------------
// Resident traversal: one launch runs the iterations one after another, the
// grid meeting at a barrier where separate launches would meet at a kernel
// boundary. The block that finishes an iteration (the last one to count into
// `done`) has already advanced the control block when it bumps bar_gen, which
// releases the others. Every wait is bounded by Ctl::stall_ns: a block that
// waits longer sets kStatusStall and leaves, and every other block leaves at
// its next wait, so the launch always ends. All blocks must be resident at
// once, which the cooperative launch attribute of the graph node guarantees.
// Data written in one iteration is read by other blocks in the next, so the
// bodies read the frontier lists, bitmaps and values with coherent loads only
// (the read-only path is used for the graph arrays alone).

// Thread 0 of a block: return once bar_gen has moved past `gen`, or once the
// wait has run out (status kStatusStall) or another block has given up.
__device__ __forceinline__ void grid_wait(Ctl* ctl, unsigned gen) {
  const unsigned long long t0 = globaltimer();
  const unsigned long long limit = *(volatile unsigned long long*)&ctl->stall_ns;
  for (unsigned k = 1;; ++k) {
    if (*(volatile unsigned*)&ctl->bar_gen != gen) break;
    if (*(volatile int*)&ctl->status & kStatusStall) break;
    __nanosleep(k < 256 ? 20 : 200);
    if ((k & 63) == 0 && globaltimer() - t0 > limit) {
      atomicOr(&ctl->status, kStatusStall);
      break;
    }
  }
}

template <int ALG, int VAR, bool DEFER>
__device__ __forceinline__ bool run_body(const Ctx& c, AnyShared<DEFER>& sh) {
  if constexpr (ALG == kMIS) {
    return body_mis(c, sh.eb);  // one style
  } else {
    const int v = VAR >= 0 ? VAR : *(volatile int*)&c.ctl->variant;  // uniform: written before the release
    switch (v) {
      case kVPThread: return body_push<ALG, kVPThread>(c, sh.st);
      case kVPWarp: return body_push<ALG, kVPWarp>(c, sh.st);
      case kVPCta: return body_edge_balanced<ALG, DEFER>(c, sh.eb);
      case kVPBlock: return body_push<ALG, kVPBlock>(c, sh.st);
      case kPullFrontier: return body_pull<ALG, true>(c, sh.st);
      case kPullTopo: return body_pull<ALG, false>(c, sh.st);
      case kEdgeTopo: return body_edge_topo<ALG>(c, sh.st);
      case kUnionFind:
        if constexpr (ALG == kCC) return body_union<ALG>(c, sh.st);
        [[fallthrough]];  // not allowed for BFS/SSSP
      default: return body_push_topo<ALG>(c, sh.st);
    }
  }
}

// VAR >= 0: that style every iteration; VAR < 0: the style picked for each
// iteration by the previous one (heuristic or learned selector).
template <int ALG, int VAR, bool DEFER = false, int MINB = (VAR < 0 ? I2_SEL_MIN_BLOCKS : I2_EB_MIN_BLOCKS)>
__global__ void __launch_bounds__(kBlock, MINB) relax_resident(Ctx c) {
  __shared__ AnyShared<DEFER> sh;
  __shared__ int s_go;
  Ctl* ctl = c.ctl;
  if (threadIdx.x == 0) s_go = !(*(volatile int*)&ctl->status & kStatusStall);
  __syncthreads();
  if (!s_go) {  // an earlier launch of this traversal gave up: end the graph's loop
    if (blockIdx.x == 0 && threadIdx.x == 0 && c.use_loop)
      cudaGraphSetConditional((cudaGraphConditionalHandle)c.loop_h, 0u);
    return;
  }
  unsigned gen = *(volatile unsigned*)&ctl->bar_gen;  // no iteration ends before every block arrives
  bool first = true;
  for (;;) {
    const bool last = run_body<ALG, VAR, DEFER>(c, sh);
    if (threadIdx.x == 0) {
      if (last && !(first && *(volatile int*)&ctl->hold)) {
        __threadfence();
        atomicAdd(&ctl->bar_gen, 1u);
      } else {
        grid_wait(ctl, gen);
      }
      __threadfence();
      s_go = *(volatile int*)&ctl->go && !(*(volatile int*)&ctl->status & kStatusStall);
    }
    first = false;
    ++gen;
    __syncthreads();
    if (!s_go) break;
  }
}

template <int ALG, int MINB = I2_SEL_MIN_BLOCKS>
__global__ void __launch_bounds__(kBlock, MINB) relax_dispatch(Ctx c) {
  __shared__ AnyShared<> sh;
  switch (c.ctl->variant) {  // same value for every thread of the launch
    case kVPThread: body_push<ALG, kVPThread>(c, sh.st); break;
    case kVPWarp: body_push<ALG, kVPWarp>(c, sh.st); break;
    case kVPCta: body_edge_balanced<ALG>(c, sh.eb); break;
    case kVPBlock: body_push<ALG, kVPBlock>(c, sh.st); break;
    case kPullFrontier: body_pull<ALG, true>(c, sh.st); break;
    case kPullTopo: body_pull<ALG, false>(c, sh.st); break;
    case kEdgeTopo: body_edge_topo<ALG>(c, sh.st); break;
    case kUnionFind:
      if constexpr (ALG == kCC) {
        body_union<ALG>(c, sh.st);
        break;
      }
      [[fallthrough]];  // not allowed for BFS/SSSP
    default: body_push_topo<ALG>(c, sh.st); break;
  }
}

}  // namespace i2
