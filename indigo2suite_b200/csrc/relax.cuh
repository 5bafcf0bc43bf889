// Relaxation kernels of the B200 engine: one persistent, grid-stride kernel per
// (algorithm, variant). Each launch performs exactly one iteration of the
// frontier contract described in common.cuh.
//
// Reference styles these variants re-create (file names under codes/cuda/):
//   kVPThread  ~ *_V_Data_Push_*_Thread_*   (e.g. BFS ..._Atomic_Thread_..._NonDup.cu)
//   kVPWarp    ~ *_V_Data_Push_*_Warp_*     (BFS_CUDA_V_Data_Push_..._Warp_..._NonDup.cu:62-84)
//   kVPBlock   ~ *_V_Data_Push_*_Block_*    (BFS_CUDA_V_Data_Push_..._Block_..._Dup.cu:62-83)
//   kVPCta     ~ *_E_Data_Push_*            (SSSP_CUDA_E_Data_Push_..._NonDup.cu:63-82): one thread per edge
//   kPullFrontier / kPullTopo ~ *_V_{Data,Topo}_Pull_* (BFS ..._V_Topo_Pull_..._Warp_...cu:57-79,
//                                           CC_CUDA_V_Topo_Pull_..._Warp_...cu:59-78)
//   kEdgeTopo  ~ *_E_Topo_Push_*            (BFS_CUDA_E_Topo_Push_..._Thread_...cu:57-72)
//   kPushTopo  ~ *_V_Topo_Push_*            (BFS_CUDA_V_Topo_Push_..._Thread_...cu:56-79)
// The B200 versions differ in mechanism, not in fixed point: frontier appends are
// staged per block in shared memory and published with one global atomic per
// round, duplicate pushes are filtered by a frontier bitmap (the reference uses
// a `time[]` stamp array), adjacency is read with 128-bit loads, and vertices of
// degree >= the heavy threshold are split into tiles shared by the whole grid.
#pragma once
#include <cooperative_groups.h>
#include <cub/block/block_scan.cuh>
#include "common.cuh"

namespace i2 {

namespace cg = cooperative_groups;

// Per-block staging of pushes into the next frontier.
struct Stage {
  int q[kQueue];
  int hq[kHQueue];
  int n;
  int hn;
  int base;
  int hbase;
  unsigned long long edges;
  int maxdeg;
  int mindist;
  int visited;
  int chunk;
  int last;
};

__device__ __forceinline__ void stage_init(Stage& s) {
  if (threadIdx.x == 0) {
    s.n = 0;
    s.hn = 0;
    s.edges = 0;
    s.maxdeg = 0;
    s.mindist = kInf;
    s.visited = 0;
    s.last = 0;
  }
}

// Append a vertex to the next frontier, bypassing the staging queue. Used only
// when a round produces more pushes than the shared queue holds.
__device__ __forceinline__ void direct_append(int* counter, int* list, int v) {
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(counter, (int)g.size());
  base = g.shfl(base, 0);
  list[base + g.thread_rank()] = v;
}

// Record vertex v in the next frontier. The bitmap bit has already been
// claimed by the caller, and the frontier minimum has already been updated.
__device__ __forceinline__ void stage_vertex(const Ctx& c, Stage& s, int nxt, int v) {
  const int beg = c.g.nindex[v];
  const int deg = c.g.nindex[v + 1] - beg;
  atomicAdd(&s.edges, (unsigned long long)deg);
  atomicMax(&s.maxdeg, deg);
  if (deg >= c.heavy) {
    const int p = atomicAdd(&s.hn, 1);
    if (p < kHQueue) s.hq[p] = v;
    else direct_append(&c.ctl->slot[nxt].hsize, c.hwl[nxt], v);
  } else {
    const int p = atomicAdd(&s.n, 1);
    if (p < kQueue) s.q[p] = v;
    else direct_append(&c.ctl->slot[nxt].size, c.wl[nxt], v);
  }
}

// Push after a successful atomicMin (old > val). The frontier minimum is
// lowered on every improvement, including repeat improvements of a vertex that
// is already in the next frontier, so it is a true lower bound of the values
// the next iteration reads.
__device__ __forceinline__ void push_vertex(const Ctx& c, Stage& s, int nxt, int v, int val, int old) {
  if (old == kInf) atomicAdd(&s.visited, 1);
  atomicMin(&s.mindist, val);
  const unsigned bit = 1u << (v & 31);
  if (atomicOr(&c.bm[nxt][v >> 5], bit) & bit) return;
  stage_vertex(c, s, nxt, v);
}

// Publish the staged pushes of this block (block-uniform call).
__device__ __forceinline__ void stage_flush(const Ctx& c, Stage& s, int nxt) {
  __syncthreads();
  const int n = min(s.n, kQueue);
  const int hn = min(s.hn, kHQueue);
  __syncthreads();  // every thread has read the counters before anyone changes them
  if (n == 0 && hn == 0) return;
  if (threadIdx.x == 0) {
    if (n) s.base = atomicAdd(&c.ctl->slot[nxt].size, n);
    if (hn) s.hbase = atomicAdd(&c.ctl->slot[nxt].hsize, hn);
    s.n = 0;
    s.hn = 0;
  }
  __syncthreads();
  int* wl = c.wl[nxt];
  for (int j = threadIdx.x; j < n; j += blockDim.x) wl[s.base + j] = s.q[j];
  int* hwl = c.hwl[nxt];
  for (int j = threadIdx.x; j < hn; j += blockDim.x) hwl[s.hbase + j] = s.hq[j];
  __syncthreads();
}

template <int ALG>
__device__ __forceinline__ void relax_edge(const Ctx& c, Stage& s, int nxt, int du, int v, int w) {
  const int cand = Op<ALG>::cand(du, w);
  if (cand < c.dist[v]) {
    const int old = atomicMin(&c.dist[v], cand);
    if (cand < old) push_vertex(c, s, nxt, v, cand, old);
  }
}

// Relax CSR entries [lo, hi) of one source with value du. The calling group has
// gsize threads and this thread is `lane` in it. Aligned 16-byte units of nlist
// (and eweight) are read with one 128-bit load; a unit that would reach past
// the end of the arrays is read element by element.
template <int ALG>
__device__ __forceinline__ void relax_range(const Ctx& c, Stage& s, int nxt, int du, int lo, int hi,
                                            int lane, int gsize) {
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  if (c.g.vec_ok && hi - lo >= 8) {
    const int q0 = lo >> 2;
    const int q1 = (hi + 3) >> 2;
    for (int q = q0 + lane; q < q1; q += gsize) {
      const int k0 = q << 2;
      int nv[4], wv[4] = {0, 0, 0, 0};
      if (k0 + 3 < c.g.edges) {
        const int4 a = __ldg(reinterpret_cast<const int4*>(nl + k0));
        nv[0] = a.x; nv[1] = a.y; nv[2] = a.z; nv[3] = a.w;
        if (Op<ALG>::kWeighted) {
          const int4 b = __ldg(reinterpret_cast<const int4*>(ew + k0));
          wv[0] = b.x; wv[1] = b.y; wv[2] = b.z; wv[3] = b.w;
        }
      } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const int k = k0 + t;
          nv[t] = (k >= lo && k < hi) ? nl[k] : 0;
          if (Op<ALG>::kWeighted) wv[t] = (k >= lo && k < hi) ? ew[k] : 0;
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int k = k0 + t;
        if (k >= lo && k < hi) relax_edge<ALG>(c, s, nxt, du, nv[t], wv[t]);
      }
    }
  } else {
    for (int k = lo + lane; k < hi; k += gsize) {
      const int w = Op<ALG>::kWeighted ? __ldg(ew + k) : 0;
      relax_edge<ALG>(c, s, nxt, du, __ldg(nl + k), w);
    }
  }
}

// Heavy frontier vertices: their adjacency is cut into tiles of kHeavyTile
// entries, and tile t of the concatenated tile sequence goes to block t % grid.
template <int ALG>
__device__ void heavy_path(const Ctx& c, Stage& s, int cur, int nxt) {
  const int nh = c.ctl->slot[cur].hsize;
  const int G = gridDim.x;
  long long tbase = 0;
  for (int j = 0; j < nh; ++j) {
    const int u = c.hwl[cur][j];
    const int du = c.dist[u];
    const int beg = c.g.nindex[u];
    const int end = c.g.nindex[u + 1];
    const int ntiles = (end - beg + kHeavyTile - 1) / kHeavyTile;
    if (Op<ALG>::valid(du)) {
      int t = (int)(((long long)blockIdx.x - (tbase % G) + G) % G);
      for (; t < ntiles; t += G) {
        const int lo = beg + t * kHeavyTile;
        const int hi = min(end, lo + kHeavyTile);
        relax_range<ALG>(c, s, nxt, du, lo, hi, threadIdx.x, blockDim.x);
        stage_flush(c, s, nxt);
      }
    }
    tbase += ntiles;
  }
}

// Clear the bitmap of F_{i-1} (slot old): by entries when it is small, by words otherwise.
__device__ __forceinline__ void clear_old(const Ctx& c, int old) {
  const int n = c.ctl->slot[old].size;
  const int hn = c.ctl->slot[old].hsize;
  unsigned* bm = c.bm[old];
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  if ((long long)(n + hn) * 4 > c.bm_words) {
    for (long long w = tid; w < c.bm_words; w += stride) bm[w] = 0u;
  } else {
    const int* wl = c.wl[old];
    for (long long j = tid; j < n; j += stride) bm[wl[j] >> 5] = 0u;
    const int* hwl = c.hwl[old];
    for (long long j = tid; j < hn; j += stride) bm[hwl[j] >> 5] = 0u;
  }
}

__device__ void finish_iteration(const Ctx& c, int i, int cur, int nxt, int old);

// Common epilogue: publish block statistics and let the last block finish the iteration.
__device__ __forceinline__ void block_epilogue(const Ctx& c, Stage& s, int i, int cur, int nxt, int old) {
  __syncthreads();
  if (threadIdx.x == 0) {
    Slot& sl = c.ctl->slot[nxt];
    if (s.edges) atomicAdd(&sl.edges, s.edges);
    if (s.maxdeg) atomicMax(&sl.maxdeg, s.maxdeg);
    if (s.mindist != kInf) atomicMin(&sl.mindist, s.mindist);
    if (s.visited) atomicAdd((unsigned long long*)&c.ctl->visited, (unsigned long long)s.visited);
    __threadfence();
    const unsigned t = atomicAdd(&c.ctl->done, 1u);
    s.last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (s.last) {
    __threadfence();
    finish_iteration(c, i, cur, nxt, old);
  }
}

__device__ __forceinline__ void block_prologue(const Ctx& c) {
  if (threadIdx.x == 0) atomicMin(&c.ctl->tstart, globaltimer());
}

// ---------------------------------------------------------------------------
// Data-driven push variants.

template <int ALG, int VAR>
__global__ void __launch_bounds__(kBlock) relax_push(Ctx c) {
  __shared__ Stage s;
  typedef cub::BlockScan<int, kBlock> Scan;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ int s_beg[kBlock];
  __shared__ int s_off[kBlock + 1];
  __shared__ int s_du[kBlock];

  block_prologue(c);
  stage_init(s);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  clear_old(c, old);
  __syncthreads();

  const int n = c.ctl->slot[cur].size;
  const int* __restrict__ wl = c.wl[cur];
  const int per = (VAR == kVPThread || VAR == kVPCta) ? kBlock : (VAR == kVPWarp ? kBlock / kWarp : 1);

  while (true) {
    if (threadIdx.x == 0) s.chunk = atomicAdd(&c.ctl->chunk, per);
    __syncthreads();
    const int base = s.chunk;
    if (base >= n) break;  // uniform
    if (VAR == kVPThread) {
      const int idx = base + threadIdx.x;
      if (idx < n) {
        const int u = wl[idx];
        const int du = c.dist[u];
        if (Op<ALG>::valid(du)) relax_range<ALG>(c, s, nxt, du, c.g.nindex[u], c.g.nindex[u + 1], 0, 1);
      }
    } else if (VAR == kVPWarp) {
      const int idx = base + threadIdx.x / kWarp;
      if (idx < n) {
        const int u = wl[idx];
        const int du = c.dist[u];
        if (Op<ALG>::valid(du))
          relax_range<ALG>(c, s, nxt, du, c.g.nindex[u], c.g.nindex[u + 1], threadIdx.x % kWarp, kWarp);
      }
    } else if (VAR == kVPBlock) {
      const int u = wl[base];
      const int du = c.dist[u];
      if (Op<ALG>::valid(du))
        relax_range<ALG>(c, s, nxt, du, c.g.nindex[u], c.g.nindex[u + 1], threadIdx.x, blockDim.x);
    } else {  // kVPCta: scan the degrees of a chunk, then one thread per edge
      const int idx = base + threadIdx.x;
      int deg = 0, beg = 0, du = kInf;
      if (idx < n) {
        const int u = wl[idx];
        du = c.dist[u];
        beg = c.g.nindex[u];
        deg = Op<ALG>::valid(du) ? c.g.nindex[u + 1] - beg : 0;
      }
      int off, total;
      Scan(scan_tmp).ExclusiveSum(deg, off, total);
      s_beg[threadIdx.x] = beg;
      s_off[threadIdx.x] = off;
      s_du[threadIdx.x] = du;
      if (threadIdx.x == 0) s_off[kBlock] = total;
      __syncthreads();
      const int* __restrict__ nl = c.g.nlist;
      const int* __restrict__ ew = c.g.eweight;
      for (int k = threadIdx.x; k < total; k += kBlock) {
        int lo = 0, hi = kBlock;  // find j with s_off[j] <= k < s_off[j+1]
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (s_off[mid] <= k) lo = mid; else hi = mid;
        }
        const int e = s_beg[lo] + (k - s_off[lo]);
        const int w = Op<ALG>::kWeighted ? __ldg(ew + e) : 0;
        relax_edge<ALG>(c, s, nxt, s_du[lo], __ldg(nl + e), w);
      }
    }
    stage_flush(c, s, nxt);
  }
  heavy_path<ALG>(c, s, cur, nxt);
  stage_flush(c, s, nxt);
  block_epilogue(c, s, i, cur, nxt, old);
}

// ---------------------------------------------------------------------------
// Bitmap-gated topology sweep: thread per vertex, light vertices only; heavy
// frontier vertices take the shared heavy path.
template <int ALG>
__global__ void __launch_bounds__(kBlock) relax_push_topo(Ctx c) {
  __shared__ Stage s;
  block_prologue(c);
  stage_init(s);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  clear_old(c, old);
  __syncthreads();
  const unsigned* __restrict__ bmc = c.bm[cur];
  const int V = c.g.nodes;
  for (long long base = (long long)blockIdx.x * kBlock; base < V; base += (long long)gridDim.x * kBlock) {
    const int v = (int)base + threadIdx.x;
    if (v < V && ((bmc[v >> 5] >> (v & 31)) & 1u)) {
      const int beg = c.g.nindex[v];
      const int end = c.g.nindex[v + 1];
      const int du = c.dist[v];
      if (end - beg < c.heavy && Op<ALG>::valid(du)) relax_range<ALG>(c, s, nxt, du, beg, end, 0, 1);
    }
    stage_flush(c, s, nxt);
  }
  heavy_path<ALG>(c, s, cur, nxt);
  stage_flush(c, s, nxt);
  block_epilogue(c, s, i, cur, nxt, old);
}

// ---------------------------------------------------------------------------
// Edge-centric sweep over all CSR entries, gated by the source's frontier bit.
template <int ALG>
__global__ void __launch_bounds__(kBlock) relax_edge_topo(Ctx c) {
  __shared__ Stage s;
  block_prologue(c);
  stage_init(s);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  clear_old(c, old);
  __syncthreads();
  const unsigned* __restrict__ bmc = c.bm[cur];
  const int E = c.g.edges;
  const long long units = ((long long)E + 3) >> 2;
  const int* __restrict__ sp = c.g.sp;
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  for (long long base = (long long)blockIdx.x * kBlock; base < units; base += (long long)gridDim.x * kBlock) {
    const long long q = base + threadIdx.x;
    if (q < units) {
      const long long k0 = q << 2;
      int su[4], nv[4], wv[4] = {0, 0, 0, 0};
      if (c.g.vec_ok && k0 + 3 < E) {
        const int4 a = __ldg(reinterpret_cast<const int4*>(sp + k0));
        su[0] = a.x; su[1] = a.y; su[2] = a.z; su[3] = a.w;
        const int4 b = __ldg(reinterpret_cast<const int4*>(nl + k0));
        nv[0] = b.x; nv[1] = b.y; nv[2] = b.z; nv[3] = b.w;
        if (Op<ALG>::kWeighted) {
          const int4 d = __ldg(reinterpret_cast<const int4*>(ew + k0));
          wv[0] = d.x; wv[1] = d.y; wv[2] = d.z; wv[3] = d.w;
        }
      } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          const long long k = k0 + t;
          su[t] = (k < E) ? sp[k] : -1;
          nv[t] = (k < E) ? nl[k] : 0;
          if (Op<ALG>::kWeighted) wv[t] = (k < E) ? ew[k] : 0;
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int u = su[t];
        if (u >= 0 && ((bmc[u >> 5] >> (u & 31)) & 1u)) {
          const int du = c.dist[u];
          if (Op<ALG>::valid(du)) relax_edge<ALG>(c, s, nxt, du, nv[t], wv[t]);
        }
      }
    }
    stage_flush(c, s, nxt);
  }
  stage_flush(c, s, nxt);
  block_epilogue(c, s, i, cur, nxt, old);
}

// ---------------------------------------------------------------------------
// Pull variants (symmetric graphs only). Thread per destination vertex; a warp
// covers 32 consecutive vertices, i.e. exactly one bitmap word, so the next
// frontier's bitmap is written with one plain store per warp. dist[v] is only
// written by v's own thread, so no atomics are needed on it.
template <int ALG, bool FRONTIER>
__global__ void __launch_bounds__(kBlock) relax_pull(Ctx c) {
  __shared__ Stage s;
  block_prologue(c);
  stage_init(s);
  const int i = c.ctl->iter;
  const int cur = i % 3, nxt = (i + 1) % 3, old = (i + 2) % 3;
  clear_old(c, old);
  __syncthreads();
  const unsigned* __restrict__ bmc = c.bm[cur];
  const int V = c.g.nodes;
  const int* __restrict__ nl = c.g.nlist;
  const int* __restrict__ ew = c.g.eweight;
  const int fmin = c.ctl->slot[cur].mindist;
  // Smallest candidate any frontier vertex can produce.
  const int bound = FRONTIER ? (fmin == kInf ? kInf : Op<ALG>::cand(fmin, c.gs.wmin)) : INT_MIN;
  for (long long base = (long long)blockIdx.x * kBlock; base < V; base += (long long)gridDim.x * kBlock) {
    const int v = (int)base + threadIdx.x;
    bool improved = false;
    int best = kInf, dv = kInf;
    if (v < V) {
      dv = c.dist[v];
      best = dv;
      if (!FRONTIER || dv > bound) {
        const int beg = c.g.nindex[v];
        const int end = c.g.nindex[v + 1];
        for (int k = beg; k < end; ++k) {
          const int u = __ldg(nl + k);
          if (FRONTIER && !((bmc[u >> 5] >> (u & 31)) & 1u)) continue;
          const int du = c.dist[u];
          if (!Op<ALG>::valid(du)) continue;
          const int cd = Op<ALG>::cand(du, Op<ALG>::kWeighted ? __ldg(ew + k) : 0);
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
      if (dv == kInf) atomicAdd(&s.visited, 1);
      atomicMin(&s.mindist, best);
      stage_vertex(c, s, nxt, v);
    }
    stage_flush(c, s, nxt);
  }
  stage_flush(c, s, nxt);
  block_epilogue(c, s, i, cur, nxt, old);
}

}  // namespace i2
