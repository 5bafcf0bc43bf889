// Shared device-side definitions of the B200 relaxation engine.
//
// The engine computes the same fixed points as the Indigo2 suite's BFS, SSSP and
// CC codes: BFS levels (codes/cuda/bfs-cuda/*, relax `atomicMin(&dist[dst], s+1)`,
// e.g. BFS_CUDA_V_Data_Push_..._Warp_..._NonDup.cu:73-79), SSSP distances with
// int32 weights (SSSP_CUDA_E_Data_Push_..._NonDup.cu:72-73) and CC minimum-ID
// labels (CC_CUDA_E_Data_Push_..._NonDup.cu:68-71). All values are int32 and
// INT_MAX marks an unreached vertex, as in include/bfs_vertex_cuda.h:46.
//
// Frontier contract shared by every variant (so a selector may switch variant
// at any iteration without changing the result):
//   at the start of iteration i, F_i is stored in slot s = i % 3 as
//     wl[s][0..size)     its vertices (those of degree >= 1),
//     woff[s][0..size)   the exclusive prefix sum of their degrees, so that
//                        the frontier's edges form one index space [0, edges),
//     hwl[s][0..hsize)   the subset of degree >= the heavy threshold, with
//     htoff[s][0..hsize) the exclusive prefix of their tile counts,
//     bm[s]              a bitmap with the bits of F_i set (vertices of
//                        degree 0 are never kept: they have nothing to relax);
//   every vertex outside F_i has already relaxed all of its out-edges against
//   the current dist[]. Iteration i propagates at least F_i and builds F_{i+1}
//   in slot (i+1) % 3 from every vertex whose value it lowered. It also clears
//   slot (i+2) % 3 (F_{i-1}), which no variant reads during iteration i.
// SSSP near/far ordering (Ctl::delta != 0) relaxes the contract in one way: a
// lowered vertex whose new distance is at or above the current threshold goes
// onto the far pile instead of F_{i+1}. The traversal ends when both F_{i+1}
// and the pile are empty. Only the edge-balanced push defers; every other
// variant pushes all lowered vertices into F_{i+1}, which is always valid.
#pragma once
#include <cstdint>
#include <climits>
#include <cuda_runtime.h>

namespace i2 {

constexpr int kInf = INT_MAX;
constexpr int kBlock = 256;          // threads per block for all relax kernels
constexpr int kWarp = 32;
constexpr int kQueue = 2048;         // per-block shared staging queue (light)
constexpr int kHQueue = 128;         // per-block shared staging queue (heavy)
constexpr int kHeavyTile = 2048;     // edges per tile of a heavy vertex
constexpr int kMaxVariants = 16;
constexpr int kFeatures = 16;        // selector input width
constexpr int kHidden = 64;          // selector hidden width (two layers)
constexpr int kHistBins = 256;       // distance histogram of the budgeted near/far ordering

enum Algo { kBFS = 0, kSSSP = 1, kCC = 2, kMIS = 3 };

// Maximal independent set: status per vertex, the reference's undecided /
// included / excluded (include/mis_vertex_cuda.h:52-54), and the priority its
// CUDA codes give vertex v (hash(v + 712313887) read as int, e.g.
// MIS_CUDA_V_Data_Pull_Determ_..._Thread.cu:51; the hash is a published
// integer mixing function: two rounds of xor-shift by 16 and multiply by
// 0x45d9f3b, then a final xor-shift). Neighbour u outranks v when its
// priority is larger, or equal with a larger ID (:70).
constexpr int kMisUndecided = 0;
constexpr int kMisIn = 1;
constexpr int kMisOut = 2;

__device__ __forceinline__ int mis_priority(int v) {
  unsigned x = (unsigned)v + 712313887u;
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  return (int)((x >> 16) ^ x);
}

__device__ __forceinline__ bool mis_outranks(int u, int pu, int v, int pv) {
  return pu > pv || (pu == pv && u > v);
}

enum Variant {
  kVPThread = 0,     // vertex push, data-driven, thread per frontier vertex
  kVPWarp = 1,       // vertex push, data-driven, warp per frontier vertex, 128-bit loads
  kVPCta = 2,        // edge-balanced push: block-scan of a frontier chunk, thread per edge
  kVPBlock = 3,      // vertex push, data-driven, block per frontier vertex
  kPullFrontier = 4, // pull from neighbours that are in the frontier bitmap (bottom-up)
  kPullTopo = 5,     // topology-driven pull over all vertices and all neighbours
  kEdgeTopo = 6,     // edge-centric sweep over all CSR entries gated by the bitmap
  kPushTopo = 7,     // topology sweep of the frontier bitmap, thread per vertex
  kUnionFind = 8,    // CC only: union-find over all edges (hook launch, then compress launch)
  kNumVariants = 9
};

// Device view of a CSR graph in the ECLgraph layout (include/ECLgraph.h:44-50).
struct DGraph {
  int nodes;
  int edges;
  const int* __restrict__ nindex;   // nodes + 1
  const int* __restrict__ nlist;    // edges
  const int* __restrict__ eweight;  // edges (SSSP only)
  const int* __restrict__ sp;       // edges: source vertex of each CSR entry (edge sweeps only)
  int vec_ok;                       // 1 when nlist/eweight bases are 16-byte aligned
};

// Whole-graph statistics used by the selector and the pull bound.
struct GStats {
  int nodes;
  int edges;
  int maxdeg;
  int nheavy;       // vertices with degree >= heavy threshold
  int wmin;         // minimum edge weight (1 for BFS)
  int symmetric;    // 1 when every (u,v,w) has a (v,u,w) partner
  float avgdeg;
  float degcv;      // coefficient of variation of the degree distribution
  float wmean;      // mean edge weight (1 for BFS)
};

// Statistics of one frontier buffer, accumulated while it is built. Entries
// and edges share one 64-bit word (entries << 32 | edges) so that a single
// atomicAdd hands out consistent positions in wl[] and offsets in woff[]; a
// frontier holds each vertex at most once, so edges <= E < 2^31 never carries
// into the entry count. The heavy list pairs entries with tiles the same way.
struct Slot {
  unsigned long long packed;  // entries << 32 | edges
  unsigned long long hpacked; // heavy entries << 32 | heavy tiles
  int maxdeg;
  int mindist;                // smallest value pushed into this frontier
};

__host__ __device__ __forceinline__ int slot_size(unsigned long long p) { return (int)(p >> 32); }
__host__ __device__ __forceinline__ unsigned slot_edges(unsigned long long p) { return (unsigned)(p & 0xffffffffu); }

struct Ctl {
  Slot slot[3];
  int iter;                 // index of the next relax launch
  int iter_cap;
  int status;               // error bits, see kStatus*
  int variant;              // variant to run at the next launch
  unsigned done;            // blocks finished in the current launch
  int chunk;                // dynamic work counter of the current launch
  int htile;                // dynamic heavy-tile counter of the current launch
  int pad0;
  unsigned long long tstart;// earliest block start of the current launch (globaltimer ns)
  long long visited;        // vertices reached so far
  int hist[kMaxVariants];   // launches per variant
  int mode;                 // 0 fixed, 1 heuristic, 2 learned, 3 fixed switch (then_at)
  int fixed_variant;
  int allowed;              // bitmask of variants allowed on this graph
  int src;                  // source vertex (BFS/SSSP)
  int nsrc;                 // number of sources (batched runs)
  int algo;
  int sel_n;                // frontier entries at the last selector evaluation
  unsigned sel_e;           // frontier edges at the last selector evaluation
  int sel_iter;             // iteration of the last selector evaluation
  // SSSP near/far ordering (delta != 0 only): relax iterations push values at
  // or above `threshold` onto far pile `pcur` instead of the next frontier;
  // when the next frontier is empty and the pile is not, the next launch is a
  // split (split = 1): the threshold rises and the pile's entries below it
  // move into the next frontier, the others onto the other pile.
  //  * delta > 0 (fixed step): the threshold rises to max(threshold, pmin) + delta.
  //  * delta < 0 (edge budget B = -delta): the threshold is set so that about
  //    B edges lie below it, from distance histograms (weighted by degree)
  //    that the launches keep of the next frontier and of the pile: a move
  //    takes the pile's B-edge quantile, and when a frontier carries more than
  //    2B edges the threshold drops to its B-edge quantile and a trim launch
  //    (split = 3) moves the entries at or above it onto the pile. A pile
  //    entry is live while its bit in fbm is set: a near push of the vertex
  //    clears it.
  int delta;
  int threshold;
  int prev_threshold;       // threshold before the last rise
  int split;                // 0 relax, 1 move from the pile, 3 trim the frontier
  int hshift;               // histogram bin width 2^hshift (budget)
  int hbase;                // frontier histogram base of the current launch (budget)
  int pbase;                // pile histogram base (budget)
  int pad2;
  int pcur;
  unsigned psize[2];
  int pmin[2];              // lower bound of the values on each pile
  int uf_phase;             // union-find CC: 1 after the hook launch (the compress launch follows)
  int then_at;              // mode 3: iteration from which then_variant runs
  int then_variant;
  int uf_giant;             // union-find CC: root of the sampled largest tree
  // Resident launches (one launch runs every iteration, the grid meeting at
  // a barrier between them).
  unsigned bar_gen;         // barrier generation, bumped once per iteration
  int go;                   // 1 while another iteration follows
  int hold;                 // test hook: the first release is withheld
  int pad1;
  unsigned long long stall_ns;  // longest wait at the barrier before giving up
  unsigned long long relax_ns;  // sum of relax launch durations
  float feat[kFeatures];    // features of the frontier the next launch consumes
};

// Union-find CC pays on graphs of 2^19 vertices or more, or of average degree
// below 6 (measured 2.5-23x faster than the best propagation style on RMAT,
// ER and grid graphs of 2^22 vertices and more; propagation up to 1.7x faster
// on RMAT and ER of 2^18 vertices with higher degrees). Both selectors take it
// before the first iteration on symmetric graphs.
__host__ __device__ inline bool union_find_pays(long long nodes, float avgdeg) {
  return nodes >= (1LL << 19) || avgdeg < 6.f;
}

// Graphs on which the selectors' kernel is compiled for the fixed styles'
// resident blocks per SM rather than I2_SEL_MIN_BLOCKS (relax.cuh).
constexpr long long kWideSelectorNodes = 1LL << 25;

enum : int {
  kStatusIterCap = 1,
  kStatusOverflow = 2,
  kStatusStall = 4,  // a resident launch's barrier wait ran out of time
};

// One record per relax launch: the frontier it consumed and its duration.
struct IterRec {
  int iter;
  int variant;
  int size;
  int hsize;
  unsigned long long edges;
  int maxdeg;
  int mindist;
  long long visited;
  unsigned long long t_ns;
  float feat[kFeatures];
  int kind;                 // Ctl::split of the launch: 0 relax, 1 move, 3 trim
  int threshold;            // near/far threshold of the launch (INT_MAX: none)
  unsigned pile;            // far-pile entries after the launch
  int pad;
};

// Everything a relax kernel needs, passed by value.
struct Ctx {
  DGraph g;
  GStats gs;
  int* dist;
  int* wl[3];
  unsigned* woff[3];
  int* hwl[3];
  unsigned* htoff[3];
  int* pile[2];             // far piles (SSSP near/far ordering), vertices
  int* pdeg[2];             // their degrees
  unsigned pile_cap;        // entries per pile
  unsigned* fbm;            // bit set: vertex is on the current far pile
  unsigned long long* hist; // 2 x kHistBins edge counts: [0] next frontier, [1] pile
  unsigned* bm[3];
  Ctl* ctl;
  IterRec* recs;
  int rec_cap;
  int heavy;                // degree threshold of the heavy list
  int bm_words;             // words per bitmap
  const float* mlp;         // selector weights (device), may be null
  const int* srcs;          // batched sources (device), may be null
  unsigned long long loop_h;   // cudaGraphConditionalHandle of the while node
  int use_loop;
};

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Relaxation operators: candidate value for dst from source value du along CSR entry k.
template <int ALG>
struct Op;

template <>
struct Op<kBFS> {
  static __device__ __forceinline__ bool valid(int du) { return du != kInf; }
  static __device__ __forceinline__ int cand(int du, int /*w*/) { return du + 1; }
  static constexpr bool kWeighted = false;
};
template <>
struct Op<kSSSP> {
  static __device__ __forceinline__ bool valid(int du) { return du != kInf; }
  static __device__ __forceinline__ int cand(int du, int w) { return du + w; }
  static constexpr bool kWeighted = true;
};
template <>
struct Op<kCC> {
  static __device__ __forceinline__ bool valid(int) { return true; }
  static __device__ __forceinline__ int cand(int du, int) { return du; }
  static constexpr bool kWeighted = false;
};

}  // namespace i2
