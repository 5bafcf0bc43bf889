// End of an iteration, shared by every relax kernel (one launch per iteration
// or resident): the last block of the iteration records it, rotates the
// frontier slots and picks the style of the next iteration. Included by each
// translation unit that instantiates relax kernels.
#pragma once
#include "common.cuh"
#include "mlp.cuh"

namespace i2 {

// ---------------------------------------------------------------------------
// Selection of the next variant.

// Fixed frontier-size rule: union-find for CC on symmetric graphs (measured
// 2.5-23x faster than the best propagation style on RMAT, ER and grid graphs
// of 2^22 vertices and more, within 2x either way on 2^18), bottom-up pull for BFS levels whose frontier
// carries more than 1/16 of the edges (direction-optimising BFS), otherwise the
// edge-balanced push, which measured fastest of the push styles on every
// family tried.
// Union-find replaces the whole traversal, so it is a choice made once, before
// the first iteration, by both selectors; the per-iteration picks are among the
// propagation styles. On graphs below 2^19 vertices with an average degree of
// 6 or more (RMAT and ER of 2^18 vertices) propagation measured up to 1.7x
// faster than union-find; on grids and on every graph of 2^20 vertices and
// more, union-find was the fastest.
static __device__ bool union_find_first(const GStats& gs, int algo, int allowed, int next_iter) {
  return algo == kCC && next_iter == 0 && ((allowed >> kUnionFind) & 1) && union_find_pays(gs.nodes, gs.avgdeg);
}

// The learned selector overrides the rule only where it predicts the rule's
// style at least 2^kLearnedMargin (about 11%) slower than its own pick: the
// rule is its fallback, and small mispredictions between close styles do not
// cost time.
constexpr float kLearnedMargin = 0.15f;

static __device__ int heuristic_pick(const GStats& gs, int algo, int allowed, int size, unsigned long long edges) {
  (void)size;
  const float fe = (float)edges;
  const float E = (float)gs.edges;
  auto ok = [&](int v) { return (allowed >> v) & 1; };
  if (algo == kBFS && ok(kPullFrontier) && fe > E * (1.f / 16.f)) return kPullFrontier;
  return ok(kVPCta) ? kVPCta : kVPThread;
}

// Executed by every thread of one block. Computes the features of the frontier
// in slot `nxt`, picks the variant for the next launch and sets the loop
// condition of the graph. `cond` tells whether another launch will happen;
// `force` >= 0 overrides the pick (the compress launch of union-find CC).
// The learned selector is re-evaluated when the frontier's entries or edges
// moved by more than a factor 1.5 since its last evaluation, or 16 iterations
// passed; otherwise the previous choice stands (long tails of small, similar
// frontiers do not pay for an inference each). On graphs with more vertices
// than any it was trained on it defers to the frequency rule (no inference):
// measured on RMAT-24 and RMAT-26 BFS, its picks there cost 1.08-1.38x the
// rule's time even with the size features clamped to the training range.
static __device__ void select_next(const Ctx& c, int next_iter, int nxt, bool cond, int force) {
  __shared__ float x[kFeatures], h1[kHidden], h2[kHidden], y[kOut];
  __shared__ int s_eval;
  Ctl* ctl = c.ctl;
  if (threadIdx.x == 0) {
    volatile Slot* sl = &ctl->slot[nxt];
    const unsigned long long p = sl->packed;
    const int n = slot_size(p);
    const unsigned e = slot_edges(p);
    frontier_features(c.gs, ctl->algo, next_iter, n, slot_size(sl->hpacked), e, sl->maxdeg,
                      *(volatile long long*)&ctl->visited, x);
    for (int k = 0; k < kFeatures; ++k) ctl->feat[k] = x[k];
    const long long sn = ctl->sel_n, se = ctl->sel_e;
    s_eval = next_iter == 0 || 2LL * n > 3LL * sn || 3LL * n < 2LL * sn || 2LL * e > 3LL * se ||
             3LL * e < 2LL * se || next_iter - ctl->sel_iter >= 16;
  }
  __syncthreads();
  const int mode = ctl->mode;
  const bool learned = c.mlp && c.gs.nodes <= kMaxTrainedNodes;
  const bool infer = mode == 2 && learned && cond && s_eval && force < 0;
  if (infer) mlp_forward_block(c.mlp, x, h1, h2, y);
  if (threadIdx.x == 0) {
    int v = ctl->fixed_variant;
    if (mode == 3) {
      v = next_iter >= ctl->then_at ? ctl->then_variant : ctl->fixed_variant;
    } else if ((mode == 1 || mode == 2) && union_find_first(c.gs, ctl->algo, ctl->allowed, next_iter)) {
      v = kUnionFind;
    } else if (mode == 1 || (mode == 2 && !learned)) {
      volatile Slot* sl = &ctl->slot[nxt];
      const unsigned long long p = sl->packed;
      v = heuristic_pick(c.gs, ctl->algo, ctl->allowed, slot_size(p), slot_edges(p));
    } else if (mode == 2) {
      v = ctl->variant;
      if (infer) {
        volatile Slot* sl = &ctl->slot[nxt];
        const unsigned long long p = sl->packed;
        const int h = heuristic_pick(c.gs, ctl->algo, ctl->allowed, slot_size(p), slot_edges(p));
        float best = 3.0e38f;
        int bv = -1;
        for (int k = 0; k < kOut; ++k)  // per-iteration styles only (see union_find_first)
          if (k != kUnionFind && ((ctl->allowed >> k) & 1) && y[k] < best) {
            best = y[k];
            bv = k;
          }
        v = (bv >= 0 && best + kLearnedMargin < y[h]) ? bv : h;
        ctl->sel_n = slot_size(p);
        ctl->sel_e = slot_edges(p);
        ctl->sel_iter = next_iter;
      }
    }
    if (force >= 0) v = force;
    ctl->variant = v;
    if (cond) ctl->hist[v] += 1;
    ctl->go = cond ? 1 : 0;
    if (c.use_loop) cudaGraphSetConditional((cudaGraphConditionalHandle)c.loop_h, cond ? 1u : 0u);
  }
}

// Edge budget of the SSSP near/far ordering (whole block; kBlock bins): the
// first bin at which each histogram's running edge count reaches the budget
// (kHistBins if it never does): [0] the next frontier's, [1] the pile's. The
// next frontier's histogram is then cleared for the next launch's pushes.
static_assert(kHistBins == kBlock, "one histogram bin per thread");
static __device__ void budget_quantiles(const Ctx& c, int* q) {
  __shared__ unsigned long long part[kBlock / kWarp];
  __shared__ int sq[2];
  const unsigned long long B = (unsigned long long)(-(long long)c.ctl->delta);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int which = 0; which < 2; ++which) {
    unsigned long long* h = c.hist + which * kHistBins;
    const unsigned long long x = *(volatile unsigned long long*)&h[threadIdx.x];
    unsigned long long incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) part[wid] = incl;
    if (threadIdx.x == 0) sq[which] = kHistBins;
    __syncthreads();
    for (int w = 0; w < wid; ++w) incl += part[w];
    if (incl >= B && incl - x < B) sq[which] = threadIdx.x;
    __syncthreads();
  }
  q[0] = sq[0];
  q[1] = sq[1];
  c.hist[threadIdx.x] = 0ull;
}

// Thread 0 of the last block, edge budget: the next launch of the ordering.
// `q` are the histogram quantiles, `n`/`e` the next frontier's entries and
// edges. Returns whether another launch follows; *clear_pile is set when the
// pile histogram must be cleared (a move rebuilds it from the entries it keeps).
static __device__ int budget_next(const Ctx& c, const int* q, long long n, unsigned e, int nxt, int* clear_pile) {
  Ctl* ctl = c.ctl;
  const long long B = -(long long)ctl->delta;
  const int shift = ctl->hshift;
  const int was = ctl->split;
  const int p = ctl->pcur;
  int cond = n > 0;
  *clear_pile = 0;
  if (was == 1) {  // the move emptied pile p onto the other one
    ctl->psize[p] = 0;
    ctl->pmin[p] = kInf;
    ctl->pcur = 1 - p;
  }
  ctl->split = 0;
  const int np = ctl->pcur;
  // move next when the frontier is empty, or so small that its last
  // iterations would cost more launches than edges (it is carried along)
  if (*(volatile unsigned*)&ctl->psize[np] > 0 && (n == 0 || (was == 0 && (long long)e * 16 < B))) {
    // at the budget's quantile of the pile (and above the pile's lower bound,
    // so that a live entry moves, or the move learns the bound)
    const int pm = *(volatile int*)&ctl->pmin[np];
    long long T = q[1] < kHistBins ? (long long)ctl->pbase + ((long long)(q[1] + 1) << shift) : (long long)kInf;
    if (pm != kInf) T = max(T, (long long)pm + 1);
    T = min(T, (long long)kInf);
    ctl->prev_threshold = ctl->threshold;
    ctl->threshold = (int)T;
    int lo = pm != kInf ? pm : ctl->pbase;  // the smallest value the move can carry
    if (n > 0) lo = min(lo, *(volatile int*)&ctl->slot[nxt].mindist);
    ctl->hbase = lo;
    ctl->pbase = (int)T;                       // kept values are at or above T
    ctl->split = 1;
    *clear_pile = 1;
    return 1;
  }
  if (n > 0 && was != 3 && (long long)e > 2 * B && q[0] < kHistBins) {
    const long long T = (long long)ctl->hbase + ((long long)(q[0] + 1) << shift);
    if (T < (long long)ctl->threshold) {  // trim the next frontier to about B edges
      ctl->threshold = (int)T;
      ctl->split = 3;
    }
  }
  ctl->hbase = *(volatile int*)&ctl->slot[nxt].mindist;
  return cond;
}

// Last block of a relax launch: record the launch, advance the iteration and
// decide whether the loop continues.
static __device__ void finish_iteration(const Ctx& c, int i, int cur, int nxt, int old) {
  __shared__ int s_cond, s_force, s_clear;
  __shared__ int s_q[2];
  Ctl* ctl = c.ctl;
  if (ctl->variant == kUnionFind && ctl->uf_phase == 0) uf_sample_giant(c);  // whole block
  if (threadIdx.x == 0) s_clear = 0;
  if (ctl->delta < 0) {
    int q[2];
    budget_quantiles(c, q);
    if (threadIdx.x == 0) {
      s_q[0] = q[0];
      s_q[1] = q[1];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const unsigned long long t1 = globaltimer();
    const unsigned long long dt = t1 - ctl->tstart;
    ctl->relax_ns += dt;
    volatile Slot* sc = &ctl->slot[cur];
    if (c.recs && i < c.rec_cap) {
      IterRec& r = c.recs[i];
      r.iter = i;
      r.variant = ctl->variant;
      r.size = slot_size(sc->packed);
      r.hsize = slot_size(sc->hpacked);
      r.edges = slot_edges(sc->packed);
      r.maxdeg = sc->maxdeg;
      r.mindist = sc->mindist;
      r.visited = *(volatile long long*)&ctl->visited;
      r.t_ns = dt;
      for (int k = 0; k < kFeatures; ++k) r.feat[k] = ctl->feat[k];
      r.kind = ctl->split;
      r.threshold = ctl->threshold;
      r.pile = ctl->delta != 0 ? *(volatile unsigned*)&ctl->psize[ctl->split == 1 ? 1 - ctl->pcur : ctl->pcur] : 0u;
    }
    Slot& so = ctl->slot[old];
    so.packed = 0;
    so.hpacked = 0;
    so.maxdeg = 0;
    so.mindist = kInf;
    ctl->done = 0;
    ctl->chunk = 0;
    ctl->htile = 0;
    ctl->tstart = ~0ull;
    ctl->iter = i + 1;
    volatile Slot* sn = &ctl->slot[nxt];
    const long long n = slot_size(sn->packed);
    int cond = n > 0;
    if (ctl->delta < 0) {
      cond = budget_next(c, s_q, n, slot_edges(sn->packed), nxt, &s_clear);
    } else if (ctl->delta > 0) {
      if (ctl->split) {  // this launch emptied pile pcur onto the other one
        const int p = ctl->pcur;
        ctl->psize[p] = 0;
        ctl->pmin[p] = kInf;
        ctl->pcur = 1 - p;
        ctl->split = 0;
      }
      const int p = ctl->pcur;
      if (n == 0 && *(volatile unsigned*)&ctl->psize[p] > 0) {
        // next launch splits the pile at a raised threshold
        const long long lo = max((long long)ctl->threshold, (long long)*(volatile int*)&ctl->pmin[p]);
        ctl->prev_threshold = ctl->threshold;
        ctl->threshold = (int)min(lo + (long long)ctl->delta, (long long)kInf);
        ctl->split = 1;
        cond = 1;
      }
    }
    int force = -1;
    if (ctl->variant == kUnionFind) {
      if (ctl->uf_phase < 2) {  // the next union-find launch follows
        ctl->uf_phase += 1;
        force = kUnionFind;
        cond = 1;
      } else {
        ctl->uf_phase = 0;  // labels final; nothing was pushed
      }
    }
    if (cond && i + 1 >= ctl->iter_cap) {
      ctl->status |= kStatusIterCap;
      cond = 0;
    }
    s_cond = cond;
    s_force = force;
  }
  __syncthreads();
  if (s_clear) c.hist[kHistBins + threadIdx.x] = 0ull;  // read above; the move rebuilds it
  select_next(c, i + 1, nxt, s_cond != 0, s_force);
}

}  // namespace i2
