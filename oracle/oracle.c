/*
 * ORACLE — test infrastructure only. Nothing in the product links or calls
 * this file; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * it as the checker.
 *
 * CPU restatement of the Indigo2 reference's serial checkers for BFS, SSSP and
 * CC (paths inside the Indigo2Suite project):
 *   oracle_bfs          include/bfs_vertex_cuda.h:75-99   (CPUserialDijkstra, unit weights)
 *   oracle_sssp         include/sssp_vertex_cuda.h:74-99, include/sssp_edge_cuda.h:74-99
 *                       (CPUserialDijkstra with eweight)
 *   oracle_cc_check     include/cc_vertex_cuda.h:142-170  (adjacent labels equal, labels
 *                       below nodes, one label per component) with an explicit stack
 *                       instead of the reference's recursion (:71-80), which overflows the
 *                       call stack on large components
 *   oracle_cc_minlabel  the minimum-ID labelling that every reference CC variant
 *                       converges to (label[v] = v, then atomicMin(label[dst], label[src]),
 *                       e.g. CC_CUDA_E_Data_Push_..._NonDup.cu:53,71)
 *   oracle_mis          the maximal independent set every deterministic reference MIS
 *                       variant converges to: priority(v) = hash(v + 712313887) read as
 *                       int (include/mis_vertex_cuda.h:170-176, e.g.
 *                       MIS_CUDA_V_Data_Pull_Determ_..._Thread.cu:51), neighbour u ranks
 *                       above v when its priority is larger or equal with a larger ID
 *                       (:70); v is in the set iff no higher-ranked neighbour is: the
 *                       greedy set in decreasing rank, computed here in that order.
 *                       Status 1 = in the set, 2 = excluded (:52-54). The CUDA variants
 *                       compare priorities as int (their data_type); the reference's C++
 *                       and OpenMP MIS variants as unsigned int (codes/cpp/mis-cpp/*.cpp:38),
 *                       which gives another set: `unsigned_priority` selects that order.
 *   oracle_synth_weights include/sssp_vertex_cuda.h:127-137
 *   oracle_sp           include/bfs_edge_cuda.h:140-146
 * Distances use int32 arithmetic with two's-complement wrap, like the reference's
 * `dv + eweight[i]`; unreachable vertices keep INT_MAX.
 *
 * Parity pin: tests/test_oracle.py checks these functions against the reference's
 * own serial checkers compiled unchanged from the reference sources
 * (oracle/Makefile, oracle/_ref/) and against the committed golden vectors.
 */
#include <limits.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int d;
  int v;
} hnode;

typedef struct {
  hnode* a;
  long long n, cap;
} heap;

static int heap_push(heap* h, int d, int v) {
  if (h->n == h->cap) {
    long long nc = h->cap ? 2 * h->cap : 1024;
    hnode* na = (hnode*)realloc(h->a, (size_t)nc * sizeof(hnode));
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  long long i = h->n++;
  while (i > 0) {
    long long p = (i - 1) / 2;
    if (h->a[p].d <= d) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i].d = d;
  h->a[i].v = v;
  return 0;
}

static hnode heap_pop(heap* h) {
  hnode top = h->a[0];
  hnode last = h->a[--h->n];
  long long i = 0;
  for (;;) {
    long long c = 2 * i + 1;
    if (c >= h->n) break;
    if (c + 1 < h->n && h->a[c + 1].d < h->a[c].d) c++;
    if (last.d <= h->a[c].d) break;
    h->a[i] = h->a[c];
    i = c;
  }
  if (h->n > 0) h->a[i] = last;
  return top;
}

/* Dijkstra from src; w == NULL means unit weights. Returns 0, or -1 on OOM. */
static int dijkstra(int nodes, const int* nindex, const int* nlist, const int* w, int src, int* dist) {
  heap h = {0, 0, 0};
  for (int i = 0; i < nodes; i++) dist[i] = INT_MAX;
  dist[src] = 0;
  if (heap_push(&h, 0, src)) return -1;
  while (h.n > 0) {
    hnode t = heap_pop(&h);
    const int v = t.v;
    if (t.d > dist[v]) continue; /* stale entry: v was settled with a smaller value */
    const int dv = dist[v];
    for (int i = nindex[v]; i < nindex[v + 1]; i++) {
      const int n = nlist[i];
      const int d = (int)((unsigned)dv + (unsigned)(w ? w[i] : 1));
      if (d < dist[n]) {
        dist[n] = d;
        if (heap_push(&h, d, n)) {
          free(h.a);
          return -1;
        }
      }
    }
  }
  free(h.a);
  return 0;
}

int oracle_bfs(int nodes, const int* nindex, const int* nlist, int src, int* dist) {
  if (nodes < 1 || src < 0 || src >= nodes) return -2;
  return dijkstra(nodes, nindex, nlist, NULL, src, dist);
}

int oracle_sssp(int nodes, const int* nindex, const int* nlist, const int* eweight, int src, int* dist) {
  if (nodes < 1 || src < 0 || src >= nodes || !eweight) return -2;
  return dijkstra(nodes, nindex, nlist, eweight, src, dist);
}

/* label[v] = smallest u from which v is reachable. Vertices are scanned in
   increasing order; a search from u stops at labelled vertices, which are
   reachable from a smaller ID and so are everything behind them. On a
   symmetric graph this is the minimum vertex ID of v's component. */
int oracle_cc_minlabel(int nodes, const int* nindex, const int* nlist, int* label) {
  int* stack = (int*)malloc(sizeof(int) * (size_t)nodes);
  if (!stack) return -1;
  for (int v = 0; v < nodes; v++) label[v] = -1;
  for (int u = 0; u < nodes; u++) {
    if (label[u] >= 0) continue;
    long long top = 0;
    label[u] = u;
    stack[top++] = u;
    while (top > 0) {
      const int v = stack[--top];
      for (int i = nindex[v]; i < nindex[v + 1]; i++) {
        const int n = nlist[i];
        if (label[n] < 0) {
          label[n] = u;
          stack[top++] = n;
        }
      }
    }
  }
  free(stack);
  return 0;
}

/* Reference CC verification restated. Returns 0 when it passes, else:
   1 adjacent vertices with different labels, 2 a label >= nodes (sentinel),
   3 a label that is not the same on every vertex of its component,
   4 component count mismatch (labels not unique per component). */
int oracle_cc_check(int nodes, const int* nindex, const int* nlist, const int* label) {
  for (int v = 0; v < nodes; v++)
    for (int i = nindex[v]; i < nindex[v + 1]; i++)
      if (label[nlist[i]] != label[v]) return 1;
  for (int v = 0; v < nodes; v++)
    if (label[v] >= nodes || label[v] < 0) return 2;
  int* nstat = (int*)malloc(sizeof(int) * (size_t)nodes);
  /* each vertex is expanded once and pushes its degree: at most edges + 1 entries */
  int* stack = (int*)malloc(sizeof(int) * ((size_t)nindex[nodes] + 1));
  char* seen = (char*)calloc((size_t)nodes, 1);
  if (!nstat || !stack || !seen) {
    free(nstat);
    free(stack);
    free(seen);
    return -1;
  }
  memcpy(nstat, label, sizeof(int) * (size_t)nodes);
  int rc = 0;
  long long distinct = 0, count = 0;
  for (int v = 0; v < nodes && !rc; v++) {
    if (!seen[label[v]]) {
      seen[label[v]] = 1;
      distinct++;
    }
    if (nstat[v] < nodes) {
      count++;
      const int id = nstat[v];
      long long top = 0;
      stack[top++] = v;
      while (top > 0 && !rc) {
        const int x = stack[--top];
        if (nstat[x] < nodes) {
          if (nstat[x] != id) rc = 3;
          nstat[x] = nodes;
          for (int i = nindex[x]; i < nindex[x + 1]; i++) stack[top++] = nlist[i];
        }
      }
    }
  }
  /* every distinct label must be exactly one component */
  if (!rc && distinct != count) rc = 4;
  free(nstat);
  free(stack);
  free(seen);
  return rc;
}

void oracle_synth_weights(int nodes, const int* nindex, const int* nlist, int* w) {
  for (int i = 0; i < nodes; i++)
    for (int j = nindex[i]; j < nindex[i + 1]; j++) {
      const int prod = (int)((unsigned)i * (unsigned)nlist[j]);
      int x = 1 + prod % nodes;
      w[j] = x < 0 ? -x : x;
    }
}

void oracle_sp(int nodes, const int* nindex, int* sp) {
  for (int i = 0; i < nodes; i++)
    for (int j = nindex[i]; j < nindex[i + 1]; j++) sp[j] = i;
}

/* ---- maximal independent set ------------------------------------------- */

/* The integer hash of the reference MIS codes (a published mixing function:
   two rounds of xor-shift by 16 and multiply by 0x45d9f3b, then a final
   xor-shift), applied to v + 712313887. */
static unsigned mis_hash(unsigned x) {
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  x = ((x >> 16) ^ x) * 0x45d9f3bu;
  return (x >> 16) ^ x;
}

int oracle_mis_priority(int v) { return (int)mis_hash((unsigned)v + 712313887u); }

static const int* g_mis_prio;
static int g_mis_unsigned;

/* descending rank: larger priority first, then larger ID */
static int mis_rank_cmp(const void* a, const void* b) {
  const int u = *(const int*)a, v = *(const int*)b;
  const int pu = g_mis_prio[u], pv = g_mis_prio[v];
  if (pu != pv) {
    if (g_mis_unsigned) return (unsigned)pu > (unsigned)pv ? -1 : 1;
    return pu > pv ? -1 : 1;
  }
  return u > v ? -1 : (u < v ? 1 : 0);
}

int oracle_mis(int nodes, const int* nindex, const int* nlist, int unsigned_priority, int* status) {
  if (nodes < 0) return 1;
  int* prio = (int*)malloc(sizeof(int) * (size_t)(nodes > 0 ? nodes : 1));
  int* order = (int*)malloc(sizeof(int) * (size_t)(nodes > 0 ? nodes : 1));
  if (!prio || !order) { free(prio); free(order); return 2; }
  for (int v = 0; v < nodes; ++v) { prio[v] = oracle_mis_priority(v); order[v] = v; status[v] = 0; }
  g_mis_prio = prio;
  g_mis_unsigned = unsigned_priority;
  qsort(order, (size_t)nodes, sizeof(int), mis_rank_cmp);
  for (int k = 0; k < nodes; ++k) {
    const int v = order[k];
    int in = 1;
    for (int i = nindex[v]; i < nindex[v + 1]; ++i) {
      const int u = nlist[i];
      if (u != v && status[u] == 1) { in = 0; break; }  /* only higher-ranked vertices are decided */
    }
    status[v] = in ? 1 : 2;
  }
  free(prio);
  free(order);
  return 0;
}
