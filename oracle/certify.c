// ORACLE — test infrastructure only.
//
// Size-independent certificates of BFS levels / SSSP distances and of
// minimum-ID connected-component labels, for graphs where the serial oracle
// (oracle.c) would take too long (RMAT scale 26: 2.1e9 CSR entries). They
// check the same properties as the reference's verifiers, which compare with
// a serial Dijkstra (include/sssp_edge_cuda.h:184-196) and check labels across
// edges and per component (include/cc_vertex_cuda.h:142-170), in parallel
// passes over the CSR with 64-bit indices.
#include <limits.h>
#include <stdlib.h>

// Distances from src with weights w >= 1 (w = NULL: every weight is 1) are the
// shortest-path distances iff dist[src] == 0, no edge out of a reached vertex
// is relaxable (so dist[v] <= d(v) by induction along a shortest path), and
// every other reached vertex has a tight in-edge (following tight edges back
// strictly lowers the value, so it ends at src: dist[v] is the length of a
// real path, >= d(v)). A reached vertex's neighbours must be reached.
// Returns 0 when the certificate holds, else the first failed check:
// 1 dist[src] != 0, 2 a negative value, 3 unreached neighbour of a reached
// vertex, 4 relaxable edge, 5 reached vertex without a tight in-edge,
// 6 a weight below 1, -1 out of memory.
int oracle_certify_distances(int nodes, const int* nindex, const int* nlist, const int* w, int src,
                             const int* dist) {
  if (nodes < 1 || src < 0 || src >= nodes) return -2;
  if (dist[src] != 0) return 1;
  unsigned char* tight = (unsigned char*)calloc((size_t)nodes, 1);
  if (!tight) return -1;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad)
  for (int u = 0; u < nodes; ++u) {
    const int du = dist[u];
    if (du == INT_MAX) continue;
    if (du < 0) {
      bad |= 1 << 2;
      continue;
    }
    for (long long e = nindex[u]; e < nindex[u + 1]; ++e) {
      const int v = nlist[e];
      const long long wt = w ? w[e] : 1;
      if (wt < 1) {
        bad |= 1 << 6;
        continue;
      }
      const int dv = dist[v];
      if (dv == INT_MAX) {
        bad |= 1 << 3;
        continue;
      }
      const long long c = (long long)du + wt;
      if ((long long)dv > c) bad |= 1 << 4;
      if ((long long)dv == c && !tight[v]) {
#pragma omp atomic write
        tight[v] = 1;
      }
    }
  }
  if (!bad) {
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int v = 0; v < nodes; ++v)
      if (v != src && dist[v] != INT_MAX && !tight[v]) bad |= 1 << 5;
  }
  free(tight);
  for (int k = 2; k <= 6; ++k)
    if (bad & (1 << k)) return k;
  return 0;
}

// Minimum-ID labels of a symmetric graph: labels are equal across every edge
// (so each component has one label), 0 <= label[v] <= v, label[label[v]] ==
// label[v] (the label is a root), and every vertex is connected to the root of
// its label (checked by one multi-source BFS from all roots, level by level).
// Then each component's label is a vertex of that component no larger than any
// of its vertices: its minimum ID.
// Returns 0 when it holds, else 1 adjacent labels differ, 2 label out of range
// or above its vertex, 3 label is not its own label, 4 a vertex not connected
// to its label's root, -1 out of memory.
int oracle_certify_cc(int nodes, const int* nindex, const int* nlist, const int* label) {
  if (nodes < 1) return -2;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad)
  for (int v = 0; v < nodes; ++v) {
    const int l = label[v];
    if (l < 0 || l > v) {
      bad |= 1 << 2;
      continue;
    }
    if (label[l] != l) bad |= 1 << 3;
    for (long long e = nindex[v]; e < nindex[v + 1]; ++e)
      if (label[nlist[e]] != l) bad |= 1 << 1;
  }
  for (int k = 1; k <= 3; ++k)
    if (bad & (1 << k)) return k;
  unsigned char* seen = (unsigned char*)calloc((size_t)nodes, 1);
  int* cur = (int*)malloc(sizeof(int) * (size_t)nodes);
  int* nxt = (int*)malloc(sizeof(int) * (size_t)nodes);
  if (!seen || !cur || !nxt) {
    free(seen);
    free(cur);
    free(nxt);
    return -1;
  }
  long long n = 0;
  for (int v = 0; v < nodes; ++v)
    if (label[v] == v) {
      seen[v] = 1;
      cur[n++] = v;
    }
  long long reached = n;
  while (n > 0) {
    long long m = 0;
#pragma omp parallel
    {
      // per-thread buffer flushed into nxt with one atomic capture per batch
      int buf[1024];
      int k = 0;
#pragma omp for schedule(dynamic, 256)
      for (long long i = 0; i < n; ++i) {
        const int u = cur[i];
        for (long long e = nindex[u]; e < nindex[u + 1]; ++e) {
          const int v = nlist[e];
          if (seen[v]) continue;
          unsigned char was;
#pragma omp atomic capture
          {
            was = seen[v];
            seen[v] = 1;
          }
          if (was) continue;
          buf[k++] = v;
          if (k == 1024) {
            long long at;
#pragma omp atomic capture
            {
              at = m;
              m += k;
            }
            for (int j = 0; j < k; ++j) nxt[at + j] = buf[j];
            k = 0;
          }
        }
      }
      if (k) {
        long long at;
#pragma omp atomic capture
        {
          at = m;
          m += k;
        }
        for (int j = 0; j < k; ++j) nxt[at + j] = buf[j];
      }
    }
    int* t = cur;
    cur = nxt;
    nxt = t;
    n = m;
    reached += m;
  }
  free(seen);
  free(cur);
  free(nxt);
  return reached == nodes ? 0 : 4;
}
