// Host side of the graph layer: ECLgraph file I/O with status codes, CSR
// validation, the reference's synthetic SSSP weights, the starting-point array,
// and the seeded synthetic graph families (ER, RMAT, 2-D grid).
//
// File format (include/ECLgraph.h:52-80): int nodes, int edges, int nindex[nodes+1],
// int nlist[edges], then optionally int eweight[edges]; a file that ends after
// nlist has no weights, a partial weight array is an error.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_set>
#include <vector>
#include <omp.h>
#include "gen_rng.h"
#include "host_graph.h"

namespace i2 {

int validate_host_csr(const i2_eclgraph* g) {
  if (!g || g->nodes < 1 || g->edges < 0) return I2_ERR_FORMAT;
  if (!g->nindex || (g->edges > 0 && !g->nlist)) return I2_ERR_ARG;
  if (g->nindex[0] != 0 || g->nindex[g->nodes] != g->edges) return I2_ERR_FORMAT;
  int bad = 0;
  const long long V = g->nodes;
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (long long v = 0; v < V; ++v)
    if (g->nindex[v + 1] < g->nindex[v]) bad = 1;
  if (bad) return I2_ERR_FORMAT;
  const long long E = g->edges;
#pragma omp parallel for reduction(| : bad) schedule(static)
  for (long long e = 0; e < E; ++e)
    if ((unsigned)g->nlist[e] >= (unsigned)g->nodes) bad = 1;
  return bad ? I2_ERR_FORMAT : I2_OK;
}

void host_degree_stats(const i2_eclgraph* g, int heavy, int* maxdeg, int* nheavy, float* avgdeg,
                       float* degcv) {
  int mx = 0;
  long long nh = 0;
  double s2 = 0.0;
  const long long V = g->nodes;
#pragma omp parallel for reduction(max : mx) reduction(+ : nh, s2) schedule(static)
  for (long long v = 0; v < V; ++v) {
    const int d = g->nindex[v + 1] - g->nindex[v];
    mx = std::max(mx, d);
    if (d >= heavy) nh++;
    s2 += (double)d * d;
  }
  const double mean = (double)g->edges / (double)V;
  const double var = std::max(0.0, s2 / (double)V - mean * mean);
  *maxdeg = mx;
  *nheavy = (int)nh;
  *avgdeg = (float)mean;
  *degcv = mean > 0 ? (float)(std::sqrt(var) / mean) : 0.0f;
}

int csr_from_pairs(int nodes, const std::vector<uint64_t>& pairs, bool weighted, uint64_t weight_seed,
                   i2_eclgraph* out) {
  const long long P = (long long)pairs.size();
  std::vector<std::atomic<long long>> deg(nodes);
  for (int v = 0; v < nodes; ++v) deg[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < P; ++p) {
    const int u = (int)(pairs[p] >> 32), v = (int)(pairs[p] & 0xffffffffu);
    if (u == v) continue;
    deg[u].fetch_add(1, std::memory_order_relaxed);
    deg[v].fetch_add(1, std::memory_order_relaxed);
  }
  std::vector<long long> off(nodes + 1);
  off[0] = 0;
  for (int v = 0; v < nodes; ++v) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
  std::vector<int> nbr((size_t)off[nodes]);
  std::vector<std::atomic<long long>> pos(nodes);
  for (int v = 0; v < nodes; ++v) pos[v].store(off[v], std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (long long p = 0; p < P; ++p) {
    const int u = (int)(pairs[p] >> 32), v = (int)(pairs[p] & 0xffffffffu);
    if (u == v) continue;
    nbr[pos[u].fetch_add(1, std::memory_order_relaxed)] = v;
    nbr[pos[v].fetch_add(1, std::memory_order_relaxed)] = u;
  }
  std::vector<long long> nd(nodes + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < nodes; ++v) {
    int* b = nbr.data() + off[v];
    int* e = nbr.data() + off[v + 1];
    std::sort(b, e);
    nd[v] = std::unique(b, e) - b;
  }
  long long E = 0;
  for (int v = 0; v < nodes; ++v) E += nd[v];
  if (E > 0x7fffffffLL) return I2_ERR_OVERFLOW;
  int st = i2_alloc_eclgraph(nodes, (int)E, weighted ? 1 : 0, out);
  if (st != I2_OK) return st;
  out->nindex[0] = 0;
  for (int v = 0; v < nodes; ++v) out->nindex[v + 1] = out->nindex[v] + (int)nd[v];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < nodes; ++v) {
    const int o = out->nindex[v];
    std::memcpy(out->nlist + o, nbr.data() + off[v], sizeof(int) * nd[v]);
    if (weighted)
      for (int k = 0; k < nd[v]; ++k) out->eweight[o + k] = edge_weight(weight_seed, v, out->nlist[o + k]);
  }
  return I2_OK;
}

}  // namespace i2

using namespace i2;

extern "C" {

int i2_alloc_eclgraph(int nodes, int edges, int weighted, i2_eclgraph* out) {
  if (!out || nodes < 1 || edges < 0) return I2_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  out->nodes = nodes;
  out->edges = edges;
  // Padding of 4 ints lets 128-bit readers run past the last entry safely.
  out->nindex = (int*)std::calloc((size_t)nodes + 1, sizeof(int));
  out->nlist = (int*)std::malloc(((size_t)edges + 4) * sizeof(int));
  out->eweight = weighted ? (int*)std::malloc(((size_t)edges + 4) * sizeof(int)) : nullptr;
  if (!out->nindex || !out->nlist || (weighted && !out->eweight)) {
    i2_free_eclgraph(out);
    return I2_ERR_NOMEM;
  }
  return I2_OK;
}

void i2_free_eclgraph(i2_eclgraph* g) {
  if (!g) return;
  std::free(g->nindex);
  std::free(g->nlist);
  std::free(g->eweight);
  g->nindex = g->nlist = g->eweight = nullptr;
}

int i2_read_eclgraph(const char* path, i2_eclgraph* out) {
  if (!path || !out) return I2_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return I2_ERR_IO;
  int hdr[2];
  if (std::fread(hdr, sizeof(int), 2, f) != 2) {
    std::fclose(f);
    return I2_ERR_FORMAT;
  }
  if (hdr[0] < 1 || hdr[1] < 0) {
    std::fclose(f);
    return I2_ERR_FORMAT;
  }
  int st = i2_alloc_eclgraph(hdr[0], hdr[1], 1, out);
  if (st != I2_OK) {
    std::fclose(f);
    return st;
  }
  const size_t nn = (size_t)hdr[0] + 1, ne = (size_t)hdr[1];
  if (std::fread(out->nindex, sizeof(int), nn, f) != nn || std::fread(out->nlist, sizeof(int), ne, f) != ne) {
    std::fclose(f);
    i2_free_eclgraph(out);
    return I2_ERR_FORMAT;
  }
  const size_t nw = ne ? std::fread(out->eweight, sizeof(int), ne, f) : 0;
  if (nw == 0) {
    std::free(out->eweight);
    out->eweight = nullptr;
  } else if (nw != ne) {
    std::fclose(f);
    i2_free_eclgraph(out);
    return I2_ERR_FORMAT;
  }
  std::fclose(f);
  st = validate_host_csr(out);
  if (st != I2_OK) i2_free_eclgraph(out);
  return st;
}

int i2_write_eclgraph(const i2_eclgraph* g, const char* path) {
  if (!g || !path) return I2_ERR_ARG;
  if (g->nodes < 1 || g->edges < 0) return I2_ERR_FORMAT;
  FILE* f = std::fopen(path, "wb");
  if (!f) return I2_ERR_IO;
  bool ok = std::fwrite(&g->nodes, sizeof(int), 1, f) == 1 && std::fwrite(&g->edges, sizeof(int), 1, f) == 1 &&
            std::fwrite(g->nindex, sizeof(int), (size_t)g->nodes + 1, f) == (size_t)g->nodes + 1 &&
            std::fwrite(g->nlist, sizeof(int), (size_t)g->edges, f) == (size_t)g->edges;
  if (ok && g->eweight)
    ok = std::fwrite(g->eweight, sizeof(int), (size_t)g->edges, f) == (size_t)g->edges;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? I2_OK : I2_ERR_IO;
}

// Reference formula (include/sssp_vertex_cuda.h:127-137): w = 1 + (i * nei) % nodes,
// negated when negative. The int product wraps in two's complement here, which is
// what the reference's compiled code computes.
int i2_synth_weights(i2_eclgraph* g) {
  if (!g || !g->nindex || g->nodes < 1) return I2_ERR_ARG;
  if (!g->eweight) {
    g->eweight = (int*)std::malloc(((size_t)g->edges + 4) * sizeof(int));
    if (!g->eweight) return I2_ERR_NOMEM;
  }
  const int V = g->nodes;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int i = 0; i < V; ++i) {
    for (int j = g->nindex[i]; j < g->nindex[i + 1]; ++j) {
      const int nei = g->nlist[j];
      const int prod = (int)((unsigned)i * (unsigned)nei);
      int w = 1 + (prod % V);
      if (w < 0) w = -w;
      g->eweight[j] = w;
    }
  }
  return I2_OK;
}

int i2_build_sp(const i2_eclgraph* g, int* sp) {
  if (!g || !sp || !g->nindex) return I2_ERR_ARG;
  const int V = g->nodes;
#pragma omp parallel for schedule(dynamic, 4096)
  for (int i = 0; i < V; ++i)
    for (int j = g->nindex[i]; j < g->nindex[i + 1]; ++j) sp[j] = i;
  return I2_OK;
}

// G(n, m): the first m distinct unordered non-loop pairs of the hash stream,
// i.e. m pairs sampled uniformly without replacement.
int i2_gen_er(int n, long long m, uint64_t seed, int weighted, i2_eclgraph* out) {
  if (!out || n < 2 || m < 0) return I2_ERR_ARG;
  const long long maxm = (long long)n * (n - 1) / 2;
  if (m > maxm || 2 * m > 0x7fffffffLL) return I2_ERR_ARG;
  long long C = m + m / 16 + 64;
  std::vector<uint64_t> pairs;
  for (;;) {
    std::vector<std::pair<uint64_t, long long>> cand((size_t)C);
#pragma omp parallel for schedule(static)
    for (long long j = 0; j < C; ++j) {
      const uint64_t u = h3(seed, kStreamErU, (uint64_t)j) % (uint64_t)n;
      const uint64_t v = h3(seed, kStreamErV, (uint64_t)j) % (uint64_t)n;
      const uint64_t lo = u < v ? u : v, hi = u < v ? v : u;
      cand[j] = {u == v ? ~0ull : ((lo << 32) | hi), j};
    }
    std::sort(cand.begin(), cand.end());
    std::vector<std::pair<long long, uint64_t>> first;
    first.reserve((size_t)C);
    for (size_t k = 0; k < cand.size(); ++k) {
      if (cand[k].first == ~0ull) break;
      if (k == 0 || cand[k].first != cand[k - 1].first) first.push_back({cand[k].second, cand[k].first});
    }
    if ((long long)first.size() >= m || C > 8 * (m + 64)) {
      if ((long long)first.size() < m) return I2_ERR_ARG;
      std::sort(first.begin(), first.end());
      pairs.resize((size_t)m);
      for (long long k = 0; k < m; ++k) pairs[k] = first[k].second;
      break;
    }
    C = C + C / 4 + 64;
  }
  return csr_from_pairs(n, pairs, weighted != 0, seed, out);
}

// RMAT with n = 2^scale vertices, edge_factor * n samples, seeded relabelling.
static int gen_rmat_n(int n, int scale, long long samples, double a, double b, double c, uint64_t seed,
                      int weighted, i2_eclgraph* out) {
  const RmatThresholds t = make_thresholds(a, b, c);
  const RmatPerm p = make_perm(seed, scale);
  std::vector<uint64_t> pairs((size_t)samples);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < samples; ++i) {
    uint64_t u, v;
    rmat_sample(seed, scale, t, (uint64_t)i, &u, &v);
    u = perm_apply(p, u);
    v = perm_apply(p, v);
    if (u >= (uint64_t)n || v >= (uint64_t)n) u = v = 0;  // rejected: becomes a dropped self-loop
    pairs[i] = (u << 32) | v;
  }
  return csr_from_pairs(n, pairs, weighted != 0, seed, out);
}

int i2_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                i2_eclgraph* out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1) return I2_ERR_ARG;
  if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return I2_ERR_ARG;
  const long long n = 1LL << scale;
  return gen_rmat_n((int)n, scale, (long long)edge_factor * n, a, b, c, seed, weighted, out);
}

int i2_gen_rmat_n(int n, int edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                  i2_eclgraph* out) {
  if (!out || n < 2 || edge_factor < 1) return I2_ERR_ARG;
  int scale = 1;
  while ((1LL << scale) < n) ++scale;
  return gen_rmat_n(n, scale, (long long)edge_factor << scale, a, b, c, seed, weighted, out);
}

// side x side 4-neighbour grid; each grid edge is dropped with probability
// remove_frac; then round(add_frac * kept) long-range edges are added, each a
// new pair (no loops, no duplicates of kept grid edges or of each other).
int i2_gen_grid(int side, double remove_frac, double add_frac, uint64_t seed, int weighted, i2_eclgraph* out) {
  if (!out || side < 2 || remove_frac < 0 || remove_frac >= 1 || add_frac < 0) return I2_ERR_ARG;
  const long long V = (long long)side * side;
  if (V > 0x7fffffffLL) return I2_ERR_ARG;
  const long long H = (long long)side * (side - 1);  // horizontal edges
  const long long G = 2 * H;
  const uint64_t drop = prob_to_u64(remove_frac);
  auto kept = [&](long long idx) { return h3(seed, kStreamGridDrop, (uint64_t)idx) >= drop; };
  std::vector<uint64_t> pairs;
  pairs.reserve((size_t)G);
  for (long long idx = 0; idx < G; ++idx) {
    if (!kept(idx)) continue;
    long long u, v;
    if (idx < H) {
      const long long r = idx / (side - 1), cc = idx % (side - 1);
      u = r * side + cc;
      v = u + 1;
    } else {
      u = idx - H;
      v = u + side;
    }
    pairs.push_back(((uint64_t)u << 32) | (uint64_t)v);
  }
  const long long K = std::llround(add_frac * (double)pairs.size());
  std::vector<uint64_t> extra;
  std::unordered_set<uint64_t> seen;
  auto grid_edge_index = [&](long long lo, long long hi) -> long long {
    if (hi == lo + 1 && (lo % side) != side - 1) return (lo / side) * (side - 1) + (lo % side);
    if (hi == lo + side) return H + lo;
    return -1;
  };
  for (long long j = 0; (long long)extra.size() < K; ++j) {
    const long long u = (long long)(h3(seed, kStreamGridU, (uint64_t)j) % (uint64_t)V);
    const long long v = (long long)(h3(seed, kStreamGridV, (uint64_t)j) % (uint64_t)V);
    if (u == v) continue;
    const long long lo = std::min(u, v), hi = std::max(u, v);
    const long long gi = grid_edge_index(lo, hi);
    if (gi >= 0 && kept(gi)) continue;
    const uint64_t key = ((uint64_t)lo << 32) | (uint64_t)hi;
    if (!seen.insert(key).second) continue;
    extra.push_back(key);
  }
  pairs.insert(pairs.end(), extra.begin(), extra.end());
  return csr_from_pairs((int)V, pairs, weighted != 0, seed, out);
}

}  // extern "C"
