// ORACLE — test infrastructure only.
//
// Independent C restatement of the engine's seeded RMAT generator, so that
// the benchmark's reference arm and the tests can build the very graph the
// engine's generators build without loading the engine library. The graph is
// defined by these rules, which this file states on its own:
//
//  * mix(z) is the SplitMix64 output function (Steele, Lea and Flood,
//    "Fast splittable pseudorandom number generators", OOPSLA 2014);
//  * hash(seed, stream, i) = mix(mix(seed ^ K1) + stream * K2 + mix(i + K3));
//  * sample i chooses, at each of `scale` levels l, the RMAT quadrant from
//    r = hash(seed, 11, 64 i + l) against the 64-bit thresholds a, a+b, a+b+c
//    (a probability p is the integer floor(p * 2^64));
//  * both endpoints are relabelled by a seeded bijection of [0, 2^scale):
//    four rounds of x = x * m_r (odd, mod 2^scale), x ^= x >> (scale/2 + 1),
//    x = x + a_r (mod 2^scale), m_r = hash(seed, 12, r) | 1, a_r = hash(seed, 13, r);
//  * the CSR holds both directions of every sampled non-loop pair, each row
//    sorted and deduplicated; the weight of {u, v} is
//    1 + hash(seed, 41, max(u,v) << 32 | min(u,v)) % 255, the same both ways.
//
// The reference (Indigo2Suite) ships no generator; its inputs are .egr files
// (include/ECLgraph.h:52-80 layout), which oracle.write_egr produces from this
// CSR.
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t i) {
  return mix(mix(seed ^ 0x5851F42D4C957F2Dull) + stream * 0xD1342543DE82EF95ull + mix(i + 0x2545F4914F6CDD1Dull));
}

static uint64_t prob64(double p) {
  if (p <= 0.0) return 0;
  if (p >= 1.0) return ~0ull;
  return (uint64_t)(p * 18446744073709551616.0);
}

static int cmp_int(const void* x, const void* y) {
  const int a = *(const int*)x, b = *(const int*)y;
  return (a > b) - (a < b);
}

static void sort_row(int* r, long long n) {
  if (n < 24) {  // insertion sort for the many short rows
    for (long long i = 1; i < n; ++i) {
      const int x = r[i];
      long long j = i - 1;
      while (j >= 0 && r[j] > x) {
        r[j + 1] = r[j];
        --j;
      }
      r[j + 1] = x;
    }
  } else {
    qsort(r, (size_t)n, sizeof(int), cmp_int);
  }
}

void oracle_graph_free(int* nindex, int* nlist, int* eweight) {
  free(nindex);
  free(nlist);
  free(eweight);
}

// Returns 0 and fills the CSR (malloc'd; free with oracle_graph_free), or a
// negative code: -1 bad arguments, -2 out of memory, -3 more than INT32_MAX
// CSR entries.
int oracle_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                    int* nodes_out, int* edges_out, int** nindex_out, int** nlist_out, int** eweight_out) {
  if (scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  const int n = 1 << scale;
  const long long S = (long long)edge_factor * n;
  const uint64_t ta = prob64(a), tab = prob64(a + b), tabc = prob64(a + b + c);
  const uint64_t mask = ((uint64_t)1 << scale) - 1;
  const int shift = scale / 2 + 1;
  uint64_t mul[4], add[4];
  for (int r = 0; r < 4; ++r) {
    mul[r] = (hash3(seed, 12, (uint64_t)r) | 1ull) & mask;
    if (mul[r] == 0) mul[r] = 1;
    add[r] = hash3(seed, 13, (uint64_t)r) & mask;
  }
  int* su = (int*)malloc(sizeof(int) * (size_t)S);
  int* sv = (int*)malloc(sizeof(int) * (size_t)S);
  long long* deg = (long long*)calloc((size_t)n + 1, sizeof(long long));
  if (!su || !sv || !deg) {
    free(su);
    free(sv);
    free(deg);
    return -2;
  }
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < S; ++i) {
    uint64_t x = 0, y = 0;
    for (int l = 0; l < scale; ++l) {
      const uint64_t r = hash3(seed, 11, (uint64_t)i * 64 + (uint64_t)l);
      const uint64_t lower = r >= tab;                              // quadrants c, d
      const uint64_t right = (r >= ta && r < tab) || r >= tabc;     // quadrants b, d
      x = (x << 1) | lower;
      y = (y << 1) | right;
    }
    for (int k = 0; k < 2; ++k) {
      uint64_t z = k ? y : x;
      for (int r = 0; r < 4; ++r) {
        z = (z * mul[r]) & mask;
        z ^= z >> shift;
        z = (z + add[r]) & mask;
      }
      if (k) y = z; else x = z;
    }
    su[i] = (int)x;
    sv[i] = (int)y;
  }
  for (long long i = 0; i < S; ++i)
    if (su[i] != sv[i]) {
      deg[su[i]]++;
      deg[sv[i]]++;
    }
  long long* off = (long long*)malloc(sizeof(long long) * ((size_t)n + 1));
  if (!off) {
    free(su);
    free(sv);
    free(deg);
    return -2;
  }
  off[0] = 0;
  for (int v = 0; v < n; ++v) off[v + 1] = off[v] + deg[v];
  int* nbr = (int*)malloc(sizeof(int) * (size_t)(off[n] > 0 ? off[n] : 1));
  if (!nbr) {
    free(su);
    free(sv);
    free(deg);
    free(off);
    return -2;
  }
  for (int v = 0; v < n; ++v) deg[v] = off[v];  // reused as fill cursors
  for (long long i = 0; i < S; ++i)
    if (su[i] != sv[i]) {
      nbr[deg[su[i]]++] = sv[i];
      nbr[deg[sv[i]]++] = su[i];
    }
  free(su);
  free(sv);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < n; ++v) {
    int* r = nbr + off[v];
    const long long len = off[v + 1] - off[v];
    sort_row(r, len);
    long long k = 0;
    for (long long j = 0; j < len; ++j)
      if (k == 0 || r[j] != r[k - 1]) r[k++] = r[j];
    deg[v] = k;
  }
  long long E = 0;
  for (int v = 0; v < n; ++v) E += deg[v];
  if (E > 0x7fffffffLL) {
    free(nbr);
    free(deg);
    free(off);
    return -3;
  }
  int* nindex = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  int* nlist = (int*)malloc(sizeof(int) * ((size_t)E + 4));
  int* ew = weighted ? (int*)malloc(sizeof(int) * ((size_t)E + 4)) : NULL;
  if (!nindex || !nlist || (weighted && !ew)) {
    free(nindex);
    free(nlist);
    free(ew);
    free(nbr);
    free(deg);
    free(off);
    return -2;
  }
  nindex[0] = 0;
  for (int v = 0; v < n; ++v) nindex[v + 1] = nindex[v] + (int)deg[v];
#pragma omp parallel for schedule(dynamic, 1024)
  for (int v = 0; v < n; ++v) {
    const int o = nindex[v];
    memcpy(nlist + o, nbr + off[v], sizeof(int) * (size_t)deg[v]);
    if (ew)
      for (int k = 0; k < (int)deg[v]; ++k) {
        const uint64_t u = (uint64_t)v, w = (uint64_t)nlist[o + k];
        const uint64_t lo = u < w ? u : w, hi = u < w ? w : u;
        ew[o + k] = 1 + (int)(hash3(seed, 41, (hi << 32) | lo) % 255ull);
      }
  }
  memset(nlist + E, 0, 4 * sizeof(int));
  if (ew) memset(ew + E, 0, 4 * sizeof(int));
  free(nbr);
  free(deg);
  free(off);
  *nodes_out = n;
  *edges_out = (int)E;
  *nindex_out = nindex;
  *nlist_out = nlist;
  *eweight_out = ew;
  return 0;
}
