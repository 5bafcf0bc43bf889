// Counter-based random numbers shared by the host and device graph generators.
// Every random choice is a pure function of (seed, stream, index), so a graph
// built on the host and the same graph built on the device are identical.
// The mixer is the SplitMix64 finaliser (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014).
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define I2_HD __host__ __device__ __forceinline__
#else
#define I2_HD inline
#endif

namespace i2 {

I2_HD uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Hash of (seed, stream, index).
I2_HD uint64_t h3(uint64_t seed, uint64_t stream, uint64_t index) {
  return mix64(mix64(seed ^ 0x5851F42D4C957F2Dull) + stream * 0xD1342543DE82EF95ull +
               mix64(index + 0x2545F4914F6CDD1Dull));
}

// Random streams.
enum : uint64_t {
  kStreamRmat = 11,
  kStreamPermMul = 12,
  kStreamPermAdd = 13,
  kStreamErU = 21,
  kStreamErV = 22,
  kStreamGridDrop = 31,
  kStreamGridU = 32,
  kStreamGridV = 33,
  kStreamWeight = 41,
};

// Weight of the undirected edge {u, v}: uniform in [1, 255], same in both directions.
I2_HD int edge_weight(uint64_t seed, int u, int v) {
  const uint64_t lo = (uint64_t)(u < v ? u : v);
  const uint64_t hi = (uint64_t)(u < v ? v : u);
  return 1 + (int)(h3(seed, kStreamWeight, (hi << 32) | lo) % 255ull);
}

// RMAT quadrant thresholds as 64-bit integers, so host and device agree exactly.
struct RmatThresholds {
  uint64_t ta, tab, tabc;
};

// Seeded bijection of [0, 2^scale) used to relabel RMAT vertices (hubs are
// otherwise the low IDs). Rounds of odd multiplication, xor-shift and addition
// modulo 2^scale, each a bijection.
struct RmatPerm {
  uint64_t mul[4];
  uint64_t add[4];
  uint64_t mask;
  int shift;
};

I2_HD uint64_t perm_apply(const RmatPerm& p, uint64_t x) {
  for (int r = 0; r < 4; ++r) {
    x = (x * p.mul[r]) & p.mask;
    x ^= x >> p.shift;
    x = (x + p.add[r]) & p.mask;
  }
  return x;
}

inline RmatPerm make_perm(uint64_t seed, int scale) {
  RmatPerm p;
  p.mask = (scale >= 64) ? ~0ull : ((1ull << scale) - 1);
  p.shift = scale / 2 + 1;
  for (int r = 0; r < 4; ++r) {
    p.mul[r] = (h3(seed, kStreamPermMul, r) | 1ull) & p.mask;
    if (p.mul[r] == 0) p.mul[r] = 1;
    p.add[r] = h3(seed, kStreamPermAdd, r) & p.mask;
  }
  return p;
}

// Directed RMAT sample i (before relabelling): one hash per level.
I2_HD void rmat_sample(uint64_t seed, int scale, const RmatThresholds& t, uint64_t i, uint64_t* u,
                       uint64_t* v) {
  uint64_t a = 0, b = 0;
  for (int l = 0; l < scale; ++l) {
    const uint64_t r = h3(seed, kStreamRmat, i * 64 + (uint64_t)l);
    const uint64_t bu = (r >= t.tab) ? 1 : 0;                           // quadrants c, d
    const uint64_t bv = (r >= t.ta && r < t.tab) || (r >= t.tabc) ? 1 : 0;  // quadrants b, d
    a = (a << 1) | bu;
    b = (b << 1) | bv;
  }
  *u = a;
  *v = b;
}

inline uint64_t prob_to_u64(double p) {
  if (p <= 0.0) return 0;
  if (p >= 1.0) return ~0ull;
  return (uint64_t)(p * 18446744073709551616.0);
}

inline RmatThresholds make_thresholds(double a, double b, double c) {
  RmatThresholds t;
  t.ta = prob_to_u64(a);
  t.tab = prob_to_u64(a + b);
  t.tabc = prob_to_u64(a + b + c);
  return t;
}

}  // namespace i2
