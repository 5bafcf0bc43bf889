// Learned style selector: layout of the MLP parameter blob, the feature vector,
// and the block-level inference routine used inside the relax kernels' epilogue.
//
// Network: x (16 features) -> standardise with (mu, sd) -> 64 ReLU -> 64 ReLU -> 9
// outputs, one predicted log2 launch time (ns) per variant. The selector picks
// the allowed variant with the smallest prediction. Weights are stored
// [in][out] so that, for a fixed input, consecutive outputs are consecutive in memory.
#pragma once
#include "common.cuh"

namespace i2 {

static_assert(kBlock == 4 * 64, "mlp_forward_block assumes 256 threads");

constexpr int kOut = kNumVariants;
constexpr int kOffMu = 0;
constexpr int kOffSd = kOffMu + kFeatures;
constexpr int kOffW1 = kOffSd + kFeatures;
constexpr int kOffB1 = kOffW1 + kFeatures * kHidden;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden * kOut;
constexpr int kParams = kOffB3 + kOut;

// Features of a frontier about to be consumed. All are finite and O(1..30).
// The features that grow with the graph (frontier size and edges, largest
// degrees, vertex and CSR-entry counts) are clamped to the largest values of
// the training sweep (graphs of up to 2^21 vertices, 2^25.9 CSR entries,
// degree 2^16.7): a larger graph is read as the largest one trained on
// instead of extrapolating the network. The iteration index is clamped to 64
// (frontiers reach their steady state by then).
constexpr float kCapLogV = 21.f;     // log2 vertices
constexpr long long kMaxTrainedNodes = 1LL << 21;  // the largest training graph's vertices
constexpr float kCapLogE = 26.f;     // log2 CSR entries (frontier edges too)
constexpr float kCapLogDeg = 17.f;   // log2 degree
__device__ __forceinline__ float capf(float x, float hi) { return fminf(x, hi); }
__device__ __forceinline__ void frontier_features(const GStats& gs, int algo, int iter, int size, int hsize,
                                                  unsigned long long edges, int maxdeg, long long visited,
                                                  float* f) {
  const float fs = (float)size + (float)hsize;
  const float fe = (float)edges;
  const float V = (float)gs.nodes;
  const float E = (float)gs.edges > 0.f ? (float)gs.edges : 1.f;
  f[0] = capf(log2f(1.f + fs), kCapLogV);
  f[1] = capf(log2f(1.f + fe), kCapLogE);
  f[2] = fs / V;
  f[3] = fe / E;
  f[4] = log2f(1.f + fe / fmaxf(1.f, fs));
  f[5] = capf(log2f(1.f + (float)maxdeg), kCapLogDeg);
  f[6] = (float)visited / V;
  f[7] = log2f(1.f + fminf((float)iter, 64.f));
  f[8] = fminf(fmaxf(log2f(V), 16.f), kCapLogV);
  f[9] = fminf(fmaxf(log2f(1.f + (float)gs.edges), 17.f), kCapLogE);
  f[10] = log2f(1.f + gs.avgdeg);
  f[11] = capf(log2f(1.f + (float)gs.maxdeg), kCapLogDeg);
  f[12] = log2f(1.f + gs.degcv);
  f[13] = algo == kSSSP ? 1.f : 0.f;
  f[14] = algo == kCC ? 1.f : 0.f;
  f[15] = fs > 0.f ? (float)hsize / fs : 0.f;
}

// Block-cooperative forward pass for a block of kBlock (256) threads. Each
// hidden unit is computed by 4 threads (partial dot products reduced with
// shuffles) and each output by one warp, so every thread issues at most 16
// independent weight loads per layer instead of a chain of 64. x and y live in
// shared memory; h1 and h2 are shared scratch.
__device__ __forceinline__ void mlp_forward_block(const float* __restrict__ P, const float* x, float* h1,
                                                  float* h2, float* y) {
  const int t = threadIdx.x;
  const int j = t >> 2;  // hidden unit
  const int q = t & 3;   // quarter of its inputs
  if (t < 4 * kHidden) {
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < kFeatures / 4; ++i) {
      const int k = q * (kFeatures / 4) + i;
      const float xs = (x[k] - P[kOffMu + k]) / P[kOffSd + k];
      acc = fmaf(xs, P[kOffW1 + k * kHidden + j], acc);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (q == 0) h1[j] = fmaxf(acc + P[kOffB1 + j], 0.f);
  }
  __syncthreads();
  if (t < 4 * kHidden) {
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < kHidden / 4; ++i) {
      const int k = q * (kHidden / 4) + i;
      acc = fmaf(h1[k], P[kOffW2 + k * kHidden + j], acc);
    }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (q == 0) h2[j] = fmaxf(acc + P[kOffB2 + j], 0.f);
  }
  __syncthreads();
  const int lane = t & 31;
  for (int o = t >> 5; o < kOut; o += kBlock / kWarp) {  // one warp per output
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < kHidden / 32; ++i) {
      const int k = lane * (kHidden / 32) + i;
      acc = fmaf(h2[k], P[kOffW3 + k * kOut + o], acc);
    }
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
    if (lane == 0) y[o] = acc + P[kOffB3 + o];
  }
  __syncthreads();
}

}  // namespace i2
