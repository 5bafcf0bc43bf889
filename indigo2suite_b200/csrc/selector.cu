// Training and batched inference of the learned style selector (mlp.cuh).
//
// Loss: masked mean squared error between predicted and measured log2 launch
// times, L = sum(M * (Y - T)^2) / sum(M), over rows of 16 features and 9
// per-variant targets. The forward and backward passes are one fused kernel:
// each block owns kRows rows, keeps the weights and the activations in shared
// memory, and writes its partial gradient to its own slot; a second kernel sums
// the slots in a fixed order, so gradients are deterministic. Sizes are tiny
// (5.8k parameters), so the math stays in fp32 SIMT: it runs once per selector
// training and is off the traversal's roofline.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>
#include "engine.h"
#include "mlp.cuh"

namespace i2 {

constexpr int kRows = 32;       // rows per block
constexpr int kTBlock = 256;

struct MlpSmem {
  float P[kParams];
  float xs[kRows][kFeatures];
  float a1[kRows][kHidden];
  float a2[kRows][kHidden];
  float d2[kRows][kHidden];  // dZ2
  float d1[kRows][kHidden];  // dZ1
  float dy[kRows][kOut];
  float loss[kTBlock];
};

// grads: [gridDim.x][kParams] partials; loss_part: [gridDim.x].
__global__ void __launch_bounds__(kTBlock) k_mlp_fwd_bwd(const float* __restrict__ P, const float* __restrict__ X,
                                                         const float* __restrict__ T, const float* __restrict__ M,
                                                         const int* __restrict__ idx, int n, float inv_cnt,
                                                         float* __restrict__ grads, float* __restrict__ loss_part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem_raw);
  const int t = threadIdx.x;
  const int r0 = blockIdx.x * kRows;
  for (int k = t; k < kParams; k += kTBlock) S.P[k] = P[k];
  __syncthreads();
  // standardised inputs
  for (int e = t; e < kRows * kFeatures; e += kTBlock) {
    const int r = e / kFeatures, k = e % kFeatures;
    const int row = r0 + r;
    float v = 0.f;
    if (row < n) {
      const int src = idx ? idx[row] : row;
      v = (X[(size_t)src * kFeatures + k] - S.P[kOffMu + k]) / S.P[kOffSd + k];
    }
    S.xs[r][k] = v;
  }
  __syncthreads();
  // layer 1
  for (int e = t; e < kRows * kHidden; e += kTBlock) {
    const int r = e / kHidden, j = e % kHidden;
    float acc = S.P[kOffB1 + j];
    for (int k = 0; k < kFeatures; ++k) acc = fmaf(S.xs[r][k], S.P[kOffW1 + k * kHidden + j], acc);
    S.a1[r][j] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  // layer 2
  for (int e = t; e < kRows * kHidden; e += kTBlock) {
    const int r = e / kHidden, j = e % kHidden;
    float acc = S.P[kOffB2 + j];
    for (int k = 0; k < kHidden; ++k) acc = fmaf(S.a1[r][k], S.P[kOffW2 + k * kHidden + j], acc);
    S.a2[r][j] = fmaxf(acc, 0.f);
  }
  __syncthreads();
  // layer 3, loss and dY
  float lsum = 0.f;
  for (int e = t; e < kRows * kOut; e += kTBlock) {
    const int r = e / kOut, o = e % kOut;
    const int row = r0 + r;
    float d = 0.f;
    if (row < n) {
      float acc = S.P[kOffB3 + o];
      for (int k = 0; k < kHidden; ++k) acc = fmaf(S.a2[r][k], S.P[kOffW3 + k * kOut + o], acc);
      const int src = idx ? idx[row] : row;
      const float m = M[(size_t)src * kOut + o];
      const float diff = acc - T[(size_t)src * kOut + o];
      lsum += m * diff * diff * inv_cnt;
      d = 2.f * m * diff * inv_cnt;
    }
    S.dy[r][o] = d;
  }
  S.loss[t] = lsum;
  __syncthreads();
  // dZ2 = (dY W3^T) * relu'(Z2)
  for (int e = t; e < kRows * kHidden; e += kTBlock) {
    const int r = e / kHidden, j = e % kHidden;
    float acc = 0.f;
    for (int o = 0; o < kOut; ++o) acc = fmaf(S.dy[r][o], S.P[kOffW3 + j * kOut + o], acc);
    S.d2[r][j] = S.a2[r][j] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // dZ1 = (dZ2 W2^T) * relu'(Z1)
  for (int e = t; e < kRows * kHidden; e += kTBlock) {
    const int r = e / kHidden, i = e % kHidden;
    float acc = 0.f;
    for (int j = 0; j < kHidden; ++j) acc = fmaf(S.d2[r][j], S.P[kOffW2 + i * kHidden + j], acc);
    S.d1[r][i] = S.a1[r][i] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  float* G = grads + (size_t)blockIdx.x * kParams;
  for (int k = t; k < kOffW1; k += kTBlock) G[k] = 0.f;  // normaliser is not trained
  for (int e = t; e < kFeatures * kHidden; e += kTBlock) {
    const int k = e / kHidden, i = e % kHidden;
    float acc = 0.f;
    for (int r = 0; r < kRows; ++r) acc = fmaf(S.xs[r][k], S.d1[r][i], acc);
    G[kOffW1 + e] = acc;
  }
  for (int i = t; i < kHidden; i += kTBlock) {
    float a = 0.f, b = 0.f;
    for (int r = 0; r < kRows; ++r) {
      a += S.d1[r][i];
      b += S.d2[r][i];
    }
    G[kOffB1 + i] = a;
    G[kOffB2 + i] = b;
  }
  for (int e = t; e < kHidden * kHidden; e += kTBlock) {
    const int i = e / kHidden, j = e % kHidden;
    float acc = 0.f;
    for (int r = 0; r < kRows; ++r) acc = fmaf(S.a1[r][i], S.d2[r][j], acc);
    G[kOffW2 + e] = acc;
  }
  for (int e = t; e < kHidden * kOut; e += kTBlock) {
    const int j = e / kOut, o = e % kOut;
    float acc = 0.f;
    for (int r = 0; r < kRows; ++r) acc = fmaf(S.a2[r][j], S.dy[r][o], acc);
    G[kOffW3 + e] = acc;
  }
  for (int o = t; o < kOut; o += kTBlock) {
    float acc = 0.f;
    for (int r = 0; r < kRows; ++r) acc += S.dy[r][o];
    G[kOffB3 + o] = acc;
  }
  if (t == 0) {
    float l = 0.f;
    for (int k = 0; k < kTBlock; ++k) l += S.loss[k];
    loss_part[blockIdx.x] = l;
  }
}

// Sum the per-block partials in block order.
__global__ void k_mlp_reduce(const float* __restrict__ parts, int nblk, float* __restrict__ out,
                             const float* __restrict__ loss_part, float* __restrict__ loss) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < kParams) {
    float acc = 0.f;
    for (int b = 0; b < nblk; ++b) acc += parts[(size_t)b * kParams + k];
    out[k] = acc;
  }
  if (k == 0) {
    float l = 0.f;
    for (int b = 0; b < nblk; ++b) l += loss_part[b];
    *loss = l;
  }
}

// Adam (Kingma and Ba, 2015) on the trainable part of the blob.
__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int k = kOffW1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kParams) return;
  const float g = G[k];
  const float a = b1 * m1[k] + (1.f - b1) * g;
  const float b = b2 * m2[k] + (1.f - b2) * g * g;
  m1[k] = a;
  m2[k] = b;
  P[k] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}

__global__ void k_mlp_predict(const float* __restrict__ P, const float* __restrict__ X, int n, int allowed,
                              int* __restrict__ choice) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  float xs[kFeatures], h1[kHidden], h2[kHidden];
  for (int k = 0; k < kFeatures; ++k) xs[k] = (X[(size_t)row * kFeatures + k] - P[kOffMu + k]) / P[kOffSd + k];
  for (int j = 0; j < kHidden; ++j) {
    float acc = P[kOffB1 + j];
    for (int k = 0; k < kFeatures; ++k) acc = fmaf(xs[k], P[kOffW1 + k * kHidden + j], acc);
    h1[j] = fmaxf(acc, 0.f);
  }
  for (int j = 0; j < kHidden; ++j) {
    float acc = P[kOffB2 + j];
    for (int k = 0; k < kHidden; ++k) acc = fmaf(h1[k], P[kOffW2 + k * kHidden + j], acc);
    h2[j] = fmaxf(acc, 0.f);
  }
  float best = 3.0e38f;
  int v = -1;
  for (int o = 0; o < kOut; ++o) {
    float acc = P[kOffB3 + o];
    for (int k = 0; k < kHidden; ++k) acc = fmaf(h2[k], P[kOffW3 + k * kOut + o], acc);
    if (((allowed >> o) & 1) && acc < best) {
      best = acc;
      v = o;
    }
  }
  choice[row] = v;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes); }
  float* f() const { return (float*)p; }
  int* i() const { return (int*)p; }
};

static size_t smem_bytes() { return sizeof(MlpSmem); }

static int prep_kernel() {
  cudaError_t e = cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_bytes());
  return cuda_status(e);
}

// grad = dL/dP on rows idx[0..n) (or 0..n); loss written to *dloss (device).
static int fwd_bwd(const float* dP, const float* dX, const float* dT, const float* dM, const int* didx, int n,
                   float inv_cnt, float* dparts, float* dlossp, float* dgrad, float* dloss, cudaStream_t s) {
  const int nblk = (n + kRows - 1) / kRows;
  k_mlp_fwd_bwd<<<nblk, kTBlock, smem_bytes(), s>>>(dP, dX, dT, dM, didx, n, inv_cnt, dparts, dlossp);
  k_mlp_reduce<<<(kParams + 255) / 256, 256, 0, s>>>(dparts, nblk, dgrad, dlossp, dloss);
  return cuda_status(cudaGetLastError());
}

}  // namespace i2

using namespace i2;

#define I2_CK2(call)                        \
  do {                                      \
    cudaError_t e_ = (call);                \
    if (e_ != cudaSuccess) {                \
      cudaGetLastError();                   \
      return cuda_status(e_);               \
    }                                       \
  } while (0)

extern "C" {

int i2_mlp_loss_grad(const float* params, const float* X, const float* T, const float* M, int n, float* loss,
                     float* grad) {
  if (!params || !X || !T || !M || n < 1 || !loss || !grad) return I2_ERR_ARG;
  int st = prep_kernel();
  if (st) return st;
  double cnt = 0.0;
  for (long long k = 0; k < (long long)n * kOut; ++k) cnt += M[k];
  if (cnt <= 0) return I2_ERR_ARG;
  const int nblk = (n + kRows - 1) / kRows;
  DevBuf dP, dX, dT, dM, parts, lossp, dg, dl;
  I2_CK2(dP.alloc(sizeof(float) * kParams));
  I2_CK2(dX.alloc(sizeof(float) * (size_t)n * kFeatures));
  I2_CK2(dT.alloc(sizeof(float) * (size_t)n * kOut));
  I2_CK2(dM.alloc(sizeof(float) * (size_t)n * kOut));
  I2_CK2(parts.alloc(sizeof(float) * (size_t)nblk * kParams));
  I2_CK2(lossp.alloc(sizeof(float) * nblk));
  I2_CK2(dg.alloc(sizeof(float) * kParams));
  I2_CK2(dl.alloc(sizeof(float)));
  I2_CK2(cudaMemcpy(dP.p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dX.p, X, sizeof(float) * (size_t)n * kFeatures, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dT.p, T, sizeof(float) * (size_t)n * kOut, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dM.p, M, sizeof(float) * (size_t)n * kOut, cudaMemcpyHostToDevice));
  st = fwd_bwd(dP.f(), dX.f(), dT.f(), dM.f(), nullptr, n, (float)(1.0 / cnt), parts.f(), lossp.f(), dg.f(), dl.f(), 0);
  if (st) return st;
  I2_CK2(cudaMemcpy(grad, dg.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  I2_CK2(cudaMemcpy(loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
  return I2_OK;
}

int i2_mlp_train(float* params, const float* X, const float* T, const float* M, int n, int epochs, int batch,
                 float lr, uint64_t seed, float* final_loss) {
  if (!params || !X || !T || !M || n < 1 || epochs < 0 || batch < 1) return I2_ERR_ARG;
  int st = prep_kernel();
  if (st) return st;
  // Normaliser: column mean and standard deviation of the training features.
  for (int k = 0; k < kFeatures; ++k) {
    double s = 0, s2 = 0;
    for (int r = 0; r < n; ++r) {
      const double v = X[(size_t)r * kFeatures + k];
      s += v;
      s2 += v * v;
    }
    const double mu = s / n;
    const double sd = std::sqrt(std::max(0.0, s2 / n - mu * mu));
    params[kOffMu + k] = (float)mu;
    params[kOffSd + k] = (float)(sd > 1e-6 ? sd : 1.0);
  }
  batch = std::min(batch, n);
  const int nblk = (batch + kRows - 1) / kRows;
  DevBuf dP, dX, dT, dM, parts, lossp, dg, dl, m1, m2, didx, fullparts, fulllossp;
  I2_CK2(dP.alloc(sizeof(float) * kParams));
  I2_CK2(dX.alloc(sizeof(float) * (size_t)n * kFeatures));
  I2_CK2(dT.alloc(sizeof(float) * (size_t)n * kOut));
  I2_CK2(dM.alloc(sizeof(float) * (size_t)n * kOut));
  I2_CK2(parts.alloc(sizeof(float) * (size_t)nblk * kParams));
  I2_CK2(lossp.alloc(sizeof(float) * nblk));
  I2_CK2(dg.alloc(sizeof(float) * kParams));
  I2_CK2(dl.alloc(sizeof(float)));
  I2_CK2(m1.alloc(sizeof(float) * kParams));
  I2_CK2(m2.alloc(sizeof(float) * kParams));
  I2_CK2(didx.alloc(sizeof(int) * (size_t)n));
  I2_CK2(cudaMemcpy(dP.p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dX.p, X, sizeof(float) * (size_t)n * kFeatures, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dT.p, T, sizeof(float) * (size_t)n * kOut, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dM.p, M, sizeof(float) * (size_t)n * kOut, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemset(m1.p, 0, sizeof(float) * kParams));
  I2_CK2(cudaMemset(m2.p, 0, sizeof(float) * kParams));
  // per-row mask counts for the minibatch normalisation
  std::vector<float> rowcnt(n);
  double tot = 0;
  for (int r = 0; r < n; ++r) {
    float c = 0;
    for (int o = 0; o < kOut; ++o) c += M[(size_t)r * kOut + o];
    rowcnt[r] = c;
    tot += c;
  }
  if (tot <= 0) return I2_ERR_ARG;
  std::vector<int> order(n);
  for (int r = 0; r < n; ++r) order[r] = r;
  std::mt19937_64 rng(seed);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  long long step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    I2_CK2(cudaMemcpy(didx.p, order.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
    for (int b0 = 0; b0 < n; b0 += batch) {
      const int nb = std::min(batch, n - b0);
      double cnt = 0;
      for (int r = b0; r < b0 + nb; ++r) cnt += rowcnt[order[r]];
      if (cnt <= 0) continue;
      st = fwd_bwd(dP.f(), dX.f(), dT.f(), dM.f(), didx.i() + b0, nb, (float)(1.0 / cnt), parts.f(), lossp.f(), dg.f(),
                   dl.f(), 0);
      if (st) return st;
      ++step;
      const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
      k_adam<<<(kParams - kOffW1 + 255) / 256, 256>>>(dP.f(), dg.f(), m1.f(), m2.f(), lr, b1, b2, eps, c1, c2);
    }
  }
  I2_CK2(cudaGetLastError());
  I2_CK2(cudaMemcpy(params, dP.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
  if (final_loss) {
    const int fb = (n + kRows - 1) / kRows;
    I2_CK2(fullparts.alloc(sizeof(float) * (size_t)fb * kParams));
    I2_CK2(fulllossp.alloc(sizeof(float) * fb));
    st = fwd_bwd(dP.f(), dX.f(), dT.f(), dM.f(), nullptr, n, (float)(1.0 / tot), fullparts.f(), fulllossp.f(), dg.f(),
                 dl.f(), 0);
    if (st) return st;
    I2_CK2(cudaMemcpy(final_loss, dl.p, sizeof(float), cudaMemcpyDeviceToHost));
  }
  return I2_OK;
}

int i2_mlp_predict(const float* params, const float* X, int n, int allowed_mask, int* choice) {
  if (!params || !X || !choice || n < 1) return I2_ERR_ARG;
  DevBuf dP, dX, dc;
  I2_CK2(dP.alloc(sizeof(float) * kParams));
  I2_CK2(dX.alloc(sizeof(float) * (size_t)n * kFeatures));
  I2_CK2(dc.alloc(sizeof(int) * (size_t)n));
  I2_CK2(cudaMemcpy(dP.p, params, sizeof(float) * kParams, cudaMemcpyHostToDevice));
  I2_CK2(cudaMemcpy(dX.p, X, sizeof(float) * (size_t)n * kFeatures, cudaMemcpyHostToDevice));
  k_mlp_predict<<<(n + 127) / 128, 128>>>(dP.f(), dX.f(), n, allowed_mask, dc.i());
  I2_CK2(cudaGetLastError());
  I2_CK2(cudaMemcpy(choice, dc.p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost));
  return I2_OK;
}

}  // extern "C"
