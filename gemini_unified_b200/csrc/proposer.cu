// Learned step/order proposer of the FK solver (no counterpart in the reference).
//
// A 3-layer MLP of width 64 (tanh) maps per-(item, phase) features to three
// outputs: the predicted work of the phase's integrations with the step-size
// control aiming at attempt 5 and at attempt 7, each as log(work / work at 6),
// and log of the factor that brings the initial step of the initial-value
// formulas (initialValues.f90, spheroidalAdjoint.f90:126-129) to the step the
// control settles on.  Before the phase kernels run, one thread per (item,
// phase) evaluates the network (FP16 weights, FP32 accumulation) and writes
// the order target (the attempt with the least predicted work) and the initial
// step factor, which the solver reads.  The plain Bulirsch-Stoer error control
// still accepts or rejects every step.
//
// Features (PROP_NF = 11), in this order: log10 f, log10(l + 1) / 4,
// horizontal slowness l v0 / (omega R) with v0 = 4 km/s, start radius / R,
// layer of the start radius / number of layers, vp, vs, rho at the knot below
// the start radius (SI / 1e4), one-hot phase (toroidal, spheroidal, adjoint).
// They are standardised with the mean and deviation stored with the weights.
//
// Training: minibatch gradient descent with Adam on a masked mean-squared
// error, run by the kernels of this file: forward and backward of 64 samples
// per CTA with gradients summed per warp and then by atomics, and an Adam update.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/gemini_fk.h"
#include "gem_device.cuh"
#include "proposer.h"

namespace gem {

// layout of the flat parameter vector
struct Net {
  static constexpr int W1 = 0;
  static constexpr int B1 = W1 + PROP_H * PROP_NF;
  static constexpr int W2 = B1 + PROP_H;
  static constexpr int B2 = W2 + PROP_H * PROP_H;
  static constexpr int W3 = B2 + PROP_H;
  static constexpr int B3 = W3 + PROP_NO * PROP_H;
  static constexpr int N = B3 + PROP_NO;
};
static_assert(Net::N == PROP_NPARAM, "parameter count");

// ---------------------------------------------------------------------------
//  Features of (item, phase)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int knot_below(const double* rk, int nk, double r) {
  if (r <= rk[1]) return 1;
  if (r >= rk[nk]) return nk;
  int lo = 1, hi = nk;   // rk ascending, 1-based
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (rk[mid] <= r) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int layer_of(const double* rb, int nlay, double r) {
  int nl = 1;
  while (nl < nlay && r > rb[nl]) ++nl;
  return nl;
}

__device__ void item_features(const PropArgs& A, int k, int ph, float* f) {
  const int2 w = A.items[k];
  const int jf = A.jf[w.x];
  const int l = w.y - 1;
  const double fr = (double)(jf - 1) * A.df;
  const double om = 2.0 * PI_F * fr;
  const double r0 = ph == 0 ? A.rstart[k] : A.rstart[A.nkf + k];
  const int kn = knot_below(A.rk, A.nk, r0);
  f[0] = (float)log10(fmax(fr, 1e-6));
  f[1] = (float)(log10((double)l + 1.0) / 4.0);
  f[2] = (float)fmin((double)l * 4000.0 / fmax(om * A.rearth, 1e-30), 10.0);
  f[3] = (float)(r0 / A.rearth);
  f[4] = (float)layer_of(A.rb, A.nlay, r0) / (float)A.nlay;
  f[5] = A.knot_feat[3 * kn + 0];
  f[6] = A.knot_feat[3 * kn + 1];
  f[7] = A.knot_feat[3 * kn + 2];
  f[8] = ph == 0 ? 1.f : 0.f;
  f[9] = ph == 1 ? 1.f : 0.f;
  f[10] = ph == 2 ? 1.f : 0.f;
}

// raw features of every (phase, item): out[(ph * nitems + k) * PROP_NF + i]
__global__ void prop_features_kernel(PropArgs A, float* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3LL * A.nitems) return;
  const int ph = (int)(t / A.nitems), k = (int)(t % A.nitems);
  float f[PROP_NF];
  item_features(A, k, ph, f);
#pragma unroll
  for (int i = 0; i < PROP_NF; ++i) out[t * PROP_NF + i] = f[i];
}

// ---------------------------------------------------------------------------
//  Inference: FP16 weights, FP32 accumulation, one thread per (item, phase)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void forward_half(const __half* __restrict__ w, const float* __restrict__ norm,
                                             const float* x_raw, float* out) {
  float x[PROP_NF], h1[PROP_H], h2[PROP_H];
#pragma unroll
  for (int i = 0; i < PROP_NF; ++i) x[i] = (x_raw[i] - norm[i]) / norm[PROP_NF + i];
  for (int o = 0; o < PROP_H; ++o) {
    float a = __half2float(w[Net::B1 + o]);
#pragma unroll
    for (int i = 0; i < PROP_NF; ++i) a = fmaf(__half2float(w[Net::W1 + o * PROP_NF + i]), x[i], a);
    h1[o] = tanhf(a);
  }
  for (int o = 0; o < PROP_H; ++o) {
    float a = __half2float(w[Net::B2 + o]);
    const __half* row = w + Net::W2 + o * PROP_H;
#pragma unroll 16
    for (int i = 0; i < PROP_H; ++i) a = fmaf(__half2float(row[i]), h1[i], a);
    h2[o] = tanhf(a);
  }
#pragma unroll
  for (int o = 0; o < PROP_NO; ++o) {
    float a = __half2float(w[Net::B3 + o]);
    const __half* row = w + Net::W3 + o * PROP_H;
#pragma unroll 16
    for (int i = 0; i < PROP_H; ++i) a = fmaf(__half2float(row[i]), h2[i], a);
    out[o] = a;
  }
}

__global__ void __launch_bounds__(128) prop_infer_kernel(PropArgs A, const __half* __restrict__ w,
                                                         const float* __restrict__ norm, signed char* kopt,
                                                         float* hs) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3LL * A.nitems) return;
  const int ph = (int)(t / A.nitems), k = (int)(t % A.nitems);
  float f[PROP_NF], o[PROP_NO];
  item_features(A, k, ph, f);
  forward_half(w, norm, f, o);
  // attempt with the least predicted work; 5 or 7 only with a predicted saving above the margin
  int best = 6;
  if (A.use & PROP_USE_ORDER) {
    float bw = -A.margin;
    if (o[0] < bw) { best = 5; bw = o[0]; }
    if (o[1] < bw) best = 7;
  }
  kopt[(long long)ph * A.nkf + k] = (signed char)best;
  hs[(long long)ph * A.nkf + k] =
      (A.use & PROP_USE_STEP) ? expf(fminf(fmaxf(o[2], -PROP_HS_CLIP), PROP_HS_CLIP)) : 1.f;
}

// ---------------------------------------------------------------------------
//  Training kernels (FP32)
// ---------------------------------------------------------------------------
constexpr int TB = 64;   // samples per CTA

// forward + backward of TB samples; gradients summed into g, the loss into loss[0]
__global__ void __launch_bounds__(TB) prop_grad_kernel(const float* __restrict__ w, const float* __restrict__ X,
                                                       const float* __restrict__ Y, const float* __restrict__ M,
                                                       const int* __restrict__ idx, int n, float inv_wsum, float* g,
                                                       float* loss) {
  __shared__ float sw[Net::N];
  for (int i = threadIdx.x; i < Net::N; i += blockDim.x) sw[i] = w[i];
  __syncthreads();
  const int s = blockIdx.x * TB + threadIdx.x;
  const bool ok = s < n;
  const int row = ok ? idx[s] : 0;
  float x[PROP_NF], h1[PROP_H], h2[PROP_H], d[PROP_NO];
#pragma unroll
  for (int i = 0; i < PROP_NF; ++i) x[i] = ok ? X[(long long)row * PROP_NF + i] : 0.f;
  for (int j = 0; j < PROP_H; ++j) {
    float a = sw[Net::B1 + j];
#pragma unroll
    for (int i = 0; i < PROP_NF; ++i) a = fmaf(sw[Net::W1 + j * PROP_NF + i], x[i], a);
    h1[j] = tanhf(a);
  }
  for (int j = 0; j < PROP_H; ++j) {
    float a = sw[Net::B2 + j];
    for (int i = 0; i < PROP_H; ++i) a = fmaf(sw[Net::W2 + j * PROP_H + i], h1[i], a);
    h2[j] = tanhf(a);
  }
  float l = 0.f;
#pragma unroll
  for (int q = 0; q < PROP_NO; ++q) {
    float a = sw[Net::B3 + q];
    for (int i = 0; i < PROP_H; ++i) a = fmaf(sw[Net::W3 + q * PROP_H + i], h2[i], a);
    const float m = ok ? M[(long long)row * PROP_NO + q] : 0.f;
    const float e = a - (ok ? Y[(long long)row * PROP_NO + q] : 0.f);
    l += m * e * e;
    d[q] = 2.f * m * e * inv_wsum;   // dL/d output
  }
  // every lane takes part (inactive samples contribute 0): warp sums, then one atomic per warp
  auto acc = [&](float* addr, float v) {
#pragma unroll
    for (int o2 = 16; o2 > 0; o2 >>= 1) v += __shfl_down_sync(0xffffffffu, v, o2);
    if ((threadIdx.x & 31) == 0 && v != 0.f) atomicAdd(addr, v);
  };
  acc(loss, ok ? l * inv_wsum : 0.f);
  float dh2[PROP_H];
  for (int i = 0; i < PROP_H; ++i) dh2[i] = 0.f;
#pragma unroll
  for (int q = 0; q < PROP_NO; ++q) {
    acc(g + Net::B3 + q, d[q]);
    for (int i = 0; i < PROP_H; ++i) {
      acc(g + Net::W3 + q * PROP_H + i, d[q] * h2[i]);
      dh2[i] = fmaf(d[q], sw[Net::W3 + q * PROP_H + i], dh2[i]);
    }
  }
  float dh1[PROP_H];
  for (int i = 0; i < PROP_H; ++i) dh1[i] = 0.f;
  for (int j = 0; j < PROP_H; ++j) {
    const float dz = dh2[j] * (1.f - h2[j] * h2[j]);
    acc(g + Net::B2 + j, dz);
    for (int i = 0; i < PROP_H; ++i) {
      acc(g + Net::W2 + j * PROP_H + i, dz * h1[i]);
      dh1[i] = fmaf(dz, sw[Net::W2 + j * PROP_H + i], dh1[i]);
    }
  }
  for (int j = 0; j < PROP_H; ++j) {
    const float dz = dh1[j] * (1.f - h1[j] * h1[j]);
    acc(g + Net::B1 + j, dz);
#pragma unroll
    for (int i = 0; i < PROP_NF; ++i) acc(g + Net::W1 + j * PROP_NF + i, dz * x[i]);
  }
}

__global__ void prop_adam_kernel(float* w, const float* g, float* m, float* v, float lr, float b1, float b2,
                                 float eps, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Net::N) return;
  const float gi = g[i];
  m[i] = b1 * m[i] + (1.f - b1) * gi;
  v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
  w[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
}

cudaError_t prop_features_launch(const PropArgs& A, float* out, cudaStream_t st) {
  prop_features_kernel<<<(unsigned)((3LL * A.nitems + 127) / 128), 128, 0, st>>>(A, out);
  return cudaGetLastError();
}

cudaError_t prop_infer_launch(const PropArgs& A, const __half* w, const float* norm, signed char* kopt, float* hs,
                              cudaStream_t st) {
  prop_infer_kernel<<<(unsigned)((3LL * A.nitems + 127) / 128), 128, 0, st>>>(A, w, norm, kopt, hs);
  return cudaGetLastError();
}

}  // namespace gem

using namespace gem;

namespace {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { cudaFree(p); }
  bool alloc(size_t n) { return cudaMalloc(&p, n) == cudaSuccess; }
};

}  // namespace

extern "C" {

int gem_prop_grad(const float* w, const float* x, const float* y, const float* mask, int n, float* grad, float* loss) {
  if (!w || !x || !y || !mask || !grad || !loss || n < 1) return GEM_ERROR;
  DevBuf dw, dx, dy, dm, di, dg, dl;
  if (!dw.alloc(Net::N * 4) || !dx.alloc((size_t)n * PROP_NF * 4) || !dy.alloc((size_t)n * PROP_NO * 4) ||
      !dm.alloc((size_t)n * PROP_NO * 4) || !di.alloc((size_t)n * 4) || !dg.alloc(Net::N * 4) || !dl.alloc(4))
    return GEM_ERROR;
  std::vector<int> id(n);
  double wsum = 0.0;
  for (int i = 0; i < n; ++i) id[i] = i;
  for (long long i = 0; i < (long long)n * PROP_NO; ++i) wsum += mask[i];
  if (cudaMemcpy(dw.p, w, Net::N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dx.p, x, (size_t)n * PROP_NF * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dy.p, y, (size_t)n * PROP_NO * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dm.p, mask, (size_t)n * PROP_NO * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(di.p, id.data(), (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(dg.p, 0, Net::N * 4) != cudaSuccess || cudaMemset(dl.p, 0, 4) != cudaSuccess)
    return GEM_ERROR;
  prop_grad_kernel<<<(n + TB - 1) / TB, TB>>>((const float*)dw.p, (const float*)dx.p, (const float*)dy.p,
                                              (const float*)dm.p, (const int*)di.p, n,
                                              (float)(1.0 / (wsum > 0 ? wsum : 1.0)), (float*)dg.p, (float*)dl.p);
  if (cudaDeviceSynchronize() != cudaSuccess) return GEM_ERROR;
  if (cudaMemcpy(grad, dg.p, Net::N * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(loss, dl.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return GEM_ERROR;
  return GEM_OK;
}

int gem_prop_train(float* w, const float* x, const float* y, const float* mask, int n, int epochs, int batch,
                   float lr, unsigned seed, float* loss_hist) {
  if (!w || !x || !y || !mask || n < 1 || epochs < 1 || batch < 1) return GEM_ERROR;
  DevBuf dw, dx, dy, dm, di, dg, dl, dmom, dvel;
  if (!dw.alloc(Net::N * 4) || !dx.alloc((size_t)n * PROP_NF * 4) || !dy.alloc((size_t)n * PROP_NO * 4) ||
      !dm.alloc((size_t)n * PROP_NO * 4) || !di.alloc((size_t)n * 4) || !dg.alloc(Net::N * 4) || !dl.alloc(4) ||
      !dmom.alloc(Net::N * 4) || !dvel.alloc(Net::N * 4))
    return GEM_ERROR;
  if (cudaMemcpy(dw.p, w, Net::N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dx.p, x, (size_t)n * PROP_NF * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dy.p, y, (size_t)n * PROP_NO * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dm.p, mask, (size_t)n * PROP_NO * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(dmom.p, 0, Net::N * 4) != cudaSuccess || cudaMemset(dvel.p, 0, Net::N * 4) != cudaSuccess)
    return GEM_ERROR;
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  unsigned long long st = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  auto rnd = [&]() { st = st * 6364136223846793005ULL + 1442695040888963407ULL; return (unsigned)(st >> 33); };
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[(int)(rnd() % (unsigned)(i + 1))]);
    if (cudaMemcpy(di.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice) != cudaSuccess) return GEM_ERROR;
    cudaMemset(dl.p, 0, 4);
    int nb = 0;
    for (int s0 = 0; s0 < n; s0 += batch, ++nb) {
      const int m = std::min(batch, n - s0);
      double wsum = 0.0;
      for (int i = s0; i < s0 + m; ++i)
        for (int q = 0; q < PROP_NO; ++q) wsum += mask[(long long)perm[i] * PROP_NO + q];
      cudaMemset(dg.p, 0, Net::N * 4);
      prop_grad_kernel<<<(m + TB - 1) / TB, TB>>>((const float*)dw.p, (const float*)dx.p, (const float*)dy.p,
                                                  (const float*)dm.p, (const int*)di.p + s0, m,
                                                  (float)(1.0 / (wsum > 0 ? wsum : 1.0)), (float*)dg.p,
                                                  (float*)dl.p);
      ++step;
      prop_adam_kernel<<<(Net::N + 255) / 256, 256>>>((float*)dw.p, (const float*)dg.p, (float*)dmom.p,
                                                      (float*)dvel.p, lr, b1, b2, eps,
                                                      1.f - powf(b1, (float)step), 1.f - powf(b2, (float)step));
    }
    if (loss_hist) {
      float l = 0.f;
      if (cudaMemcpy(&l, dl.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return GEM_ERROR;
      loss_hist[ep] = l / (float)nb;
    }
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return GEM_ERROR;
  if (cudaMemcpy(w, dw.p, Net::N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return GEM_ERROR;
  return GEM_OK;
}

}  // extern "C"
