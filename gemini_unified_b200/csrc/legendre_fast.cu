// Legendre tables of the fast form (legendreFunctions.f90:48-157).
//
// Same tables as legendre_kernel (synth.cu): tab[(kind * lcap + l) * nsta + sta]
// with kinds plm_m (m), dP/dtheta (3 + m) and P/sin(theta) (5 + m), one thread
// per (station, m) running the upward recurrence in l.  The plain kernel divides
// by (l - m) at every degree, which puts a software FP64 division on the
// dependent chain and leaves the few warps of this kernel (3 nsta threads)
// waiting on it.  Here the recurrence is written as
//   p_l = alpha_l p_{l-1} + beta_l p_{l-2},
//   alpha_l = ct (2l - 1) / (l - m),  beta_l = -(l + m - 1) / (l - m),
// with 1/(l - m) read from a shared-memory table, so one FMA per degree sits on
// the chain and the rest is independent work.  The values differ from the plain
// form's by rounding only (relative 1e-13 at l = 3200: the recurrence is the
// dominant solution and does not amplify them).
#include <cuda_runtime.h>

#include "synth.h"

namespace gem {

namespace {

constexpr int LF_THREADS = 64;

// poles (sin theta = 0): the plain form's special values, rare, kept operation
// for operation (legendreFunctions.f90:116-127)
__device__ void legendre_pole(int m, int lmax, double ct, double st, long long stride, double* tp, double* td,
                              double* ts) {
  double pmm = 1.0, fact = 1.0;
  for (int j = 1; j <= m; ++j) { pmm = pmm * fact * st; fact = fact + 2.0; }
  const int isct = ct >= 0.0 ? 1 : -1;
  double pl2 = 0.0, pl1 = 0.0;
  for (int l = 0; l <= lmax; ++l) {
    double p;
    if (l < m) p = 0.0;
    else if (l == m) p = pmm;
    else if (l == m + 1) p = ct * (double)(2 * m + 1) * pmm;
    else p = (ct * (double)(2 * l - 1) * pl1 - (double)(l + m - 1) * pl2) / (double)(l - m);
    double dp = 0.0, ps = 0.0;
    long long sg = 1;
    if (m == 1) { for (int i = 0; i < l; ++i) sg *= isct; dp = 0.5 * (double)((long long)l * (l + 1) * sg); }
    if (m == 1 && l >= 1) { long long s2 = sg * isct; ps = 0.5 * (double)((long long)l * (l + 1) * s2); }
    tp[l * stride] = p;
    td[l * stride] = dp;
    if (ts) ts[l * stride] = ps;
    pl2 = pl1;
    pl1 = p;
  }
}

__global__ void __launch_bounds__(LF_THREADS) legendre_fast_kernel(int nsta, int lmax, int lcap,
                                                                   const double* __restrict__ theta,
                                                                   double* __restrict__ tab) {
  extern __shared__ double rcp[];   // rcp[n] = 1/n, n = 1..lmax
  for (int n = threadIdx.x + 1; n <= lmax; n += blockDim.x) rcp[n] = 1.0 / (double)n;
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nsta * 3) return;
  const int sta = idx % nsta, m = idx / nsta;
  const double ct = cos(theta[sta]), st = sin(theta[sta]);
  const long long stride = nsta, plane = (long long)lcap * nsta;
  double* tp = tab + (long long)m * plane + sta;
  double* td = tab + (long long)(3 + m) * plane + sta;
  double* ts = m >= 1 ? tab + (long long)(5 + m) * plane + sta : nullptr;
  if (!(st > 0.0)) {
    legendre_pole(m, lmax, ct, st, stride, tp, td, ts);
    return;
  }
  double pmm = 1.0, fact = 1.0;
  for (int j = 1; j <= m; ++j) { pmm = pmm * fact * st; fact = fact + 2.0; }
  const double rst = 1.0 / st;
  long long o = 0;
  for (int l = 0; l < m && l <= lmax; ++l, o += stride) {
    tp[o] = 0.0;
    td[o] = 0.0;
    if (ts) ts[o] = 0.0;
  }
  if (m > lmax) return;
  // l = m
  tp[o] = pmm;
  td[o] = (double)m * ct * pmm * rst;
  if (ts) ts[o] = pmm * rst;
  if (m + 1 > lmax) return;
  o += stride;
  // l = m + 1
  const double p1 = ct * (double)(2 * m + 1) * pmm;
  double dl = (double)(m + 1);
  tp[o] = p1;
  td[o] = fma(dl * ct, p1, -(dl + (double)m) * pmm) * rst;
  if (ts) ts[o] = p1 * rst;
  o += stride;
  double pl2 = pmm, pl1 = p1;
  const double mm1 = (double)(m - 1), md = (double)m;
#pragma unroll 4
  for (int l = m + 2; l <= lmax; ++l, o += stride) {
    dl += 1.0;
    const double r = rcp[l - m];
    const double alpha = ct * fma(2.0, dl, -1.0) * r;
    const double bp = -(dl + mm1) * r * pl2;          // off the chain: pl2 is known a degree early
    const double p = fma(alpha, pl1, bp);
    tp[o] = p;
    td[o] = fma(dl * ct, p, -(dl + md) * pl1) * rst;
    if (ts) ts[o] = p * rst;
    pl2 = pl1;
    pl1 = p;
  }
}

}  // namespace

bool legendre_fast_supported(int lmax) { return (size_t)(lmax + 1) * sizeof(double) <= 200 * 1024; }

cudaError_t legendre_fast_launch(int nsta, int lmax, int lcap, const double* theta, double* tab, cudaStream_t st) {
  const size_t smem = (size_t)(lmax + 1) * sizeof(double);
  if (!legendre_fast_supported(lmax)) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(legendre_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  legendre_fast_kernel<<<(nsta * 3 + LF_THREADS - 1) / LF_THREADS, LF_THREADS, smem, st>>>(nsta, lmax, lcap, theta,
                                                                                          tab);
  return cudaGetLastError();
}

}  // namespace gem
