// Inverse FFT of real seismogram traces, fast form (FP64, FMA).
//
// Computes the same time series as transformFrequencyTime (frequencyTime.f90:
// 55-113): the Hermitian spectrum of bins nf1..nf2, its unnormalised inverse
// transform of length N = ns, then ts(i) = x(ndec*(i-1)+1) * df * fac(i).  The
// reference runs a radix-2 transform with twiddle angles built on the
// single-precision pi (fourierTransform.f90:128-147); this form evaluates the
// exact inverse DFT, which differs from it by about 1e-7 relative.
//
// Real output from a half-length complex transform: with H = N/2,
//   Z_k = (X_k + conj X_{H-k}) + i w^k (X_k - conj X_{H-k}),  w = e^{2 pi i/N},
//   z_n = sum_k Z_k e^{2 pi i kn/H},  x_{2n} = Re z_n,  x_{2n+1} = Im z_n,
// where X_{H-k} stands for X_{k+H} of the Hermitian spectrum.  The H-point
// transform is a Stockham autosort of radix-16 passes (one of radix 2, 4 or 8
// when log2 H is not a multiple of 4): each of the H/16 threads keeps 16
// points in registers per pass and the passes exchange through shared memory.
// One CTA per trace.
#include <cuda_runtime.h>

#include "synth.h"

namespace gem {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 times_i(double2 a) { return make_double2(-a.y, a.x); }

// shared-memory position of point p: one pad element per 16 keeps the strided
// accesses of the passes off a single bank group
__device__ __forceinline__ int pad(int p) { return p + (p >> 4); }

// 4-point inverse DFT in place: out_k = sum_n a_n i^{nk}
__device__ __forceinline__ void dft4(double2& a0, double2& a1, double2& a2, double2& a3) {
  const double2 p = cadd(a0, a2), m = csub(a0, a2), q = cadd(a1, a3), d = times_i(csub(a1, a3));
  a0 = cadd(p, q);
  a2 = csub(p, q);
  a1 = cadd(m, d);
  a3 = csub(m, d);
}

// e^{2 pi i n/16}, n = 0..9 (the exponents r0*k0 of the 4 x 4 split)
__device__ __forceinline__ double2 w16(int n) {
  constexpr double C1 = 0.92387953251128675613, S1 = 0.38268343236508977173, H2 = 0.70710678118654752440;
  switch (n) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(C1, S1);
    case 2: return make_double2(H2, H2);
    case 3: return make_double2(S1, C1);
    case 4: return make_double2(0.0, 1.0);
    case 6: return make_double2(-H2, H2);
    default: return make_double2(-C1, -S1);   // n = 9
  }
}

// 16-point inverse DFT in place (4 x 4: rows r = 4 r1 + r0, outputs k = k0 + 4 k1)
__device__ __forceinline__ void dft16(double2* v) {
#pragma unroll
  for (int r0 = 0; r0 < 4; ++r0) dft4(v[r0], v[4 + r0], v[8 + r0], v[12 + r0]);
  // v[r0 + 4 k0] now holds Y[r0][k0]; twiddle by w16^(r0 k0)
#pragma unroll
  for (int r0 = 1; r0 < 4; ++r0)
#pragma unroll
    for (int k0 = 1; k0 < 4; ++k0) v[r0 + 4 * k0] = cmul(v[r0 + 4 * k0], w16(r0 * k0));
  double2 o[16];
#pragma unroll
  for (int k0 = 0; k0 < 4; ++k0) {
    double2 a0 = v[0 + 4 * k0], a1 = v[1 + 4 * k0], a2 = v[2 + 4 * k0], a3 = v[3 + 4 * k0];
    dft4(a0, a1, a2, a3);
    o[k0] = a0; o[k0 + 4] = a1; o[k0 + 8] = a2; o[k0 + 12] = a3;
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = o[k];
}

__device__ __forceinline__ void dft2(double2* v) {
  const double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

__device__ __forceinline__ void dft8(double2* v) {
  // even/odd split: X_k = E_k + w8^k O_k, X_{k+4} = E_k - w8^k O_k
  double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4(e0, e1, e2, e3);
  dft4(o0, o1, o2, o3);
  constexpr double H2 = 0.70710678118654752440;
  o1 = cmul(o1, make_double2(H2, H2));
  o2 = times_i(o2);
  o3 = cmul(o3, make_double2(-H2, H2));
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int R>
__device__ __forceinline__ void dftR(double2* v) {
  if constexpr (R == 16) dft16(v);
  else if constexpr (R == 8) dft8(v);
  else if constexpr (R == 4) dft4(v[0], v[1], v[2], v[3]);
  else dft2(v);
}

// One Stockham pass of radix R over the H points in shared memory (NS: length of
// the sub-transforms already done).  Each of the H/16 threads runs 16/R
// butterflies.  The last pass hands its 16 results (point indices idx) back.
// twp: the pass's twiddles twp[(r - 1) NS + k] = e^{2 pi i r k / (NS R)}, laid out
// so that the threads of a warp (consecutive k) read consecutive entries.
template <int H, int R, int NS, bool LAST>
__device__ __forceinline__ void stockham_pass(double2* buf, double2* v, int* idx, const double2* __restrict__ twp) {
  constexpr int T = H / 16, NB = 16 / R;
  const int tid = threadIdx.x;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = tid + b * T;
#pragma unroll
    for (int r = 0; r < R; ++r) v[b * R + r] = buf[pad(j + r * (H / R))];
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = tid + b * T;
    const int k = j % NS;
    if (NS > 1) {
      // w^r, r = 1..R-1, of w = e^{2 pi i k/(NS R)}: R = 16 loads w, w^4 and w^8 and forms the
      // others by products (a few ulps; 3 loads in place of 15, the L1 pipe bounds this kernel)
      if constexpr (R == 16) {
        const double2 w1 = twp[k], w4 = twp[3 * NS + k], w8 = twp[7 * NS + k];
        const double2 w2 = cmul(w1, w1), w3 = cmul(w2, w1);
        double2* u = v + b * R;
        u[1] = cmul(u[1], w1); u[2] = cmul(u[2], w2); u[3] = cmul(u[3], w3);
#pragma unroll
        for (int q = 1; q < 4; ++q) {   // rows 4q .. 4q + 3 with base w^{4q}
          const double2 wb = q == 1 ? w4 : (q == 2 ? w8 : cmul(w8, w4));
          u[4 * q] = cmul(u[4 * q], wb);
          u[4 * q + 1] = cmul(u[4 * q + 1], cmul(wb, w1));
          u[4 * q + 2] = cmul(u[4 * q + 2], cmul(wb, w2));
          u[4 * q + 3] = cmul(u[4 * q + 3], cmul(wb, w3));
        }
      } else {
#pragma unroll
        for (int r = 1; r < R; ++r) v[b * R + r] = cmul(v[b * R + r], twp[(r - 1) * NS + k]);
      }
    }
    dftR<R>(v + b * R);
    const int d = (j / NS) * NS * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (LAST) idx[b * R + r] = d + r * NS;
      else buf[pad(d + r * NS)] = v[b * R + r];
    }
  }
  if (!LAST) __syncthreads();
}

}  // namespace

// tw[m] = e^{2 pi i m / N}, m < N, then the pass tables: tw + N + IFFT_TWA for the
// pass (NS 16, R 16) and tw + N + IFFT_TWB for the last pass (NS 256, R H/256),
// entry (r - 1) NS + k = e^{2 pi i r k / (NS R)}.  Both angles are the same double
// as the m = r k N / (NS R) of the full table, so the entries equal tw[m].
__global__ void ifft_fast_twiddles(int N, double2* tw) {
  const int H = N / 2, RB = H / 256;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < N + IFFT_TW_EXTRA; m += blockDim.x * gridDim.x) {
    long long num = 0, den = 1;
    if (m < N) {
      num = m; den = N;
    } else if (m < N + IFFT_TWB) {
      const int a = m - N - IFFT_TWA;
      if (a < 15 * 16) { num = (long long)(a / 16 + 1) * (a % 16); den = 256; }
    } else {
      const int b = m - N - IFFT_TWB;
      if (b < (RB - 1) * 256) { num = (long long)(b / 256 + 1) * (b % 256); den = 256LL * RB; }
    }
    double s, c;
    sincospi(2.0 * (double)num / (double)den, &s, &c);
    tw[m] = make_double2(c, s);
  }
}

template <int H>
__global__ void __launch_bounds__(H / 16, H == 4096 ? 3 : 1) ifft_fast_kernel(SynthDev S, const double2* __restrict__ X,
                                                          const double2* __restrict__ tw,
                                                          const double* __restrict__ fac, float* traces) {
  extern __shared__ double2 buf[];
  constexpr int T = H / 16;
  const int N = 2 * H;
  const int tid = threadIdx.x;
  const long long tr = blockIdx.x;
  const double2* x = X + tr * S.ldx;
  const int lo = S.nf1 - 1, hi = S.nf2 - 1;   // 0-based bins of the spectrum
  double2 v[16];
  int idx[16];
  // ---- pass 0 (radix 16, NS = 1): Z_k formed on the fly, k = tid + r T.  Z_k is
  // zero unless k or H - k is a bin of the band, so a block of T consecutive k
  // outside both ranges skips its loads (a branch uniform over the CTA)
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int k = tid + r * T;
    const int ka = r * T, kb = r * T + T - 1;
    if (!((ka <= hi && kb >= lo) || (H - kb <= hi && H - ka >= lo))) {
      v[r] = make_double2(0.0, 0.0);
      continue;
    }
    const double2 a = (k >= lo && k <= hi) ? x[k] : make_double2(0.0, 0.0);
    const int kk = H - k;
    double2 b = make_double2(0.0, 0.0);
    if (k > 0 && kk >= lo && kk <= hi) { b = x[kk]; b.y = -b.y; }
    const double2 s = cadd(a, b), d = csub(a, b), w = tw[k];
    // Z = s + i w d
    v[r] = make_double2(s.x - w.y * d.x - w.x * d.y, s.y + w.x * d.x - w.y * d.y);
  }
  dft16(v);
#pragma unroll
  for (int r = 0; r < 16; ++r) buf[pad(tid * 16 + r)] = v[r];
  __syncthreads();
  // ---- remaining passes
  if constexpr (H == 256) {
    stockham_pass<H, 16, 16, true>(buf, v, idx, tw + N + IFFT_TWA);
  } else if constexpr (H == 512) {
    stockham_pass<H, 16, 16, false>(buf, v, idx, tw + N + IFFT_TWA);
    stockham_pass<H, 2, 256, true>(buf, v, idx, tw + N + IFFT_TWB);
  } else if constexpr (H == 1024) {
    stockham_pass<H, 16, 16, false>(buf, v, idx, tw + N + IFFT_TWA);
    stockham_pass<H, 4, 256, true>(buf, v, idx, tw + N + IFFT_TWB);
  } else if constexpr (H == 2048) {
    stockham_pass<H, 16, 16, false>(buf, v, idx, tw + N + IFFT_TWA);
    stockham_pass<H, 8, 256, true>(buf, v, idx, tw + N + IFFT_TWB);
  } else {
    static_assert(H == 4096, "supported half lengths: 256..4096");
    stockham_pass<H, 16, 16, false>(buf, v, idx, tw + N + IFFT_TWA);
    stockham_pass<H, 16, 256, true>(buf, v, idx, tw + N + IFFT_TWB);
  }
  // ---- x_{2n} = Re z_n, x_{2n+1} = Im z_n; ts(i) = x(ndec i) df fac(i)
  float* out = traces + tr * S.nsamp;
  const int ndec = S.ndec;
  if constexpr (H == 4096) {
    // the last pass leaves thread tid the points n = tid + 256 q: samples 2 tid + 512 q (+1), whose factors are
    // df fac(2 tid) expo^(512 q) (+1), formed by products with fac(512) = expo^512 instead of 32 table loads
    // (the table is the running product expo^i; the products differ from it by a few ulps of a double)
    if (ndec == 1 && S.nsamp > 512) {
      const double2 f01 = *reinterpret_cast<const double2*>(fac + 2 * tid);
      const double ratio = fac[512];
      double g0 = S.df * f01.x, g1 = S.df * f01.y;
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int t0 = 2 * tid + 512 * q, t1 = t0 + 1;
        if (t1 < S.nsamp) *reinterpret_cast<float2*>(out + t0) = make_float2((float)(v[q].x * g0), (float)(v[q].y * g1));
        else if (t0 < S.nsamp) out[t0] = (float)(v[q].x * g0);
        g0 *= ratio;
        g1 *= ratio;
      }
      return;
    }
  }
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int n = idx[q];
    const int t0 = 2 * n, t1 = 2 * n + 1;
    if (ndec == 1) {
      if (t1 < S.nsamp) {
        const double2 f = *reinterpret_cast<const double2*>(fac + t0);   // t0 even: 16-byte aligned
        *reinterpret_cast<float2*>(out + t0) = make_float2((float)(v[q].x * S.df * f.x), (float)(v[q].y * S.df * f.y));
      } else if (t0 < S.nsamp) {
        out[t0] = (float)(v[q].x * S.df * fac[t0]);
      }
    } else {
      if (t0 % ndec == 0 && t0 / ndec < S.nsamp) out[t0 / ndec] = (float)(v[q].x * S.df * fac[t0 / ndec]);
      if (t1 % ndec == 0 && t1 / ndec < S.nsamp) out[t1 / ndec] = (float)(v[q].y * S.df * fac[t1 / ndec]);
    }
  }
}

// Launch: ns in 512..8192.  tw: the ns + IFFT_TW_EXTRA twiddles of ifft_fast_twiddles; fac: nsamp factors.
cudaError_t ifft_fast_launch(const SynthDev& S, long long ntr, const double2* X, const double2* tw, const double* fac,
                             float* traces, cudaStream_t st) {
  const int H = S.ns / 2;
  const size_t smem = (size_t)(H + H / 16) * sizeof(double2);
  auto go = [&](auto kern, int threads) -> cudaError_t {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)   // all of the unified L1 as shared memory: more CTAs of the longest transforms per SM
      e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)ntr, threads, smem, st>>>(S, X, tw, fac, traces);
    return cudaGetLastError();
  };
  switch (H) {
    case 256: return go(ifft_fast_kernel<256>, 16);
    case 512: return go(ifft_fast_kernel<512>, 32);
    case 1024: return go(ifft_fast_kernel<1024>, 64);
    case 2048: return go(ifft_fast_kernel<2048>, 128);
    case 4096: return go(ifft_fast_kernel<4096>, 256);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t ifft_fast_twiddles_launch(int N, double2* tw, cudaStream_t st) {
  ifft_fast_twiddles<<<(N + IFFT_TW_EXTRA + 255) / 256, 256, 0, st>>>(N, tw);
  return cudaGetLastError();
}

}  // namespace gem
