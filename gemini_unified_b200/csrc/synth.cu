// Synthetic seismograms from FK spectra (phase 2 of the hot path).
//
// Reference: computeSyntheticSeismograms.f90:311-414 (station loop),
// displacementSpectra.f90:49-113, harmonicDegreeSums.f90:231-369,
// legendreFunctions.f90:48-157, singleFrequencyDisplacement.f90:108-125,
// eventFilter.f90:40-83, butterworthFilter.f90:49-96, axesRotation.f90:560-568,
// frequencyTime.f90:55-113, fourierTransform.f90:118-192.
//
// The station loop of the reference evaluates, per station and frequency, 14
// (moment tensor) or 7 (single force, harmonicDegreeSums.f90:110-171,
// singleFrequencyDisplacement.f90:35-46) dot products of length nwn(f).  Here
// all stations are batched: for each of
// the 8 Legendre table kinds the sums form one matrix product
//     C[(f, sum, re/im), station] = sum_l A[(f, sum, re/im), l] * T[l, station]
// with A holding the FK coefficients times (2l+1)/4pi, the degree factor and
// the cos^2 taper (zero beyond nwn(f)), and T the Legendre table.  The
// products run as tiled FP64 kernels; ZRT assembly, filters, rotation and the
// inverse FFT follow per trace.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/gemini_fk.h"
#include "gem_device.cuh"
#include "synth.h"

namespace gem {

// table kinds: 0 plm0 1 plm1 2 plm2 3 dpdt0 4 dpdt1 5 dpdt2 6 pdst1 7 pdst2
// sums k of source type t (first index: 0 single force, k = 1..7,
// harmonicDegreeSums.f90:110-171; 1 moment tensor, k = 1..14, :297-351):
// kind, first l, factor, FK column (0-based offset of (component, jump),
// greenFKSpectra.f90:204-212, with 2 spheroidal jumps for forces and 4 for moments)
__constant__ int c_sum_kind[2][14] = {{0, 1, 3, 4, 6, 4, 6}, {0, 0, 1, 2, 3, 3, 4, 5, 6, 7, 4, 5, 6, 7}};
__constant__ int c_sum_l0[2][14] = {{0, 1, 1, 1, 1, 1, 1}, {0, 0, 1, 2, 1, 1, 1, 2, 1, 2, 1, 2, 1, 2}};
__constant__ double c_sum_fac[2][14] = {{0, -2, 0, -2, -2, 2, 2}, {0, 0, 2, 2, 0, 0, 2, 2, 2, 4, 2, -2, 2, -4}};
__constant__ int c_sum_col[2][14] = {{0, 1, 2, 3, 4, 4, 3}, {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 8, 9, 6, 7}};
// sums of each source type and sums per table kind (host copies of the tables above)
constexpr int SUMS_OF_TYPE[2] = {7, 14};
constexpr int SUMS_PER_KIND[2][8] = {{1, 1, 0, 1, 2, 0, 2, 0}, {2, 1, 1, 2, 2, 2, 2, 2}};

// rank of sum k among the sums of its table kind: its row pair within the kind
__device__ __forceinline__ int sum_rank(int t, int k) {
  const int kind = c_sum_kind[t][k];
  int s = 0;
  for (int q = 0; q < k; ++q) s += c_sum_kind[t][q] == kind;
  return s;
}

// ---------------------------------------------------------------------------
//  Legendre tables (legendreFunctions.f90:48-157), one thread per (station, m)
//  tab[(kind * lcap + l) * nsta + sta]
// ---------------------------------------------------------------------------
__global__ void legendre_kernel(int nsta, int lmax, int lcap, const double* __restrict__ theta, double* tab) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nsta * 3) return;
  int sta = idx % nsta, m = idx / nsta;
  double ct = cos(theta[sta]), st = sin(theta[sta]);
  bool atpoles = !(st > 0.0);
  auto T = [&](int kind, int l) -> double& { return tab[((long long)kind * lcap + l) * nsta + sta]; };
  const int kp = m, kd = 3 + m, ks = m >= 1 ? 5 + m : -1;   // plm, dpdt, pdst kinds of this m
  double pmm = 1.0, fact = 1.0;
  for (int j = 1; j <= m; ++j) { pmm = pmm * fact * st; fact = fact + 2.0; }
  double rst = 1.0 / st;
  int isct = ct >= 0.0 ? 1 : -1;
  double pl2 = 0.0, pl1 = 0.0;
  for (int l = 0; l <= lmax; ++l) {
    double p;
    if (l < m) p = 0.0;
    else if (l == m) p = pmm;
    else if (l == m + 1) p = ct * (double)(2 * m + 1) * pmm;
    else p = (ct * (double)(2 * l - 1) * pl1 - (double)(l + m - 1) * pl2) / (double)(l - m);
    double dp = 0.0, ps = 0.0;
    if (!atpoles) {
      if (l == m) dp = (double)m * ct * p * rst;
      else if (l > m) dp = ((double)l * ct * p - (double)(l + m) * pl1) * rst;
      if (m >= 1 && l >= m) ps = p * rst;
    } else {
      long long sg = 1;
      if (m == 1) { for (int i = 0; i < l; ++i) sg *= isct; dp = 0.5 * (double)((long long)l * (l + 1) * sg); }
      if (m == 1 && l >= 1) { long long s2 = sg * isct; ps = 0.5 * (double)((long long)l * (l + 1) * s2); }
    }
    T(kp, l) = p;
    T(kd, l) = dp;
    if (ks >= 0) T(ks, l) = ps;
    pl2 = pl1;
    pl1 = p;
  }
}

// ---------------------------------------------------------------------------
//  Coefficient matrices A_kind[row][l], row = 2*(slot*nsk + s) + re/im where s
//  runs over the sums of that kind (harmonicDegreeSums.f90:238-351,356-369).
//  A layout: A[kind][row][lcap]; rowoff[kind], nsk[kind] describe the rows.
// ---------------------------------------------------------------------------
__global__ void coef_kernel(SynthDev S, const float* __restrict__ gr, const float* __restrict__ gi, double* A) {
  long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = S.nf2 - S.nf1 + 1;
  const int t = S.istyp, nsum = S.nsum;
  if (idx >= (long long)nf * nsum * S.lcap) return;
  int l = (int)(idx % S.lcap);
  int k = (int)((idx / S.lcap) % nsum);
  int slot = (int)(idx / ((long long)S.lcap * nsum));
  const int jf = S.nf1 + slot;
  const int nwn = S.nwn[jf - 1];
  const int kind = c_sum_kind[t][k];
  long long row = 2LL * ((long long)slot * S.nsk[kind] + sum_rank(t, k));
  double* Ar = A + (long long)S.aoff[kind] + row * S.lcap;
  double* Ai = Ar + S.lcap;
  double vr = 0.0, vi = 0.0;
  const int lmaxf = nwn - 1;
  if (l >= c_sum_l0[t][k] && l <= lmaxf) {
    // cos^2 taper of this frequency (harmonicDegreeSums.f90:356-369), TAPFRAC = 0.2
    const double tapfrac = 0.2;
    int jt = (int)floor((double)lmaxf * (1.0 - tapfrac) + 0.5);
    jt = jt < lmaxf ? jt : lmaxf;
    jt = jt > 1 ? jt : 1;
    double tap = 1.0;
    if (l >= jt) {
      double c1 = (double)lmaxf * tapfrac * 2.0 / PI_F;
      double c2 = (1.0 - tapfrac) / tapfrac * 0.5 * PI_F;
      double c = cos((double)(float)l / c1 - c2);
      tap = c * c;
    }
    const long long o = (long long)S.col_off[c_sum_col[t][k]] * S.nkf + S.koff[slot] + l;
    double g_r = (double)gr[o], g_i = (double)gi[o];
    double w = 1.0;
    double fac = c_sum_fac[t][k];
    if (fac != 0.0) w = fac / (double)(float)(l * (l + 1));
    double sc = w * (2.0 * (double)l + 1.0) / (4.0 * PI_F) * tap;
    vr = sc * g_r;
    vi = sc * g_i;
  }
  Ar[l] = vr;
  Ai[l] = vi;
}


// ---------------------------------------------------------------------------
//  Regional mode: wavenumber integrals (wavenumberIntegrals.f90:320-491)
//
//  Integral k of frequency f at distance x is a sum over the wavenumbers j of
//  G_f(j) taper_f(j) kern_k(wn_j, J(wn_j x)) w(j, x) with the weights of the
//  reference's rule: dk for 2 <= j < j3 (trapezoid, kx < 3), dk/2 + F at j3 and
//  2F beyond (Filon, F = (1 - cos x dk)/(x dk x)), times R^2/(2 pi).  The
//  products run as the degree sums do: T[kind][j][sta] holds kern x weight x
//  R^2/(2 pi) for the 8 kernel kinds, the coefficient rows hold G taper sign.
//  What depends on both f and x -- the end of the frequency's wavenumber range
//  and the Neumann (Y) end terms -- is added afterwards per (f, x).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double wn_kernel(int kind, double wn, double b0, double b1, double b2, double re,
                                            double x) {
  switch (kind) {   // moment integrals; force integrals (wavenumberIntegrals.f90:160-168)
    case 0: return wn * b0;                                         // 1, 2;    force 1
    case 1: return 2.0 / re * b1;                                   // 3;       force -2
    case 2: return wn * 2.0 * b2;                                   // 4
    case 3: return wn * (-wn * re) * b1;                            // 5, 6;    force 3
    case 4: return wn * 2.0 * (b0 - b1 / (wn * x));                 // 7, 11;   force -4, 6
    case 5: return wn * 2.0 * wn * re * (b1 - 2.0 * b2 / (wn * x)); // 8, -12
    case 6: return wn * 2.0 * b1 / (wn * x);                        // 9, 13;   force -5, 7
    default: return wn * 4.0 * wn * re * b2 / (wn * x);             // 10, -14
  }
}
// sign of each integral's kernel against its kind's table (forces, moments)
__constant__ double c_wn_sign[2][14] = {{1, -1, 1, -1, -1, 1, 1}, {1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, -1, 1, -1}};

struct WnGeom {   // the rule's geometry at distance xx (wavenumberIntegrals.f90:337-348)
  double x, xdk, F;
  int j3;
};
__device__ __forceinline__ WnGeom wn_geom(double xx, double dwn) {
  WnGeom g;
  g.x = xx < 3.0 / (dwn * 1.e9) ? 3.0 / (dwn * 1.e9) : xx;
  g.j3 = (int)(3.0 / g.x / dwn) + 2;
  g.xdk = g.x * dwn;
  g.F = (1.0 - cos(g.xdk)) / g.xdk / g.x;
  return g;
}
__device__ __forceinline__ double wn_kernel_at(int kind, double wn, double x, double re, bool neumann) {
  const double a = wn * x;
  const double b0 = neumann ? y0(a) : j0(a), b1 = neumann ? y1(a) : j1(a);
  const double b2 = -b0 + 2.0 / a * b1;
  return wn_kernel(kind, wn, b0, b1, b2, re, x);
}

// tab[(kind * lcap + j-1) * nsta + sta], j = 1..lcap (1-based wavenumber index)
__global__ void bessel_tab_kernel(SynthDev S, const double* __restrict__ theta, double* tab) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S.lcap * S.nsta) return;
  const int sta = (int)(idx % S.nsta);
  const int j = (int)(idx / S.nsta) + 1;
  const WnGeom g = wn_geom(theta[sta] * S.rearth, S.dwn);
  double w = 0.0;
  if (j >= 2 && j < g.j3) w = S.dwn;
  else if (j >= 2 && j == g.j3) w = 0.5 * S.dwn + g.F;
  else if (j > g.j3) w = 2.0 * g.F;
  const double scale = S.rearth * S.rearth / (2.0 * PI_F);
  const double wn = (double)(j - 1) * S.dwn;
  double b0 = 0, b1 = 0, b2 = 0;
  if (w != 0.0) { const double a = wn * g.x; b0 = j0(a); b1 = j1(a); b2 = -b0 + 2.0 / a * b1; }
  for (int kind = 0; kind < 8; ++kind) {
    const double v = w != 0.0 ? wn_kernel(kind, wn, b0, b1, b2, S.rearth, g.x) * w * scale : 0.0;
    tab[((long long)kind * S.lcap + (j - 1)) * S.nsta + sta] = v;
  }
}

// cos^2 taper of the wavenumber integrals (wavenumberIntegrals.f90:480-491), 1-based j
__device__ __forceinline__ double wn_taper(int nwn, double dwn, int j) {
  const double tapfrac = 0.2;
  int jt = (int)floor((double)nwn * (1.0 - tapfrac) + 0.5);
  jt = jt < nwn ? jt : nwn;
  jt = jt > 1 ? jt : 1;
  if (j < jt) return 1.0;
  const double c1 = (double)(nwn - 1) * dwn * tapfrac * 2.0 / PI_F;
  const double c2 = (1.0 - tapfrac) / tapfrac * 0.5 * PI_F;
  const double c = cos((double)(j - 1) * dwn / c1 - c2);
  return c * c;
}

// coefficient rows of the integrals, the layout of coef_kernel: sign G taper
__global__ void bessel_coef_kernel(SynthDev S, const float* __restrict__ gr, const float* __restrict__ gi, double* A) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = S.nf2 - S.nf1 + 1;
  const int t = S.istyp, nsum = S.nsum;
  if (idx >= (long long)nf * nsum * S.lcap) return;
  const int jj = (int)(idx % S.lcap);   // j - 1
  const int k = (int)((idx / S.lcap) % nsum);
  const int slot = (int)(idx / ((long long)S.lcap * nsum));
  const int nwn = S.nwn[S.nf1 + slot - 1];
  const int kind = c_sum_kind[t][k];
  const long long row = 2LL * ((long long)slot * S.nsk[kind] + sum_rank(t, k));
  double* Ar = A + (long long)S.aoff[kind] + row * S.lcap;
  double vr = 0.0, vi = 0.0;
  if (jj < nwn) {
    const long long o = (long long)S.col_off[c_sum_col[t][k]] * S.nkf + S.koff[slot] + jj;
    const double tp = wn_taper(nwn, S.dwn, jj + 1) * c_wn_sign[t][k];
    vr = (double)gr[o] * tp;
    vi = (double)gi[o] * tp;
  }
  Ar[jj] = vr;
  Ar[S.lcap + jj] = vi;
}

// end terms per (frequency, integral, station) added to the products C
__global__ void bessel_corr_kernel(SynthDev S, const float* __restrict__ gr, const float* __restrict__ gi,
                                   const double* __restrict__ theta, double* C) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = S.nf2 - S.nf1 + 1;
  const int t = S.istyp, nsum = S.nsum;
  if (idx >= (long long)nf * nsum * S.nsta) return;
  const int sta = (int)(idx % S.nsta);
  const int k = (int)((idx / S.nsta) % nsum);
  const int slot = (int)(idx / ((long long)S.nsta * nsum));
  const int nwn = S.nwn[S.nf1 + slot - 1];
  if (nwn < 2) return;
  const int kind = c_sum_kind[t][k];
  const double re = S.rearth, dwn = S.dwn;
  const WnGeom g = wn_geom(theta[sta] * re, dwn);
  const long long o = (long long)S.col_off[c_sum_col[t][k]] * S.nkf + S.koff[slot];
  const double sg = c_wn_sign[t][k];
  auto G = [&](int j) { return dz{(double)gr[o + j - 1], (double)gi[o + j - 1]}; };
  auto kern = [&](int j) { return sg * wn_kernel_at(kind, (double)(j - 1) * dwn, g.x, re, false); };
  dz corr{0.0, 0.0};
  if (nwn > g.j3) {
    // Filon end at nwn has weight F (the table holds 2F); Neumann terms at both ends
    const double tn = wn_taper(nwn, dwn, nwn), t3 = wn_taper(nwn, dwn, g.j3);
    const double wne = (double)(nwn - 1) * dwn, wn3 = (double)(g.j3 - 1) * dwn;
    const double ybn = sg * wn_kernel_at(kind, wne, g.x, re, true), yb3 = sg * wn_kernel_at(kind, wn3, g.x, re, true);
    corr = corr - (G(nwn) * kern(nwn)) * (tn * g.F);
    corr = corr + ((G(nwn) * ybn) * tn - (G(g.j3) * yb3) * t3) / g.x * (1.0 - sin(g.xdk) / g.xdk);
  } else if (nwn == g.j3) {
    corr = corr - (G(nwn) * kern(nwn)) * (wn_taper(nwn, dwn, nwn) * g.F);   // no Filon part
  } else {
    corr = corr - (G(nwn) * kern(nwn)) * (wn_taper(nwn, dwn, nwn) * 0.5 * dwn);   // trapezoid end
  }
  corr = corr * (re * re / (2.0 * PI_F));
  const long long row = 2LL * ((long long)slot * S.nsk[kind] + sum_rank(t, k));
  double* Ck = C + S.coff[kind];
  Ck[row * S.nsta + sta] += corr.re;
  Ck[(row + 1) * S.nsta + sta] += corr.im;
}

// ---------------------------------------------------------------------------
//  FP64 tiled product C[kind][row][sta] = sum_l A[kind][row][l] * T[kind][l][sta]
//  64x64 output tile per block of 256 threads, 4x4 per thread, K step 16.  Rows
//  2 (slot nsk + rank) + re/im hold zero coefficients from degree
//  nwn[nf1 - 1 + slot] on, so a tile's K loop ends at its largest count (the
//  skipped terms would add exact zeros).
// ---------------------------------------------------------------------------
constexpr int GT_M = 64, GT_N = 64, GT_K = 16;

__global__ void __launch_bounds__(256) sums_gemm_kernel(SynthDev S, const double* __restrict__ A,
                                                        const double* __restrict__ T, double* C) {
  const int kind = blockIdx.z;
  const int M = 2 * (S.nf2 - S.nf1 + 1) * S.nsk[kind];
  const int N = S.nsta;
  const int m0 = blockIdx.y * GT_M, n0 = blockIdx.x * GT_N;
  if (m0 >= M) return;
  int K = 0;
  {
    const int nf = S.nf2 - S.nf1 + 1, s0 = m0 / (2 * S.nsk[kind]);
    const int s1 = min(nf - 1, (m0 + GT_M - 1) / (2 * S.nsk[kind]));
    for (int s = s0; s <= s1; ++s) K = max(K, S.nwn[S.nf1 - 1 + s]);
    K = min(K, S.lmax + 1);
  }
  const double* Ak = A + S.aoff[kind];
  const double* Tk = T + (long long)kind * S.lcap * N;
  double* Ck = C + S.coff[kind];
  __shared__ double As[GT_K][GT_M + 1];
  __shared__ double Bs[GT_K][GT_N];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += GT_K) {
    for (int i = threadIdx.x; i < GT_M * GT_K; i += 256) {
      int mm = i / GT_K, kk = i % GT_K;
      int gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < K) ? Ak[(long long)gm * S.lcap + gk] : 0.0;
    }
    for (int i = threadIdx.x; i < GT_K * GT_N; i += 256) {
      int kk = i / GT_N, nn = i % GT_N;
      int gk = k0 + kk, gn = n0 + nn;
      Bs[kk][nn] = (gk < K && gn < N) ? Tk[(long long)gk * N + gn] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < GT_K; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int gm = m0 + ty * 4 + i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int gn = n0 + tx * 4 + j;
      if (gn < N) Ck[(long long)gm * N + gn] = acc[i][j];
    }
  }
}

// ---------------------------------------------------------------------------
//  ZRT spectra from the sums, filters, velocity, rotation; writes the FFT
//  input of every trace (sta, mt, comp) at bins nf1..nf2 (1-based).
//  X[trace][ldx] complex (double2).  One thread per (station, frequency) of a
//  tile of SP_STA stations x SP_SLOT frequencies: the sums are read along
//  stations (coalesced), and per moment tensor the tile's spectra pass through
//  shared memory so that each trace's SP_SLOT consecutive bins are written as
//  one contiguous run.
// ---------------------------------------------------------------------------
constexpr int SP_STA = 32, SP_SLOT = 16, SP_THREADS = SP_STA * SP_SLOT;
__global__ void __launch_bounds__(SP_THREADS) spectra_kernel(SynthDev S, const double* __restrict__ C,
                                                             const double2* __restrict__ evf,
                                                             const double* __restrict__ phi,
                                                             const double* __restrict__ propdir,
                                                             const double* __restrict__ mt, double2* X) {
  __shared__ double2 tile[3][SP_STA][SP_SLOT + 1];
  const int nf = S.nf2 - S.nf1 + 1;
  const int tx = threadIdx.x % SP_STA, ty = threadIdx.x / SP_STA;
  const int sta0 = blockIdx.x * SP_STA, slot0 = blockIdx.y * SP_SLOT;
  const int sta = min(sta0 + tx, S.nsta - 1), slot = min(slot0 + ty, nf - 1);   // clamped: edge threads compute
  const int jf = S.nf1 + slot;                                                   // a copy that is not written
  const int t = S.istyp;
  dz w[15];
  for (int k = 0; k < S.nsum; ++k) {
    int kind = c_sum_kind[t][k];
    long long row = 2LL * ((long long)slot * S.nsk[kind] + sum_rank(t, k));
    const double* Ck = C + S.coff[kind];
    w[k + 1] = dz{Ck[row * S.nsta + sta], Ck[(row + 1) * S.nsta + sta]};
  }
  const double ph = phi[sta];
  const double sphi = sin(ph), cphi = cos(ph);
  const double s2phi = sin(2.0 * ph), c2phi = cos(2.0 * ph);
  const double ca = cos(propdir[sta]), sa = sin(propdir[sta]);
  const dz ci{0.0, 1.0};
  const dz ef = dz{evf[jf].x, evf[jf].y};
  const double tred = S.tred_sta ? S.tred_sta[sta] : S.tred;
  dz tsf = zexp_dev(((ci * TWO_PI_F) * (double)(jf - 1)) * S.df * tred) * exp(S.sigma * tred);
  for (int im = 0; im < S.nmt; ++im) {
    dz z[3];
    if (t == 1) {   // momentSingleFrequencyDisplacement (singleFrequencyDisplacement.f90:108-125)
      const double* m = mt + im * 6;
      double t1 = m[3] * cphi + m[4] * sphi;
      double t2 = (m[2] - m[1]) * c2phi - 2.0 * m[5] * s2phi;
      double t3 = m[4] * cphi - m[3] * sphi;
      double t4 = (m[2] - m[1]) * s2phi + 2.0 * m[5] * c2phi;
      z[0] = w[1] * m[0] + w[2] * (m[1] + m[2]) + w[3] * t1 + w[4] * t2;
      z[1] = w[5] * m[0] + w[6] * (m[1] + m[2]) + (w[7] + w[9]) * t1 + (w[8] + w[10]) * t2;
      z[2] = (w[11] + w[13]) * t3 + (w[12] + w[14]) * t4;
    } else {        // forceSingleFrequencyDisplacement (singleFrequencyDisplacement.f90:35-46), (Fr, Ft, Ff)
      const double* f = mt + im * 3;
      const double fh = f[1] * cphi + f[2] * sphi;
      z[0] = w[1] * f[0] + w[2] * fh;
      z[1] = w[3] * f[0] + (w[4] + w[5]) * fh;
      z[2] = (w[6] + w[7]) * (f[1] * sphi - f[2] * cphi);
    }
    for (int c = 0; c < 3; ++c) {
      dz sf{1.0, 0.0};   // station filter (computeSyntheticSeismograms.f90:361-363), unit by default
      if (S.stafil) {
        const double2 q = S.stafil[((long long)sta * 3 + c) * S.nf2 + (jf - 1)];
        sf = dz{q.x, q.y};
      }
      z[c] = ((z[c] * ef) * sf) * tsf;
    }
    if (S.velocity) {
      dz zom{TWO_PI_F * (double)(jf - 1) * S.df, -S.sigma};
      for (int c = 0; c < 3; ++c) z[c] = (z[c] * ci) * zom;
    }
    dz ue = sa * z[1] + ca * z[2];
    dz un = (-ca) * z[1] + sa * z[2];
    dz out[3] = {z[0], un, ue};
    for (int c = 0; c < 3; ++c) tile[c][tx][ty] = make_double2(out[c].re, out[c].im);
    __syncthreads();
    // the tile's 3 SP_STA traces of this moment tensor, SP_SLOT consecutive bins each
    for (int e = threadIdx.x; e < 3 * SP_STA * SP_SLOT; e += SP_THREADS) {
      const int s = e % SP_SLOT, c = (e / SP_SLOT) % 3, r = e / (3 * SP_SLOT);
      if (sta0 + r < S.nsta && slot0 + s < nf) {
        const long long tr = ((long long)(sta0 + r) * S.nmt + im) * 3 + c;
        X[tr * S.ldx + (S.nf1 - 1 + slot0 + s)] = tile[c][r][s];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
//  Inverse FFT of one trace per block (frequencyTime.f90:55-113,
//  fourierTransform.f90:118-192): Hermitian fill, radix-2 decimation in
//  frequency with the reference's twiddles (host table), bit reversal,
//  ts = Re * df * exp(sigma t).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) ifft_kernel(SynthDev S, const double2* __restrict__ X,
                                                   const double2* __restrict__ tw, const double* __restrict__ fac,
                                                   float* traces) {
  extern __shared__ double2 buf[];
  const int ns = S.ns, nslog = S.nslog;
  const long long tr = blockIdx.x;
  const double2* x = X + tr * S.ldx;
  // bins 1..nf2 (1-based index i <-> frequency (i-1) df); zero below nf1 and above nf2
  for (int i = threadIdx.x; i < ns; i += blockDim.x) {
    int i1 = i + 1;   // 1-based
    double2 v = make_double2(0.0, 0.0);
    if (i1 <= ns / 2 + 1) {
      if (i1 >= S.nf1 && i1 <= S.nf2) v = x[i];
    } else {
      int j1 = ns - i1 + 2;
      if (j1 >= S.nf1 && j1 <= S.nf2) { double2 u = x[j1 - 1]; v = make_double2(u.x, -u.y); }
    }
    buf[i] = v;
  }
  __syncthreads();
  // stages m = 1..nslog: nar = 2^(m-1) groups of length lar = ns/nar
  int twoff = 0;
  for (int m = 1; m <= nslog; ++m) {
    const int nar = 1 << (m - 1), lar = ns / nar, larh = lar / 2;
    for (int t = threadIdx.x; t < ns / 2; t += blockDim.x) {
      const int jr = t % larh, nr = t / larh;   // jr 0-based (reference jr-1)
      const int ja = nr * lar + jr, jb = ja + larh;
      const double2 c = tw[twoff + jr];
      double2 a = buf[ja], b = buf[jb];
      double zx = a.x - b.x, zy = a.y - b.y;
      buf[ja] = make_double2(a.x + b.x, a.y + b.y);
      buf[jb] = make_double2(zx * c.x - zy * c.y, zx * c.y + zy * c.x);
    }
    twoff += larh;
    __syncthreads();
  }
  // bit reversal is a permutation: read element rev(i) for output i
  for (int i = threadIdx.x; i < S.nsamp; i += blockDim.x) {
    int src = (int)(__brev((unsigned)(S.ndec * i)) >> (32 - nslog));
    traces[tr * S.nsamp + i] = (float)(buf[src].x * S.df * fac[i]);
  }
}

// Twiddles (cos beta, sin beta), beta = (2 pi_f32 / lar) (jr - 1), of every
// radix-2 stage in the order ifft_kernel reads them (fourierTransform.f90:
// 139-147, is = +1), and fac[i] = expo^i as the reference's running product
// fac = fac*expo (frequencyTime.f90:105-110): one thread keeps that product
// sequential, so its rounding is the reference's.
__global__ void ifft_tables_kernel(int ns, int nslog, int nsamp, double expo, double2* tw, double* fac) {
  const double piz = 2.0 * PI_F;
  int off = 0;
  for (int m = 1; m <= nslog; ++m) {
    const int lar = ns >> (m - 1), larh = lar / 2;
    const double alpha = piz / (double)lar;
    for (int jr = threadIdx.x + blockIdx.x * blockDim.x; jr < larh; jr += blockDim.x * gridDim.x) {
      double sn, cs;
      sincos(alpha * (double)jr, &sn, &cs);
      tw[off + jr] = make_double2(cs, sn);
    }
    off += larh;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double f = 1.0;
    for (int i = 0; i < nsamp; ++i) { fac[i] = f; f = f * expo; }
  }
}

}  // namespace gem

// ===========================================================================
//  Host side
// ===========================================================================
using namespace gem;

namespace {

// convolveWithSourceWavelet (computeSyntheticSeismograms.f90:463-484), one block per trace,
// in place: the trace and the wavelet are staged in shared memory first.  The sum over the
// wavelet runs in double and is stored to single precision after every term, as the
// reference's real f(k).  Samples at and beyond nd (nsamp_true of the station) become 0.
__global__ void __launch_bounds__(256) wavelet_kernel(int nsamp, int nmt, const int* __restrict__ nstrue, int nstf,
                                                      int nhm, double dt, const float* __restrict__ stf,
                                                      float* traces) {
  extern __shared__ float wsm[];
  float* u = wsm;
  float* w = wsm + nsamp;
  const long long tr = blockIdx.x;
  const int sta = (int)(tr / (3LL * nmt));
  const int nd = nstrue ? nstrue[sta] : nsamp;
  float* t = traces + tr * nsamp;
  for (int i = threadIdx.x; i < nsamp; i += blockDim.x) u[i] = t[i];
  for (int i = threadIdx.x; i < nstf; i += blockDim.x) w[i] = stf[i];
  __syncthreads();
  for (int k = threadIdx.x + 1; k <= nsamp; k += blockDim.x) {
    float out = 0.0f;
    if (k <= nd) {
      if (nstf > 0) {
        const int n0 = max(1, k - nd + nhm + 1), n1 = min(k + nhm, nstf);
        for (int n = n0; n <= n1; ++n) out = (float)((double)out + (dt * (double)u[k - (n - nhm)]) * (double)w[n - 1]);
      } else {
        out = u[k - 1];
      }
    }
    t[k - 1] = out;
  }
}

struct SynthBuffers {
  double* tab = nullptr;
  double* A = nullptr;
  double* C = nullptr;
  double2* X = nullptr;
  double2* evf = nullptr;
  double2* tw = nullptr;
  double2* twx = nullptr;   // e^{2 pi i m/ns} of the fast-form transform
  double* fac = nullptr;
  int* nwn = nullptr;
  int* koff = nullptr;
  double *theta = nullptr, *phi = nullptr, *propdir = nullptr, *mt = nullptr;
};

int nint_(double x) { return x >= 0 ? (int)std::floor(x + 0.5) : -(int)std::floor(-x + 0.5); }

// complex Butterworth band-pass at f - i sigma/2pi (butterworthFilter.f90:49-96)
void event_filter(const gem_synth_params* p, std::vector<double2>& h) {
  const int nf1 = p->nf1, nf2 = p->nf2, nf = nf2 - nf1 + 1;
  const double PIF = PI_F, TPF = TWO_PI_F;
  std::vector<dz> hh(nf, dz{1, 0}), hl(nf, dz{1, 0});
  const double fmin = (double)(nf1 - 1) * p->df;
  const dz ci{0.0, 1.0};
  auto cexp_ = [](dz z) { double e = std::exp(z.re); return dz{e * std::cos(z.im), e * std::sin(z.im)}; };
  dz zfna = (fmin - (ci * p->sigma) / TPF) / p->fc_highpass;
  for (int j = 1; j <= p->order_highpass; ++j) {
    dz zfn = zfna;
    dz ep = cexp_(((ci * PIF) * ((double)j - 0.5)) / (double)p->order_highpass);
    for (int i = 0; i < nf; ++i) { hh[i] = (hh[i] * zfn) / (zfn - ep); zfn = zfn + p->df / p->fc_highpass; }
  }
  zfna = (fmin - (ci * p->sigma) / TPF) / p->fc_lowpass;
  for (int j = 1; j <= p->order_lowpass; ++j) {
    dz zfn = zfna;
    dz ep = cexp_(((ci * PIF) * ((double)j - 0.5)) / (double)p->order_lowpass);
    for (int i = 0; i < nf; ++i) { hl[i] = (hl[i] * (-ci)) / (zfn - ep); zfn = zfn + p->df / p->fc_lowpass; }
  }
  h.assign(nf2 + 1, make_double2(0, 0));
  for (int i = 0; i < nf; ++i) { dz v = hh[i] * hl[i]; h[nf1 + i] = make_double2(v.re, v.im); }
}

}  // namespace

namespace gem {
void event_filter_host(const gem_synth_params* p, std::vector<double2>& h) { event_filter(p, h); }

const char* fft_geometry(int nf1, int nf2, double df, int nsamp, double dt, FftGeometry& g) {
  if (nf1 < 1 || nf2 < nf1 || nsamp < 1 || !(df > 0) || !(dt > 0)) return "ifft: invalid frequency range or sampling";
  if (nf2 > IFFT_MAX_NS / 2 || nsamp > IFFT_MAX_NS) return "ifft: FFT length above 8192 (2*nf2 and nsamp must be <= 8192)";
  g.nslog = (int)std::ceil((double)std::log((float)nf2) / std::log(2.0)) + 1;
  g.ns = 1 << g.nslog;
  g.decimated = false;
  if (g.ns <= nsamp) {
    g.ns = nsamp;
    double lb = std::ceil(-std::log(df * dt) / std::log(2.0));
    if (!(lb >= 1.0 && lb <= 13.0)) return "ifft: nsamp * dt * df must be 1 with nsamp a power of two <= 8192";
    g.nslog = (int)lb;
    g.dts = dt;
    g.ndec = 1;
  } else {
    g.decimated = true;
    g.dts = 1.0 / (df * g.ns);
    double r = dt / g.dts;
    if (!(r >= 0.5 && r < 1e6)) return "Non-integer ratio of desired dt and dt defined from frequency spectrum";
    g.ndec = (int)std::floor(r + 0.5);
    if (std::fabs(dt - g.ndec * g.dts) > 1.e-5) return "Non-integer ratio of desired dt and dt defined from frequency spectrum";
  }
  if ((1 << g.nslog) != g.ns) return "ifft: nsamp * dt * df must be 1 with nsamp a power of two <= 8192";
  if ((long long)g.ndec * (nsamp - 1) >= g.ns) return "ifft: nsamp * dt exceeds the period 1/df of the spectrum";
  return nullptr;
}
}  // namespace gem

extern "C" int gem_synth_run_device(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gr,
                                    const float* d_gi, int nsta, const double* theta, const double* phi,
                                    const double* propdir, int nmt, const double* mt, float* d_traces,
                                    void* stream);

namespace {
// Phase-2 run on device FK spectra (d_gr/d_gi: float32 (nkfmax, nsp)), host station/moment
// arrays; o (may be null) holds the per-station options of the station loop.
int synth_run(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gr, const float* d_gi, int nsta,
              const double* theta, const double* phi, const double* propdir, int nmt, const double* mt,
              const gem_synth_station_opts* o, float* d_traces, void* stream) {
  if (!ctx || !p || !nwn || !theta || !phi || !propdir || !mt) return GEM_ERROR;
  const int nstf = o ? o->nstf : 0;
  if (o) {
    if (nstf < 0 || nstf > 8192 || (nstf > 0 && !o->stf))
      return gem_set_error(ctx, "synthetics: the source wavelet needs 1..8192 samples");
    if (p->nsamp > 8192) return gem_set_error(ctx, "synthetics: station options need nsamp <= 8192");
    if (o->nsamp_true)
      for (int i = 0; i < nsta; ++i)
        if (o->nsamp_true[i] < 1 || o->nsamp_true[i] > p->nsamp)
          return gem_set_error(ctx, "synthetics: nsamp_true must be 1..nsamp");
  }
  if (p->istyp != 1 && p->istyp != 0) return gem_set_error(ctx, "synthetics: source type must be 0 (force) or 1 (moment)");
  if (p->global_ != 1 && p->global_ != 0) return gem_set_error(ctx, "synthetics: GLOBAL must be 0 or 1");
  if (p->global_ == 0 && (!(p->dwn > 0) || !(p->rearth > 0)))
    return gem_set_error(ctx, "synthetics: the regional mode needs the wavenumber spacing and the earth radius");
  if (p->istyp == 1 && p->nsp < 10)
    return gem_set_error(ctx, "synthetics: expected the 10 moment spectra U,V (4 jumps) and W (2 jumps)");
  if (p->istyp == 0 && p->nsp < 5)
    return gem_set_error(ctx, "synthetics: expected the 5 force spectra U,V (2 jumps) and W (1 jump)");
  if (nsta < 1 || nmt < 1 || p->nf1 < 2 || p->nf2 < p->nf1 || p->nwnmax < 3) return gem_set_error(ctx, "synthetics: invalid sizes");
  cudaStream_t st = (cudaStream_t)stream;
  // ---- time axis (frequencyTime.f90:55-84)
  FftGeometry fg;
  if (const char* why = fft_geometry(p->nf1, p->nf2, p->df, p->nsamp, p->dt, fg)) return gem_set_error(ctx, why);
  int nslog = fg.nslog, ns = fg.ns, ndec = fg.ndec;
  double dts = fg.dts;
  // ---- layout
  SynthDev S{};
  S.nf1 = p->nf1; S.nf2 = p->nf2; S.nsta = nsta; S.nmt = nmt; S.lmax = p->nwnmax - 1; S.lcap = p->nwnmax;
  S.nkf = p->nkfmax; S.df = p->df; S.sigma = p->sigma; S.tred = p->tred; S.velocity = p->velocity;
  S.dwn = p->dwn; S.rearth = p->rearth;
  S.istyp = p->istyp; S.nsum = SUMS_OF_TYPE[p->istyp];
  const int nfo = p->istyp == 1 ? 6 : 3;   // moment tensor elements or force components per source
  S.ns = ns; S.nslog = nslog; S.nsamp = p->nsamp; S.ndec = ndec; S.ldx = p->nf2;
  const int* nsk_h = SUMS_PER_KIND[p->istyp];
  const int nf = p->nf2 - p->nf1 + 1;
  long long ao = 0, co = 0;
  for (int k = 0; k < 8; ++k) {
    S.nsk[k] = nsk_h[k];
    S.aoff[k] = ao; S.coff[k] = co;
    ao += 2LL * nf * nsk_h[k] * S.lcap;
    co += 2LL * nf * nsk_h[k] * nsta;
  }
  for (int c = 0; c < 10; ++c) S.col_off[c] = c;
  // frequency offsets in the FK slab
  std::vector<int> koff(nf);
  long long kk = 0;
  // the FK file starts at nf1: frequencies below it hold no wavenumbers
  for (int s = 0; s < nf; ++s) { koff[s] = (int)kk; kk += nwn[p->nf1 + s - 1]; }
  if (kk > p->nkfmax) return gem_set_error(ctx, "synthetics: nwn does not fit nkfmax");
  for (int s = 0; s < nf; ++s) if (nwn[p->nf1 + s - 1] > p->nwnmax) return gem_set_error(ctx, "synthetics: nwn > nwnmax");
  // ---- host tables: event filter, twiddles, exp(sigma t)
  std::vector<double2> evf;
  event_filter(p, evf);
  std::vector<double2> tw;
  const double piz = 2.0 * PI_F;
  for (int m = 1; m <= nslog; ++m) {
    int nar = 1 << (m - 1), lar = ns / nar, larh = lar / 2;
    double alpha = piz / (double)lar;
    for (int jr = 1; jr <= larh; ++jr) {
      double beta = alpha * (double)(jr - 1);
      tw.push_back(make_double2(std::cos(beta), std::sin(beta)));
    }
  }
  std::vector<double> fac(p->nsamp);
  double f = 1.0, expo = std::exp(p->sigma * dts);
  for (int i = 0; i < p->nsamp; ++i) { fac[i] = f; f = f * expo; }
  // ---- device buffers
  SynthBuffers b;
  const long long ntr = (long long)nsta * nmt * 3;
  // all buffers of one run in one context-owned allocation, grown on demand
  const bool fast_fft = gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST && ifft_fast_supported(ns);
  const bool o_tred = o && o->tred, o_ns = o && o->nsamp_true, o_sf = o && o->stafilter;
  const size_t sizes[18] = {(size_t)8 * S.lcap * nsta * sizeof(double), (size_t)ao * sizeof(double),
                            (size_t)co * sizeof(double), (size_t)ntr * S.ldx * sizeof(double2),
                            evf.size() * sizeof(double2), tw.size() * sizeof(double2), fac.size() * sizeof(double),
                            (size_t)p->nf2 * sizeof(int), (size_t)nf * sizeof(int), nsta * sizeof(double),
                            nsta * sizeof(double), nsta * sizeof(double), (size_t)nmt * nfo * sizeof(double),
                            fast_fft ? ifft_fast_twiddle_bytes(ns) : 0,
                            o_tred ? nsta * sizeof(double) : 0, o_ns ? nsta * sizeof(int) : 0,
                            o_sf ? (size_t)nsta * 3 * p->nf2 * sizeof(double2) : 0, (size_t)nstf * sizeof(float)};
  size_t total = 0;
  for (size_t z : sizes) total += (z + 255) / 256 * 256;
  char* pool = (char*)gem_ctx_aux(ctx, 4, total);
  if (!pool) return GEM_ERROR;
  void* parts[18];
  for (int i = 0; i < 18; ++i) { parts[i] = sizes[i] ? pool : nullptr; pool += (sizes[i] + 255) / 256 * 256; }
  b.tab = (double*)parts[0]; b.A = (double*)parts[1]; b.C = (double*)parts[2]; b.X = (double2*)parts[3];
  b.evf = (double2*)parts[4]; b.tw = (double2*)parts[5]; b.fac = (double*)parts[6]; b.nwn = (int*)parts[7];
  b.koff = (int*)parts[8]; b.theta = (double*)parts[9]; b.phi = (double*)parts[10]; b.propdir = (double*)parts[11];
  b.mt = (double*)parts[12]; b.twx = (double2*)parts[13];
  cudaMemcpyAsync(b.evf, evf.data(), evf.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.tw, tw.data(), tw.size() * sizeof(double2), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.fac, fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.nwn, nwn, (size_t)p->nf2 * sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.koff, koff.data(), nf * sizeof(int), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.theta, theta, nsta * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.phi, phi, nsta * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.propdir, propdir, nsta * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b.mt, mt, (size_t)nmt * nfo * sizeof(double), cudaMemcpyHostToDevice, st);
  S.nwn = b.nwn; S.koff = b.koff;
  S.tred_sta = o_tred ? (const double*)parts[14] : nullptr;
  S.stafil = o_sf ? (const double2*)parts[16] : nullptr;
  const int* d_nstrue = o_ns ? (const int*)parts[15] : nullptr;
  if (o_tred) cudaMemcpyAsync(parts[14], o->tred, nsta * sizeof(double), cudaMemcpyHostToDevice, st);
  if (o_ns) cudaMemcpyAsync(parts[15], o->nsamp_true, nsta * sizeof(int), cudaMemcpyHostToDevice, st);
  if (o_sf)
    cudaMemcpyAsync(parts[16], o->stafilter, (size_t)nsta * 3 * p->nf2 * sizeof(double2), cudaMemcpyHostToDevice, st);
  if (nstf > 0) cudaMemcpyAsync(parts[17], o->stf, (size_t)nstf * sizeof(float), cudaMemcpyHostToDevice, st);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0); cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  nvtxRangePushA("gem_synth: sums, spectra, inverse FFT");   // profiler range (no cost without a tool)
  long long ncoef = (long long)nf * S.nsum * S.lcap;
  if (p->global_ == 1) {
    if (gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST && legendre_fast_supported(S.lmax))
      legendre_fast_launch(nsta, S.lmax, S.lcap, b.theta, b.tab, st);
    else
      legendre_kernel<<<(nsta * 3 + 127) / 128, 128, 0, st>>>(nsta, S.lmax, S.lcap, b.theta, b.tab);
    coef_kernel<<<(unsigned)((ncoef + 255) / 256), 256, 0, st>>>(S, d_gr, d_gi, b.A);
  } else {
    const long long ntab = (long long)S.lcap * nsta;
    bessel_tab_kernel<<<(unsigned)((ntab + 255) / 256), 256, 0, st>>>(S, b.theta, b.tab);
    bessel_coef_kernel<<<(unsigned)((ncoef + 255) / 256), 256, 0, st>>>(S, d_gr, d_gi, b.A);
  }
  if (gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST) {
    // sliced-integer products on the tensor cores (6 INT8 slices per operand, exact INT32 accumulation)
    const long long mtot = 2LL * nf * S.nsum;
    const TcProblem TP = tc_problem_of(S);
    const size_t wsb = sums_tc_workspace(TP, mtot, nullptr);
    void* ws = gem_ctx_aux(ctx, 3, wsb);
    const char* why = ws ? sums_tc_run(TP, nwn, mtot, b.tab, b.A, b.C, ws, wsb, gem_ctx_tc_wait_ns(ctx), st) : "";
    if (why) {
      nvtxRangePop();
      cudaEventDestroy(e0); cudaEventDestroy(e1);
      return ws ? gem_set_error(ctx, why) : GEM_ERROR;
    }
  } else {
    int mmax = 2 * nf * 2;
    dim3 g((nsta + GT_N - 1) / GT_N, (mmax + GT_M - 1) / GT_M, 8);
    sums_gemm_kernel<<<g, 256, 0, st>>>(S, b.A, b.tab, b.C);
  }
  if (p->global_ == 0) {
    const long long ncorr = (long long)nf * S.nsum * nsta;
    bessel_corr_kernel<<<(unsigned)((ncorr + 255) / 256), 256, 0, st>>>(S, d_gr, d_gi, b.theta, b.C);
  }
  spectra_kernel<<<dim3((unsigned)((nsta + SP_STA - 1) / SP_STA), (unsigned)((nf + SP_SLOT - 1) / SP_SLOT)), SP_THREADS, 0,
                   st>>>(S, b.C, b.evf, b.phi, b.propdir, b.mt, b.X);
  if (fast_fft) {
    ifft_fast_twiddles_launch(ns, b.twx, st);
    ifft_fast_launch(S, ntr, b.X, b.twx, b.fac, d_traces, st);
  } else {
    size_t smem = (size_t)ns * sizeof(double2);
    cudaFuncSetAttribute(ifft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ifft_kernel<<<(unsigned)ntr, 512, smem, st>>>(S, b.X, b.tw, b.fac, d_traces);
  }
  if (o_ns || nstf > 0) {   // source wavelet and samples kept per station
    const size_t smem = (size_t)(p->nsamp + nstf) * sizeof(float);
    const int nhm = o ? (int)std::floor(std::fabs(o->tanf_stf) / p->dt + 0.5) : 0;
    cudaFuncSetAttribute(wavelet_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    wavelet_kernel<<<(unsigned)ntr, 256, smem, st>>>(p->nsamp, nmt, d_nstrue, nstf, nhm, p->dt,
                                                     (const float*)parts[17], d_traces);
  }
  nvtxRangePop();
  cudaEventRecord(e1, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaGetLastError();
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  gem_note_synth_ms(ctx, ms);
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  if (e != cudaSuccess) return gem_set_error(ctx, cudaGetErrorString(e));
  return GEM_OK;
}

int synth_run_host(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gr, const float* gi,
                   int nsta, const double* theta, const double* phi, const double* propdir, int nmt, const double* mt,
                   const gem_synth_station_opts* o, float* traces);
}  // namespace

extern "C" int gem_synth_run_device(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gr,
                                    const float* d_gi, int nsta, const double* theta, const double* phi,
                                    const double* propdir, int nmt, const double* mt, float* d_traces,
                                    void* stream) {
  return synth_run(ctx, p, nwn, d_gr, d_gi, nsta, theta, phi, propdir, nmt, mt, nullptr, d_traces, stream);
}

extern "C" int gem_synth_run_device_opts(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gr,
                                         const float* d_gi, int nsta, const double* theta, const double* phi,
                                         const double* propdir, int nmt, const double* mt,
                                         const gem_synth_station_opts* opts, float* d_traces, void* stream) {
  return synth_run(ctx, p, nwn, d_gr, d_gi, nsta, theta, phi, propdir, nmt, mt, opts, d_traces, stream);
}

extern "C" int gem_synth_run(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gr, const float* gi,
                             int nsta, const double* theta, const double* phi, const double* propdir, int nmt,
                             const double* mt, float* traces) {
  return synth_run_host(ctx, p, nwn, gr, gi, nsta, theta, phi, propdir, nmt, mt, nullptr, traces);
}

extern "C" int gem_synth_run_opts(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gr,
                                  const float* gi, int nsta, const double* theta, const double* phi,
                                  const double* propdir, int nmt, const double* mt,
                                  const gem_synth_station_opts* opts, float* traces) {
  return synth_run_host(ctx, p, nwn, gr, gi, nsta, theta, phi, propdir, nmt, mt, opts, traces);
}

namespace {
int synth_run_host(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gr, const float* gi,
                   int nsta, const double* theta, const double* phi, const double* propdir, int nmt, const double* mt,
                   const gem_synth_station_opts* o, float* traces) {
  if (!ctx || !p || !gr || !gi || !traces) return GEM_ERROR;
  size_t nin = (size_t)p->nkfmax * p->nsp;
  size_t nout = (size_t)nsta * nmt * 3 * p->nsamp;
  if (cudaSetDevice(gem_ctx_device(ctx)) != cudaSuccess) return gem_set_error(ctx, "synthetics: cudaSetDevice failed");
  float* dgr = (float*)gem_ctx_aux(ctx, 5, nin * sizeof(float));
  float* dgi = dgr ? (float*)gem_ctx_aux(ctx, 6, nin * sizeof(float)) : nullptr;
  float* dtr = dgi ? (float*)gem_ctx_aux(ctx, 7, nout * sizeof(float)) : nullptr;
  if (!dtr) return GEM_ERROR;
  int rc = GEM_OK;
  if (cudaMemcpy(dgr, gr, nin * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dgi, gi, nin * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
    rc = gem_set_error(ctx, "synthetics: copy of the FK spectra failed");
  }
  if (rc != GEM_OK) return rc;
  // Into pinned host memory the traces of a group of stations travel while the
  // next group is computed; otherwise all stations at once, then one copy.
  cudaPointerAttributes pa{};
  const bool pinned = cudaPointerGetAttributes(&pa, traces) == cudaSuccess && pa.type == cudaMemoryTypeHost;
  cudaGetLastError();   // clear the error state of a failed query (pageable memory on some drivers)
  const int ngroups = (pinned && nsta >= 1024) ? 4 : 1;
  if (ngroups == 1) {
    rc = synth_run(ctx, p, nwn, dgr, dgi, nsta, theta, phi, propdir, nmt, mt, o, dtr, nullptr);
    if (rc == GEM_OK && cudaMemcpy(traces, dtr, nout * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = gem_set_error(ctx, "synthetics: copy of the traces failed");
    return rc;
  }
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess)
    return gem_set_error(ctx, "synthetics: copy stream creation failed");
  const size_t per_sta = (size_t)nmt * 3 * p->nsamp;
  double ms_sum = 0.0;
  for (int g = 0; g < ngroups && rc == GEM_OK; ++g) {
    const int s0 = (int)((long long)nsta * g / ngroups), s1 = (int)((long long)nsta * (g + 1) / ngroups);
    gem_synth_station_opts og{};
    const gem_synth_station_opts* op = nullptr;
    if (o) {
      og = *o;
      if (o->tred) og.tred = o->tred + s0;
      if (o->nsamp_true) og.nsamp_true = o->nsamp_true + s0;
      if (o->stafilter) og.stafilter = o->stafilter + (size_t)s0 * 3 * p->nf2 * 2;
      op = &og;
    }
    rc = synth_run(ctx, p, nwn, dgr, dgi, s1 - s0, theta + s0, phi + s0, propdir + s0, nmt, mt, op,
                   dtr + (size_t)s0 * per_sta, nullptr);
    gem_stats stt;
    if (rc == GEM_OK && gem_stats_get(ctx, &stt) == GEM_OK) ms_sum += stt.synth_ms;
    if (rc == GEM_OK &&
        cudaMemcpyAsync(traces + (size_t)s0 * per_sta, dtr + (size_t)s0 * per_sta, (size_t)(s1 - s0) * per_sta *
                        sizeof(float), cudaMemcpyDeviceToHost, cs) != cudaSuccess)
      rc = gem_set_error(ctx, "synthetics: copy of the traces failed");
  }
  if (cudaStreamSynchronize(cs) != cudaSuccess && rc == GEM_OK) rc = gem_set_error(ctx, "synthetics: copy of the traces failed");
  cudaStreamDestroy(cs);
  gem_note_synth_ms(ctx, (float)ms_sum);   // device time of all groups
  return rc;
}
}  // namespace

// ---------------------------------------------------------------------------
//  Batched transformFrequencyTime on device buffers (frequencyTime.f90:55-113)
// ---------------------------------------------------------------------------
extern "C" int gem_ifft_run_device(gem_ctx* ctx, int nf1, int nf2, double df, double sigma, int ntr,
                                   const double* d_sp, long long ldsp, int nsamp, double dt, float* d_ts,
                                   void* stream) {
  if (!ctx) return GEM_ERROR;
  if (!d_sp || !d_ts) return gem_set_error(ctx, "ifft: null spectrum or time-series buffer");
  if (ntr < 1 || ldsp < nf2) return gem_set_error(ctx, "ifft: need ntr >= 1 and ldsp >= nf2");
  FftGeometry g;
  if (const char* why = fft_geometry(nf1, nf2, df, nsamp, dt, g)) return gem_set_error(ctx, why);
  if (cudaSetDevice(gem_ctx_device(ctx)) != cudaSuccess) return gem_set_error(ctx, "ifft: cudaSetDevice failed");
  const bool fast = gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST && ifft_fast_supported(g.ns);
  const size_t tbytes = ifft_table_bytes(g.ns, nsamp);
  char* tab = (char*)gem_ctx_aux(ctx, 0, tbytes + (fast ? ifft_fast_twiddle_bytes(g.ns) + 16 : 0));
  if (!tab) return GEM_ERROR;
  double2* tw = (double2*)tab;
  double* fac = (double*)(tab + (size_t)g.ns * sizeof(double2));
  cudaStream_t st = (cudaStream_t)stream;
  SynthDev S{};
  S.nf1 = nf1; S.nf2 = nf2; S.ns = g.ns; S.nslog = g.nslog; S.nsamp = nsamp; S.ndec = g.ndec; S.df = df;
  S.sigma = sigma; S.ldx = ldsp;
  const double expo = std::exp(sigma * g.dts);
  ifft_tables_kernel<<<8, 256, 0, st>>>(g.ns, g.nslog, nsamp, expo, tw, fac);
  if (fast) {
    double2* twx = (double2*)(tab + (tbytes + 15) / 16 * 16);
    ifft_fast_twiddles_launch(g.ns, twx, st);
    ifft_fast_launch(S, ntr, (const double2*)d_sp, twx, fac, d_ts, st);
  } else {
    const size_t smem = (size_t)g.ns * sizeof(double2);
    cudaFuncSetAttribute(ifft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    ifft_kernel<<<(unsigned)ntr, IFFT_THREADS, smem, st>>>(S, (const double2*)d_sp, tw, fac, d_ts);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return gem_set_error(ctx, cudaGetErrorString(e));
  if (g.decimated) {
    gem_set_error(ctx, "Downsampling to less than 1./(2*fny) requested");
    return GEM_WARNING;
  }
  return GEM_OK;
}

extern "C" int gem_ifft_run(gem_ctx* ctx, int nf1, int nf2, double df, double sigma, int ntr, const double* sp,
                            long long ldsp, int nsamp, double dt, float* ts) {
  if (!ctx) return GEM_ERROR;
  if (!sp || !ts) return gem_set_error(ctx, "ifft: null spectrum or time-series buffer");
  if (ntr < 1 || ldsp < nf2 || nsamp < 1) return gem_set_error(ctx, "ifft: need ntr >= 1, ldsp >= nf2, nsamp >= 1");
  if (cudaSetDevice(gem_ctx_device(ctx)) != cudaSuccess) return gem_set_error(ctx, "ifft: cudaSetDevice failed");
  const size_t nin = (size_t)ntr * ldsp * 2 * sizeof(double), nout = (size_t)ntr * nsamp * sizeof(float);
  void* din = gem_ctx_aux(ctx, 1, nin);
  if (!din) return GEM_ERROR;
  void* dout = gem_ctx_aux(ctx, 2, nout);
  if (!dout) return GEM_ERROR;
  if (cudaMemcpy(din, sp, nin, cudaMemcpyHostToDevice) != cudaSuccess)
    return gem_set_error(ctx, "ifft: copy of the spectra failed");
  int rc = gem_ifft_run_device(ctx, nf1, nf2, df, sigma, ntr, (const double*)din, ldsp, nsamp, dt, (float*)dout, nullptr);
  if (rc >= GEM_ERROR) return rc;
  if (cudaMemcpy(ts, dout, nout, cudaMemcpyDeviceToHost) != cudaSuccess)
    return gem_set_error(ctx, "ifft: copy of the time series failed");
  return rc;
}
