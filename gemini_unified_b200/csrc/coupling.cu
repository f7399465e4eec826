// Synthetics for SPECFEM coupling on the GPU: displacement (as velocity) and
// traction at the boundary points of a SPECFEM box, from the DSV spectra with
// radial derivatives of the points' node (computeSyntheticsForSpecfemCoupling.f90:
// computeSynthetics :714-793, computeTension :677-705; moment and force sources).
//
//   cpl_legendre_kernel  P_l^m, dP/dtheta, P/sin, d2P/dtheta2, d/dtheta(P/sin)
//                        for m <= 2 at every point (legendreFunctions.f90:48-157)
//   cpl_coef_kernel      coefficient rows (frequency, sum) x degree of each
//                        table kind: taper, (2l+1)/4pi, factor and spectrum
//                        (harmonicDegreeSums.f90:95-369, index map :34-45)
//   cpl_gemm_kernel      the degree sums of every (frequency, sum, point) as one
//                        FP64 tiled product per table kind; with the fast
//                        backend the same 13 products run on the tensor cores
//                        as sliced-INT8 integer products (sums_tc.cu)
//   cpl_point_kernel     displacement and its derivatives, strain, stress, the
//                        rotation to the box frame, traction = stress * n,
//                        event filter, i omega and time shift
//                        (singleFrequencyDisplacement.f90:108-262)
//   gem_ifft_run_device  the six time series of every point
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "synth.h"

namespace gem {
namespace {

constexpr int CPL_NSUM = 42;
constexpr int CPL_NKIND = 13;   // plm m0-2, dpdt m0-2, pdst m1-2, d2pdt2 m0-2, dtpdst m1-2
static_assert(CPL_NKIND <= TC_MAX_KIND, "the tensor-core sums take at most TC_MAX_KIND table kinds");

// per sum: table kind, first degree, factor numerator over l(l+1) (0: none),
// column of its (component, jump) in the DSV spectra U, V, dU/dr, dV/dr (x 4
// jumps), W, dW/dr (x 2 jumps)
struct CplSum { int kind, l0; double fac; int col; };
#define CPL_MOMENT_SUMS {                                   \
    {0, 0, 0.0, 0}, {0, 0, 0.0, 1}, {1, 1, 2.0, 2}, {2, 2, 2.0, 3}, \
    {3, 1, 0.0, 4}, {3, 1, 0.0, 5}, {4, 1, 2.0, 6}, {5, 2, 2.0, 7}, \
    {6, 1, 2.0, 16}, {7, 2, 4.0, 17}, {4, 1, 2.0, 16}, {5, 2, -2.0, 17}, \
    {6, 1, 2.0, 6}, {7, 2, -4.0, 7}, {0, 0, 0.0, 8}, {0, 0, 0.0, 9}, \
    {1, 1, 2.0, 10}, {2, 2, 2.0, 11}, {3, 1, 0.0, 12}, {3, 1, 0.0, 13}, \
    {4, 1, 2.0, 14}, {5, 2, 2.0, 15}, {6, 1, 2.0, 18}, {7, 2, 4.0, 19}, \
    {4, 1, 2.0, 18}, {5, 2, -2.0, 19}, {6, 1, 2.0, 14}, {7, 2, -4.0, 15}, \
    {3, 1, 0.0, 0}, {3, 1, 0.0, 1}, {4, 1, 2.0, 2}, {5, 2, 2.0, 3}, \
    {8, 1, 0.0, 4}, {8, 1, 0.0, 5}, {9, 1, 2.0, 6}, {10, 2, 2.0, 7}, \
    {11, 1, 2.0, 16}, {12, 2, 4.0, 17}, {9, 1, 2.0, 16}, {10, 2, -2.0, 17}, \
    {11, 1, 2.0, 6}, {12, 2, -4.0, 7}}
__constant__ CplSum c_cpl[CPL_NSUM] = CPL_MOMENT_SUMS;
const CplSum h_cpl[CPL_NSUM] = CPL_MOMENT_SUMS;

// the 21 force sums (harmonicDegreeSums.f90:95-167): columns of U, V, dU/dr,
// dV/dr (x 2 jumps), W, dW/dr (1 jump)
#define CPL_FORCE_SUMS {                                    \
    {0, 0, 0.0, 0}, {1, 1, -2.0, 1}, {3, 1, 0.0, 2}, {4, 1, -2.0, 3}, \
    {6, 1, -2.0, 8}, {4, 1, 2.0, 8}, {6, 1, 2.0, 3},        \
    {0, 0, 0.0, 4}, {1, 1, -2.0, 5}, {3, 1, 0.0, 6}, {4, 1, -2.0, 7}, \
    {6, 1, -2.0, 9}, {4, 1, 2.0, 9}, {6, 1, 2.0, 7},        \
    {3, 1, 0.0, 0}, {4, 1, -2.0, 1}, {8, 1, 0.0, 2}, {9, 1, -2.0, 3}, \
    {11, 1, -2.0, 8}, {9, 1, 2.0, 8}, {11, 1, 2.0, 3}}
__constant__ CplSum c_cplf[21] = CPL_FORCE_SUMS;
const CplSum h_cplf[21] = CPL_FORCE_SUMS;

struct CplDev {
  int nf1, nf2, npts, lcap, spectra, istyp, nsum;
  long long nkf;
  double df, sigma, re, tred;
  double thetas, phis, thetac, phic;
  double mt[6];
  const int* nwn;       // [nf2]
  const int* koff;      // [nf] first wavenumber index of each frequency in the spectra
  const double* delta;  // [npts]
  const double* xi;     // [npts]
  const double* nrm;    // [npts * 3]
  const double2* evf;   // [nf2 + 1]
  const double2* zel;   // [nf2 * 7]
  // sums per table kind, rank of each sum within its kind, offsets of each kind's
  // coefficient rows A[row][lcap] and results C[row][npts]; row = 2 (slot nsk + rank) + re/im
  int nsk[CPL_NKIND];
  int rank[CPL_NSUM];
  long long aoff[CPL_NKIND], coff[CPL_NKIND];
};

// tab[(kind * lcap + l) * npts + pt] of one (point, m), in the reference's operation order
__device__ void cpl_legendre_series(int pt, int m, int npts, int lmax, int lcap, double ct, double st, double* tab) {
  const bool atpoles = !(st > 0.0);
  auto row = [&](int kind) { return tab + (long long)kind * lcap * npts + pt; };
  double* Tp = row(m);
  double* Td = row(3 + m);
  double* Ts = m >= 1 ? row(5 + m) : nullptr;
  double* T2 = row(8 + m);
  double* Tt = m >= 1 ? row(10 + m) : nullptr;
  double pmm = 1.0, fact = 1.0;
  for (int j = 1; j <= m; ++j) { pmm = pmm * fact * st; fact = fact + 2.0; }
  const double rst = 1.0 / st;
  const double isct = ct >= 0.0 ? 1.0 : -1.0;
  double pl2 = 0.0, pl1 = 0.0;
  for (int l = 0; l <= lmax; ++l) {
    double p;
    if (l < m) p = 0.0;
    else if (l == m) p = pmm;
    else if (l == m + 1) p = ct * (double)(2 * m + 1) * pmm;
    else p = (ct * (double)(2 * l - 1) * pl1 - (double)(l + m - 1) * pl2) / (double)(l - m);
    double dp = 0.0, ps = 0.0, d2 = 0.0, dts = 0.0;
    const double ll1 = (double)l * (double)(l + 1);
    if (!atpoles) {
      if (l == m) dp = (double)m * ct * p * rst;
      else if (l > m) dp = ((double)l * ct * p - (double)(l + m) * pl1) * rst;
      if (l >= m) {
        if (m >= 1) ps = p * rst;
        d2 = ((-ct) * rst) * dp + ((double)(m * m) * (rst * rst) - ll1) * p;
        if (m >= 1) dts = rst * (dp - (ct * rst) * p);
      }
    } else {
      const double sl = (l % 2 == 0) ? 1.0 : isct;          // isct^l
      const double sl1 = (l % 2 == 0) ? isct : 1.0;         // isct^(l+1)
      const double q = (double)(l + 2) * (double)(l + 1) * (double)l * (double)(l - 1);
      if (m == 1) dp = 0.5 * ll1 * sl;
      if (m == 1 && l >= 1) ps = 0.5 * ll1 * sl1;
      if (m == 0) d2 = 0.5 * ll1 * sl;
      if (m == 2) d2 = 0.25 * q * sl;
      if (m == 2 && l >= 1) dts = 0.125 * q * sl1;
    }
    if (l < lcap) {
      const long long o = (long long)l * npts;
      Tp[o] = p; Td[o] = dp; T2[o] = d2;
      if (Ts) Ts[o] = ps;
      if (Tt) Tt[o] = dts;
    }
    pl2 = pl1;
    pl1 = p;
  }
}
// tab[(kind * lcap + l) * npts + pt]; one thread per (point, m)
__global__ void cpl_legendre_kernel(int npts, int lmax, int lcap, const double* __restrict__ delta, double* tab) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npts * 3) return;
  const int pt = idx % npts, m = idx / npts;
  cpl_legendre_series(pt, m, npts, lmax, lcap, cos(delta[pt]), sin(delta[pt]), tab);
}

// Fast form (fast backend): the same tables with the upward recurrence written as
// p_l = alpha_l p_{l-1} + beta_l p_{l-2} and 1/(l - m) from a shared-memory
// table, so one FMA per degree sits on the dependent chain (the plain form's
// software division leaves the 3 npts threads of this kernel waiting on it); the
// derivative tables follow in FMA form.  Rounding differs from the plain form's
// only (relative 1e-13 at l = 3200).  Poles keep the plain form's special values.
constexpr int CPL_LF_THREADS = 64;
__global__ void __launch_bounds__(CPL_LF_THREADS) cpl_legendre_fast_kernel(int npts, int lmax, int lcap,
                                                                           const double* __restrict__ delta,
                                                                           double* tab) {
  extern __shared__ double rcp[];   // rcp[n] = 1/n, n = 1..lmax
  for (int n = threadIdx.x + 1; n <= lmax; n += blockDim.x) rcp[n] = 1.0 / (double)n;
  __syncthreads();
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= npts * 3) return;
  const int pt = idx % npts, m = idx / npts;
  const double ct = cos(delta[pt]), st = sin(delta[pt]);
  if (!(st > 0.0)) {
    cpl_legendre_series(pt, m, npts, lmax, lcap, ct, st, tab);
    return;
  }
  auto row = [&](int kind) { return tab + (long long)kind * lcap * npts + pt; };
  double* Tp = row(m);
  double* Td = row(3 + m);
  double* Ts = m >= 1 ? row(5 + m) : nullptr;
  double* T2 = row(8 + m);
  double* Tt = m >= 1 ? row(10 + m) : nullptr;
  const long long stride = npts;
  double pmm = 1.0, fact = 1.0;
  for (int j = 1; j <= m; ++j) { pmm = pmm * fact * st; fact = fact + 2.0; }
  const double rst = 1.0 / st, ctr = ct * rst, m2r2 = (double)(m * m) * (rst * rst);
  // d2P/dtheta2 = -(cos/sin) dP/dtheta + (m^2/sin^2 - l(l+1)) P,  d/dtheta (P/sin) = (dP/dtheta - (cos/sin) P)/sin
  auto put = [&](long long o, double p, double dp, double ll1) {
    Tp[o] = p;
    Td[o] = dp;
    T2[o] = fma(-ctr, dp, (m2r2 - ll1) * p);
    if (Ts) Ts[o] = p * rst;
    if (Tt) Tt[o] = rst * fma(-ctr, p, dp);
  };
  long long o = 0;
  for (int l = 0; l < m && l <= lmax; ++l, o += stride) {
    Tp[o] = 0.0; Td[o] = 0.0; T2[o] = 0.0;
    if (Ts) Ts[o] = 0.0;
    if (Tt) Tt[o] = 0.0;
  }
  if (m > lmax) return;
  put(o, pmm, (double)m * ct * pmm * rst, (double)m * (double)(m + 1));   // l = m
  if (m + 1 > lmax) return;
  o += stride;
  const double p1 = ct * (double)(2 * m + 1) * pmm;   // l = m + 1
  double dl = (double)(m + 1);
  put(o, p1, fma(dl * ct, p1, -(dl + (double)m) * pmm) * rst, dl * (dl + 1.0));
  o += stride;
  double pl2 = pmm, pl1 = p1;
  const double mm1 = (double)(m - 1), md = (double)m;
#pragma unroll 2
  for (int l = m + 2; l <= lmax; ++l, o += stride) {
    dl += 1.0;
    const double r = rcp[l - m];
    const double alpha = ct * fma(2.0, dl, -1.0) * r;
    const double bp = -(dl + mm1) * r * pl2;   // off the chain: pl2 is known a degree early
    const double p = fma(alpha, pl1, bp);
    put(o, p, fma(dl * ct, p, -(dl + md) * pl1) * rst, dl * (dl + 1.0));
    pl2 = pl1;
    pl1 = p;
  }
}

// A[aoff[kind] + row * lcap + l], row = 2 (slot nsk[kind] + rank) + re/im: the
// terms of sum k of frequency nf1 + slot without the table value, zero outside
// the sum's degrees; one thread per (slot, sum, degree)
__global__ void cpl_coef_kernel(CplDev S, const float* __restrict__ gr, const float* __restrict__ gi, double* A) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = S.nf2 - S.nf1 + 1;
  if (idx >= (long long)nf * S.nsum * S.lcap) return;
  const int l = (int)(idx % S.lcap);
  const int k = (int)((idx / S.lcap) % S.nsum);
  const int slot = (int)(idx / ((long long)S.lcap * S.nsum));
  const CplSum cs = S.istyp == 1 ? c_cpl[k] : c_cplf[k];
  const int jf = S.nf1 + slot, nwn = S.nwn[jf - 1], lmax = nwn - 1;
  double vr = 0.0, vi = 0.0;
  if (l >= cs.l0 && l <= lmax) {
    // cos^2 taper of this frequency (harmonicDegreeSums.f90:356-369), TAPFRAC = 0.2
    const double tapfrac = 0.2;
    int jt = (int)floor((double)lmax * (1.0 - tapfrac) + 0.5);
    jt = jt < lmax ? jt : lmax;
    jt = jt > 1 ? jt : 1;
    double tap = 1.0;
    if (l >= jt) {
      const double c1 = (double)lmax * tapfrac * 2.0 / PI_F;
      const double c2 = (1.0 - tapfrac) / tapfrac * 0.5 * PI_F;
      const double c = cos((double)(float)l / c1 - c2);
      tap = c * c;
    }
    double c = (2.0 * (double)l + 1.0) / (4.0 * PI_F) * tap;
    if (cs.fac != 0.0) c = c * (cs.fac / (double)(float)(l * (l + 1)));
    const long long o = (long long)cs.col * S.nkf + S.koff[slot] + l;
    vr = c * (double)gr[o];
    vi = c * (double)gi[o];
  }
  const long long row = 2LL * ((long long)slot * S.nsk[cs.kind] + S.rank[k]);
  double* Ar = A + S.aoff[cs.kind] + row * S.lcap;
  Ar[l] = vr;
  Ar[S.lcap + l] = vi;
}

// FP64 tiled product C[kind][row][pt] = sum_l A[kind][row][l] * T[kind][l][pt]:
// 128 x 128 output tile per block of 256 threads, 8 x 8 per thread (rows ty + 16 i,
// points tx + 16 j: conflict-free shared reads, coalesced stores), K step 16.  The
// next K tile is loaded into registers while the current one is multiplied.  A
// tile's degree loop ends at the largest degree count of its frequencies (the
// coefficients beyond a frequency's count are zero).
constexpr int CT_M = 128, CT_N = 128, CT_K = 16;
constexpr int CT_LOADS = CT_M * CT_K / 256;   // elements of each operand tile per thread
static_assert(CT_M * CT_K == CT_N * CT_K && CT_LOADS == 8, "tile shape");
__global__ void __launch_bounds__(256, 1) cpl_gemm_kernel(CplDev S, const double* __restrict__ A,
                                                          const double* __restrict__ T, double* C) {
  const int kind = blockIdx.z;
  const int nsk = S.nsk[kind];
  const int nf = S.nf2 - S.nf1 + 1;
  const int M = 2 * nf * nsk, N = S.npts;
  const int m0 = blockIdx.y * CT_M, n0 = blockIdx.x * CT_N;
  if (m0 >= M) return;
  int K = 0;
  {
    const int s0 = m0 / (2 * nsk), s1 = min(nf - 1, (m0 + CT_M - 1) / (2 * nsk));
    for (int sl = s0; sl <= s1; ++sl) K = max(K, S.nwn[S.nf1 - 1 + sl]);
    K = min(K, S.lcap);
  }
  const double* Ak = A + S.aoff[kind];
  const double* Tk = T + (long long)kind * S.lcap * N;
  double* Ck = C + S.coff[kind];
  __shared__ double As[CT_K][CT_M + 1];
  __shared__ double Bs[CT_K][CT_N];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  double ra[CT_LOADS], rb[CT_LOADS];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < CT_LOADS; ++q) {
      const int i = tid + 256 * q;
      const int gm = m0 + i / CT_K, gk = k0 + i % CT_K;
      ra[q] = (gm < M && gk < K) ? Ak[(long long)gm * S.lcap + gk] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < CT_LOADS; ++q) {
      const int i = tid + 256 * q;
      const int gk = k0 + i / CT_N, gn = n0 + i % CT_N;
      rb[q] = (gk < K && gn < N) ? Tk[(long long)gk * N + gn] : 0.0;
    }
  };
  if (K > 0) load(0);
  for (int k0 = 0; k0 < K; k0 += CT_K) {
#pragma unroll
    for (int q = 0; q < CT_LOADS; ++q) {
      const int i = tid + 256 * q;
      As[i % CT_K][i / CT_K] = ra[q];
      Bs[i / CT_N][i % CT_N] = rb[q];
    }
    __syncthreads();
    if (k0 + CT_K < K) load(k0 + CT_K);
#pragma unroll
    for (int kk = 0; kk < CT_K; ++kk) {
      double a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gn = n0 + tx + 16 * j;
      if (gn < N) Ck[(long long)gm * N + gn] = acc[i][j];
    }
  }
}

__device__ __forceinline__ void vec_lc_from_ls(double d, double x, const dz* u, dz* o) {
  const double cd = cos(d), sd = sin(d), cx = cos(x), sx = sin(x);
  o[0] = ((sd * cx) * u[0] + (cd * cx) * u[1]) - sx * u[2];
  o[1] = ((sd * sx) * u[0] + (cd * sx) * u[1]) + cx * u[2];
  o[2] = cd * u[0] - sd * u[1];
}
__device__ __forceinline__ void vec_gc_from_lc(double t, double p, const dz* u, dz* o) {
  const double ct = cos(t), st = sin(t), cp = cos(p), sp = sin(p);
  o[0] = ((ct * cp) * u[0] - sp * u[1]) + (st * cp) * u[2];
  o[1] = ((ct * sp) * u[0] + cp * u[1]) + (st * sp) * u[2];
  o[2] = (-st) * u[0] + ct * u[2];
}
__device__ __forceinline__ void vec_lc_from_gc(double t, double p, const dz* u, dz* o) {
  const double ct = cos(t), st = sin(t), cp = cos(p), sp = sin(p);
  o[0] = ((ct * cp) * u[0] + (ct * sp) * u[1]) - st * u[2];
  o[1] = (-sp) * u[0] + cp * u[1];
  o[2] = ((st * cp) * u[0] + (st * sp) * u[1]) + ct * u[2];
}
// T' = R T R^T: every column, then every row through the vector rule
// (axesRotation.f90:199-212,377-426,486-560)
template <int W>
__device__ __forceinline__ void ten_rot(double a, double b, const dz t[3][3], dz o[3][3]) {
  auto f = [&](const dz* u, dz* v) {
    if (W == 0) vec_lc_from_ls(a, b, u, v);
    else if (W == 1) vec_gc_from_lc(a, b, u, v);
    else vec_lc_from_gc(a, b, u, v);
  };
  dz tp[3][3];
  for (int j = 0; j < 3; ++j) {
    dz col[3] = {t[0][j], t[1][j], t[2][j]}, r[3];
    f(col, r);
    for (int i = 0; i < 3; ++i) tp[i][j] = r[i];
  }
  for (int i = 0; i < 3; ++i) {
    dz row[3] = {tp[i][0], tp[i][1], tp[i][2]}, r[3];
    f(row, r);
    for (int j = 0; j < 3; ++j) o[i][j] = r[j];
  }
}

// one thread per (point, frequency): X[(pt * 6 + c) * nf2 + jf - 1], c = displacement
// (or velocity) x, y, z, traction x, y, z in the box frame (x east, y north)
__global__ void cpl_point_kernel(CplDev S, const double* __restrict__ C, double2* X) {
  const int nf = S.nf2 - S.nf1 + 1;
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)S.npts * nf) return;
  const int slot = (int)(idx % nf), pt = (int)(idx / nf);
  const int jf = S.nf1 + slot;
  dz w[CPL_NSUM + 1];
  for (int k = 0; k < S.nsum; ++k) {
    const int kind = S.istyp == 1 ? c_cpl[k].kind : c_cplf[k].kind;
    const long long row = 2LL * ((long long)slot * S.nsk[kind] + S.rank[k]);
    const double* Ck = C + S.coff[kind] + row * S.npts + pt;
    w[k + 1] = dz{Ck[0], Ck[S.npts]};
  }
  const double* m = S.mt;
  const double phi = S.xi[pt], dl = S.delta[pt], re = S.re;
  const double sphi = sin(phi), cphi = cos(phi), s2phi = sin(2.0 * phi), c2phi = cos(2.0 * phi);
  const double rst = re * sin(dl);
  dz u[3], ur[3], ut[3], uf[3];
  if (S.istyp == 0) {   // force{,RadDeriv,ThetaDeriv,PhiDeriv}SingleFrequencyDisplacement (:35-103)
    const double fh = m[1] * cphi + m[2] * sphi, ft = m[1] * sphi - m[2] * cphi;
    const double fp = (-m[1]) * sphi + m[2] * cphi, fq = m[1] * cphi + m[2] * sphi;
    for (int q = 0; q < 3; ++q) {
      dz* v = q == 0 ? u : (q == 1 ? ur : ut);
      const int o = 7 * q;
      v[0] = w[o + 1] * m[0] + w[o + 2] * fh;
      v[1] = w[o + 3] * m[0] + (w[o + 4] + w[o + 5]) * fh;
      v[2] = (w[o + 6] + w[o + 7]) * ft;
    }
    for (int c = 0; c < 3; ++c) ut[c] = ut[c] / re;
    uf[0] = w[2] * fp;
    uf[1] = (w[4] + w[5]) * fp;
    uf[2] = (w[6] + w[7]) * fq;
    for (int c = 0; c < 3; ++c) uf[c] = uf[c] / rst;
  } else {
    const double t1 = m[3] * cphi + m[4] * sphi, t2 = (m[2] - m[1]) * c2phi - 2.0 * m[5] * s2phi;
    const double t3 = m[4] * cphi - m[3] * sphi, t4 = (m[2] - m[1]) * s2phi + 2.0 * m[5] * c2phi;
    u[0] = w[1] * m[0] + w[2] * (m[1] + m[2]) + w[3] * t1 + w[4] * t2;
    u[1] = w[5] * m[0] + w[6] * (m[1] + m[2]) + (w[7] + w[9]) * t1 + (w[8] + w[10]) * t2;
    u[2] = (w[11] + w[13]) * t3 + (w[12] + w[14]) * t4;
    ur[0] = w[15] * m[0] + w[16] * (m[1] + m[2]) + w[17] * t1 + w[18] * t2;
    ur[1] = w[19] * m[0] + w[20] * (m[1] + m[2]) + (w[21] + w[23]) * t1 + (w[22] + w[24]) * t2;
    ur[2] = (w[25] + w[27]) * t3 + (w[26] + w[28]) * t4;
    ut[0] = w[29] * m[0] + w[30] * (m[1] + m[2]) + w[31] * t1 + w[32] * t2;
    ut[1] = w[33] * m[0] + w[34] * (m[1] + m[2]) + (w[35] + w[37]) * t1 + (w[36] + w[38]) * t2;
    ut[2] = (w[39] + w[41]) * t3 + (w[40] + w[42]) * t4;
    for (int c = 0; c < 3; ++c) ut[c] = ut[c] / re;
    const double p1 = (-m[3]) * sphi + m[4] * cphi;
    const double p2 = (-2.0) * (m[2] - m[1]) * s2phi - 4.0 * m[5] * c2phi;
    const double p3 = (-m[4]) * sphi - m[3] * cphi;
    const double p4 = 2.0 * (m[2] - m[1]) * c2phi - 4.0 * m[5] * s2phi;
    uf[0] = w[3] * p1 + w[4] * p2;
    uf[1] = (w[7] + w[9]) * p1 + (w[8] + w[10]) * p2;
    uf[2] = (w[11] + w[13]) * p3 + (w[12] + w[14]) * p4;
    for (int c = 0; c < 3; ++c) uf[c] = uf[c] / rst;
  }
  // strain and stress (singleFrequencyDisplacement.f90:229-262)
  const double rtd = re * tan(dl);
  dz e[3][3];
  e[0][0] = ur[0];
  e[1][1] = ut[1] + u[0] / re;
  e[2][2] = (uf[2] + u[0] / re) + u[1] / rtd;
  e[0][1] = 0.5 * ((ut[0] + ur[1]) - u[1] / re);
  e[0][2] = 0.5 * ((uf[0] + ur[2]) - u[2] / re);
  e[1][2] = 0.5 * ((uf[1] + ut[2]) - u[2] / rtd);
  e[2][1] = e[1][2]; e[2][0] = e[0][2]; e[1][0] = e[0][1];
  dz el[5];
  for (int c = 0; c < 5; ++c) { const double2 v = S.zel[(long long)(jf - 1) * 7 + c]; el[c] = dz{v.x, v.y}; }
  dz sg[3][3];
  sg[0][0] = el[1] * e[0][0] + el[2] * (e[1][1] + e[2][2]);
  sg[1][1] = (el[2] * e[0][0] + el[0] * (e[1][1] + e[2][2])) - (2.0 * el[4]) * e[2][2];
  sg[2][2] = (el[2] * e[0][0] + el[0] * (e[1][1] + e[2][2])) - (2.0 * el[4]) * e[1][1];
  sg[0][1] = (2.0 * el[3]) * e[0][1];
  sg[0][2] = (2.0 * el[3]) * e[0][2];
  sg[1][2] = (2.0 * el[4]) * e[1][2];
  sg[1][0] = sg[0][1]; sg[2][0] = sg[0][2]; sg[2][1] = sg[1][2];
  // to the box frame (computeTension, :677-705)
  const double gam = 0.5 * PI_F;
  dz a[3], b[3];
  vec_lc_from_ls(dl, phi, u, a);
  vec_gc_from_lc(S.thetas, S.phis, a, b);
  vec_lc_from_gc(S.thetac, S.phic, b, a);
  vec_lc_from_gc(0.0, gam, a, b);
  dz ta[3][3], tb[3][3];
  ten_rot<0>(dl, phi, sg, ta);
  ten_rot<1>(S.thetas, S.phis, ta, tb);
  ten_rot<2>(S.thetac, S.phic, tb, ta);
  ten_rot<2>(0.0, gam, ta, tb);
  const double* n = S.nrm + 3 * pt;
  dz tr[3];
  for (int i = 0; i < 3; ++i) tr[i] = ((dz{0.0, 0.0} + tb[i][0] * n[0]) + tb[i][1] * n[1]) + tb[i][2] * n[2];
  if (!S.spectra) {
    const dz ci{0.0, 1.0};
    const dz ef{S.evf[jf].x, S.evf[jf].y};
    const dz zom{TWO_PI_F * (double)(jf - 1) * S.df, -S.sigma};
    const dz tsf = zexp_dev(((ci * TWO_PI_F) * (double)(jf - 1)) * S.df * S.tred) * exp(S.sigma * S.tred);
    for (int c = 0; c < 3; ++c) {
      b[c] = (((b[c] * ef) * ci) * zom) * tsf;
      tr[c] = (tr[c] * ef) * tsf;
    }
  }
  for (int c = 0; c < 3; ++c) {
    X[((long long)pt * 6 + c) * S.nf2 + (jf - 1)] = make_double2(b[c].re, b[c].im);
    X[((long long)pt * 6 + 3 + c) * S.nf2 + (jf - 1)] = make_double2(tr[c].re, tr[c].im);
  }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace gem

using namespace gem;

// SPECFEM-coupling synthetics of a moment or force source at npts boundary points of one
// node (the loops of computeSyntheticsForSpecfemCoupling.f90:509-549, 571-590 over
// computeSynthetics :714-793).  d_gr/d_gi: float32 DSV spectra with radial
// derivatives of the node, (nkfmax, nsp >= 20).  Host arrays: nwn[nf2], zelcon
// [nf2 * 7] interleaved complex elastic constants of the node per frequency
// (getComplexConstantsSelectedExternalRadialNodes), mt[6], delta/xi[npts] (rad),
// nrm[npts * 3] box-frame normals.  Outputs (device): spectra != 0:
// d_spec[(p * 6 + c) * nf2 + jf - 1] complex, unfiltered; otherwise
// d_traces[(p * 6 + c) * nsamp + i], c = velocity x, y, z, traction x, y, z.
extern "C" int gem_coupling_run_device(gem_ctx* ctx, const gem_coupling_params* p, const int* nwn, const float* d_gr,
                                       const float* d_gi, const double* zelcon, const double* mt, int npts,
                                       const double* delta, const double* xi, const double* nrm, double* d_spec,
                                       float* d_traces, void* stream) {
  if (!ctx) return GEM_ERROR;
  if (!p || !nwn || !d_gr || !d_gi || !zelcon || !mt || !delta || !xi || !nrm)
    return gem_set_error(ctx, "coupling: null argument");
  if (npts < 1) return gem_set_error(ctx, "coupling: no boundary points");
  if (p->nf2 - p->nf1 + 1 > 65535) return gem_set_error(ctx, "coupling: more than 65535 frequencies");
  if (p->istyp != 0 && p->istyp != 1) return gem_set_error(ctx, "coupling: invalid source type");
  if (p->nsp < (p->istyp == 1 ? 20 : 10))
    return gem_set_error(ctx, "coupling: the DSV spectra need radial derivatives (nsp >= 20 moment, 10 force)");
  if (p->nf1 < 1 || p->nf2 < p->nf1 || p->nwnmax < 1 || !(p->re > 0))
    return gem_set_error(ctx, "coupling: invalid frequency range, degrees or radius");
  if (p->spectra ? !d_spec : !d_traces) return gem_set_error(ctx, "coupling: null output");
  const int nf = p->nf2 - p->nf1 + 1;
  std::vector<int> koff(nf);
  long long k = 0;
  for (int jf = 1; jf < p->nf1; ++jf) k += nwn[jf - 1];
  for (int s = 0; s < nf; ++s) {
    const int n = nwn[p->nf1 + s - 1];
    if (n < 1 || n > p->nwnmax) return gem_set_error(ctx, "coupling: number of degrees outside 1..nwnmax");
    koff[s] = (int)k;
    k += n;
  }
  if (k > p->nkfmax) return gem_set_error(ctx, "coupling: the wavenumber counts exceed nkfmax");
  if (cudaSetDevice(gem_ctx_device(ctx)) != cudaSuccess) return gem_set_error(ctx, "coupling: cudaSetDevice failed");
  cudaStream_t st = (cudaStream_t)stream;
  // event filter at the synthetics' frequencies (Butterworth band-pass, eventFilter.f90:40-83)
  gem_synth_params sp{};
  sp.nf1 = p->nf1; sp.nf2 = p->nf2; sp.df = p->df; sp.sigma = p->sigma;
  sp.order_highpass = p->order_highpass; sp.fc_highpass = p->fc_highpass;
  sp.order_lowpass = p->order_lowpass; sp.fc_lowpass = p->fc_lowpass;
  std::vector<double2> evf;
  if (p->spectra) evf.assign(p->nf2 + 1, make_double2(0, 0));
  else event_filter_host(&sp, evf);
  // sums per table kind and the rank of each sum within its kind
  const int nsum = p->istyp == 1 ? CPL_NSUM : 21;
  const CplSum* sums = p->istyp == 1 ? h_cpl : h_cplf;
  CplDev S{};
  for (int k = 0; k < nsum; ++k) S.rank[k] = S.nsk[sums[k].kind]++;
  const int lcap = p->nwnmax;
  long long ao = 0, co = 0;
  for (int kd = 0; kd < CPL_NKIND; ++kd) {
    S.aoff[kd] = ao; S.coff[kd] = co;
    ao += 2LL * nf * S.nsk[kd] * lcap;
    co += 2LL * nf * S.nsk[kd] * npts;
  }
  // workspace: tables, coefficient rows, sums, spectra, small inputs
  const size_t b_tab = align256((size_t)npts * CPL_NKIND * lcap * sizeof(double));
  const size_t b_a = align256((size_t)ao * sizeof(double));
  const size_t b_hd = align256((size_t)co * sizeof(double));
  const size_t b_x = align256((size_t)npts * 6 * p->nf2 * sizeof(double2));
  const size_t b_in = align256((size_t)nf * sizeof(int)) + align256((size_t)p->nf2 * sizeof(int)) +
                      3 * align256((size_t)npts * 3 * sizeof(double)) + align256(evf.size() * sizeof(double2)) +
                      align256((size_t)p->nf2 * 7 * sizeof(double2));
  char* ws = (char*)gem_ctx_aux(ctx, 12, b_tab + b_a + b_hd + b_x + b_in);
  if (!ws) return GEM_ERROR;
  double* tab = (double*)ws;
  double* A = (double*)(ws + b_tab);
  double* C = (double*)(ws + b_tab + b_a);
  double2* X = p->spectra ? (double2*)d_spec : (double2*)(ws + b_tab + b_a + b_hd);
  char* q = ws + b_tab + b_a + b_hd + b_x;
  auto take = [&](size_t bytes) { char* r = q; q += align256(bytes); return r; };
  int* d_koff = (int*)take((size_t)nf * sizeof(int));
  int* d_nwn = (int*)take((size_t)p->nf2 * sizeof(int));
  double* d_delta = (double*)take((size_t)npts * 3 * sizeof(double));
  double* d_xi = (double*)take((size_t)npts * 3 * sizeof(double));
  double* d_nrm = (double*)take((size_t)npts * 3 * sizeof(double));
  double2* d_evf = (double2*)take(evf.size() * sizeof(double2));
  double2* d_zel = (double2*)take((size_t)p->nf2 * 7 * sizeof(double2));
  if (cudaMemcpyAsync(d_koff, koff.data(), (size_t)nf * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_nwn, nwn, (size_t)p->nf2 * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_delta, delta, (size_t)npts * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_xi, xi, (size_t)npts * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_nrm, nrm, (size_t)npts * 3 * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_evf, evf.data(), evf.size() * sizeof(double2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_zel, zelcon, (size_t)p->nf2 * 7 * sizeof(double2), cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemsetAsync(X, 0, (size_t)npts * 6 * p->nf2 * sizeof(double2), st) != cudaSuccess)
    return gem_set_error(ctx, "coupling: input copy failed");
  S.nf1 = p->nf1; S.nf2 = p->nf2; S.npts = npts; S.lcap = lcap; S.spectra = p->spectra; S.nkf = p->nkfmax;
  S.df = p->df; S.sigma = p->sigma; S.re = p->re; S.tred = p->tred;
  S.thetas = p->thetas; S.phis = p->phis; S.thetac = p->thetac; S.phic = p->phic;
  S.istyp = p->istyp; S.nsum = nsum;
  for (int i = 0; i < (p->istyp == 1 ? 6 : 3); ++i) S.mt[i] = mt[i];
  S.nwn = d_nwn; S.koff = d_koff; S.delta = d_delta; S.xi = d_xi; S.nrm = d_nrm; S.evf = d_evf; S.zel = d_zel;
  const size_t rcp_bytes = (size_t)p->nwnmax * sizeof(double);
  if (gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST && rcp_bytes <= 200 * 1024) {
    cudaFuncSetAttribute(cpl_legendre_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rcp_bytes);
    cpl_legendre_fast_kernel<<<(npts * 3 + CPL_LF_THREADS - 1) / CPL_LF_THREADS, CPL_LF_THREADS, rcp_bytes, st>>>(
        npts, p->nwnmax - 1, lcap, d_delta, tab);
  } else {
    cpl_legendre_kernel<<<(npts * 3 + 127) / 128, 128, 0, st>>>(npts, p->nwnmax - 1, lcap, d_delta, tab);
  }
  const long long ncoef = (long long)nf * nsum * lcap;
  cpl_coef_kernel<<<(unsigned)((ncoef + 255) / 256), 256, 0, st>>>(S, d_gr, d_gi, A);
  int maxnsk = 0;
  for (int kd = 0; kd < CPL_NKIND; ++kd) maxnsk = std::max(maxnsk, S.nsk[kd]);
  const dim3 ggrid((unsigned)((npts + CT_N - 1) / CT_N), (unsigned)((2 * nf * maxnsk + CT_M - 1) / CT_M), CPL_NKIND);
  if (gem_ctx_backend(ctx) == GEM_BACKEND_GPU_FAST) {
    // the degree sums on tcgen05: 6 INT8 slices per operand, exact INT32 accumulation
    TcProblem TP{};
    TP.nkind = CPL_NKIND; TP.ncol = npts; TP.lcap = lcap; TP.lmax = p->nwnmax - 1; TP.nf1 = p->nf1; TP.nf2 = p->nf2;
    TP.nslice = 7;   // 49 bits: strain, stress and traction cancel between the 42 sums
    long long mtot = 0;
    for (int kd = 0; kd < CPL_NKIND; ++kd) {
      TP.nsk[kd] = S.nsk[kd];
      TP.coff[kd] = S.coff[kd];
      mtot += 2LL * nf * S.nsk[kd];
    }
    const size_t wsb = sums_tc_workspace(TP, mtot, nullptr);
    void* tws = gem_ctx_aux(ctx, 14, wsb);
    if (!tws) return GEM_ERROR;
    if (const char* why = sums_tc_run(TP, nwn, mtot, tab, A, C, tws, wsb, gem_ctx_tc_wait_ns(ctx), st))
      return gem_set_error(ctx, why);
  } else {
    cpl_gemm_kernel<<<ggrid, 256, 0, st>>>(S, A, tab, C);
  }
  const long long nthr = (long long)npts * nf;
  cpl_point_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, st>>>(S, C, X);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return gem_set_error(ctx, cudaGetErrorString(e));
  if (p->spectra) return GEM_OK;
  return gem_ifft_run_device(ctx, p->nf1, p->nf2, p->df, p->sigma, npts * 6, (const double*)X, p->nf2, p->nsamp,
                             p->dt, d_traces, stream);
}

// Same with host buffers (blocking): spectra gr/gi (nkfmax, nsp) float32, outputs
// spec [npts * 6 * nf2] complex or traces [npts * 6 * nsamp] float32.
extern "C" int gem_coupling_run(gem_ctx* ctx, const gem_coupling_params* p, const int* nwn, const float* gr,
                                const float* gi, const double* zelcon, const double* mt, int npts,
                                const double* delta, const double* xi, const double* nrm, double* spec,
                                float* traces) {
  if (!ctx) return GEM_ERROR;
  if (!p || !gr || !gi || npts < 1) return gem_set_error(ctx, "coupling: null argument or no boundary points");
  if (p->nsp < 1 || p->nkfmax < 1) return gem_set_error(ctx, "coupling: invalid spectra extent");
  if (p->spectra ? !spec : !traces) return gem_set_error(ctx, "coupling: null output");
  if (cudaSetDevice(gem_ctx_device(ctx)) != cudaSuccess) return gem_set_error(ctx, "coupling: cudaSetDevice failed");
  const size_t nin = (size_t)p->nkfmax * p->nsp;
  const size_t nout = p->spectra ? (size_t)npts * 6 * p->nf2 * 2 * sizeof(double)
                                 : (size_t)npts * 6 * p->nsamp * sizeof(float);
  char* buf = (char*)gem_ctx_aux(ctx, 13, 2 * align256(nin * sizeof(float)) + align256(nout));
  if (!buf) return GEM_ERROR;
  float* dgr = (float*)buf;
  float* dgi = (float*)(buf + align256(nin * sizeof(float)));
  char* dout = buf + 2 * align256(nin * sizeof(float));
  if (cudaMemcpy(dgr, gr, nin * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(dgi, gi, nin * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
    return gem_set_error(ctx, "coupling: copy of the spectra failed");
  int rc = gem_coupling_run_device(ctx, p, nwn, dgr, dgi, zelcon, mt, npts, delta, xi, nrm,
                                   p->spectra ? (double*)dout : nullptr, p->spectra ? nullptr : (float*)dout,
                                   nullptr);
  if (rc) return rc;
  if (cudaMemcpy(p->spectra ? (void*)spec : (void*)traces, dout, nout, cudaMemcpyDeviceToHost) != cudaSuccess)
    return gem_set_error(ctx, "coupling: copy of the results failed");
  return GEM_OK;
}
