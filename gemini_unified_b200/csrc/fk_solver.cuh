// FP64 radial ODE solver of the FK hot path: one (omega, l) item per thread.
//
// The arithmetic of every step restates the reference (file:line cited per
// function) in the same operation order; the control structure is the
// GPU's own:
//   * system matrices are evaluated at each modified-midpoint sub-step instead
//     of being cached on the 1/48 grid (same values, no per-thread cache);
//   * matrix-vector products skip the structural zeros of each system (adding
//     a zero product leaves a sum unchanged);
//   * results at nodes go to a per-thread scratch slot laid out
//     element-major across threads, so a warp's stores coalesce;
//   * a warp integrates its 32 items in lockstep (see fk_kernel.cu);
//   * the spheroidal adjoint is integrated only for the unit jumps whose
//     Green functions reach a stored component (jumps 2 and 4 without
//     stresses), and only as far as the last node it feeds.
#pragma once
#include "gem_device.cuh"
#include "fk_types.cuh"

// Compiled twice: GEM_NS = gem_plain (GEM_FAST 0, built with --fmad=false, the
// parity path) and GEM_NS = gem_fast (GEM_FAST 1, FMA contraction, division-free
// spline evaluation, reciprocal-based complex inverses).
#ifndef GEM_NS
#error "define GEM_NS and GEM_FAST before including fk_solver.cuh"
#endif

namespace GEM_NS {
using namespace gem;

// Bulirsch-Stoer subdivision scheme (parametersBulirschStep.f90:28-48)
__device__ __constant__ const int SEQDIV[7] = {2, 4, 6, 8, 12, 16, 24};
__device__ __constant__ const int NXDIV[7] = {3, 2, 4, 4, 4, 8, 8};
// flop weights of one system-matrix evaluation (incl. spline) and of one
// midpoint matrix-vector update, per ODE system (minors, fluid, radial,
// toroidal, adjoint); identical to the oracle's accounting.
__device__ __constant__ const int FLOP_SYSMAT[5] = {230, 150, 175, 140, 215};
__device__ __constant__ const int FLOP_MV[5] = {8 * 19 + 4 * 5, 8 * 3 + 4 * 2, 8 * 4 + 4 * 2,
                                               8 * 4 + 4 * 2, 8 * 14 + 4 * 4};

// ------------------------------------------------------------------------
//  locate (locatePoint.f90:72-101), 1-based x in the parameter block
// ------------------------------------------------------------------------
__device__ __forceinline__ int locate(double xx, int n, const double* x) {
  int lidx = 0, ridx = n + 1;
  bool asc = x[n] > x[1];
  while (ridx - lidx > 1) {
    int midx = (lidx + ridx) >> 1;
    bool gt = xx > x[midx];
    if (asc) { if (gt) lidx = midx; else ridx = midx; }
    else { if (gt) ridx = midx; else lidx = midx; }
  }
  return lidx;
}

// getLayerIndexNodeEarthmodel (nodeEarthmodel.f90:599-607)
__device__ __forceinline__ void layer_index(const FKStatic& P, double r, int& nl, int& top) {
  nl = locate(r, P.nlay, P.rb) + 1;
  int nlc = nl < P.nlay ? nl : P.nlay;
  top = fabs(r / P.rb[nlc] - 1.0) < EPS_D ? 1 : 0;
}

// ------------------------------------------------------------------------
//  Spline evaluation (splineEarthmodelCoefficients.f90:118-162).
//  MASK selects the elastic constants (bit c -> constant c of A,C,F,L,N,K,M).
// ------------------------------------------------------------------------
template <unsigned MASK>
__device__ __forceinline__ void eval_spline(const FKStatic& P, const Env& e, double r, int nl, double& ro,
                                            dz* el) {
  const Tab* __restrict__ T = e.tab;
#if GEM_FAST
  {
    // cubic in t = r - rk(j) per knot interval, Horner form (no divisions)
    int j;
    double t;
    if (nl == 1) {
      j = T->iktop[1];
      t = 0.0;
    } else {
      int j1 = T->iktop[nl - 1] + 1, j2 = T->iktop[nl];
      if (j2 - j1 == 1) {
        j = j1;
      } else if (P.equidis == 1) {
        j = (int)((r - T->rk[j1]) * T->rdrk[nl]) + j1;
        j = j < j1 ? j1 : (j > j2 - 1 ? j2 - 1 : j);
      } else {
        j = j1 - 1;
        int jr = j2 + 1;
        while (jr - j > 1) {
          int m = (j + jr) >> 1;
          if (r > T->rk[m]) j = m; else jr = m;
        }
        if (j == j1 - 1) j = j1;
      }
      j = j < 1 ? 1 : (j > P.nk - 1 ? P.nk - 1 : j);
      t = r - T->rk[j];
    }
    const double* __restrict__ q = e.poly + (long long)j * POLY_STRIDE;
    auto horner = [&](int v) {
      double2 c32 = __ldg(reinterpret_cast<const double2*>(q + 4 * v));
      double2 c10 = __ldg(reinterpret_cast<const double2*>(q + 4 * v + 2));
      return fma(fma(fma(c32.x, t, c32.y), t, c10.x), t, c10.y);
    };
    ro = horner(0);
#pragma unroll
    for (int c = 0; c < 7; ++c)
      if (MASK & (1u << c)) el[c] = dz{horner(1 + 2 * c), horner(2 + 2 * c)};
    return;
  }
#endif
  const double* __restrict__ spl = e.spl;
  // One code path for every layer, so lanes of a warp stay converged:
  //  * layer 1 (homogeneous sphere) reads knot iktop(1) with weights (1,0,0,0);
  //  * two-knot layers use the cubic formula with their zero second
  //    derivatives, which adds exact zeros to the linear interpolant.
  int j;
  double a, b, cc, dd;
  if (nl == 1) {
    j = T->iktop[1];
    a = 1.0; b = 0.0; cc = 0.0; dd = 0.0;
  } else {
    int j1 = T->iktop[nl - 1] + 1, j2 = T->iktop[nl];
    if (j2 - j1 == 1) {
      j = j1;
    } else if (P.equidis == 1) {
      j = (int)((r - T->rk[j1]) / T->drk[nl]) + j1;
      if (j == j2) j = j2 - 1;
    } else {
      j = j1 - 1;
      int jr = j2 + 1;
      while (jr - j > 1) {
        int m = (j + jr) >> 1;
        if (r > T->rk[m]) j = m; else jr = m;
      }
      if (j == j1 - 1) j = j1;
    }
    j = j < 1 ? 1 : (j > P.nk - 1 ? P.nk - 1 : j);   // memory guard (in-range inputs unaffected)
    double x1 = T->rk[j], x2 = T->rk[j + 1], h = x2 - x1;
    a = (x2 - r) / h;
    b = 1.0 - a;
    cc = h * h * a * (a * a - 1.0) / 6.0;
    dd = h * h * b * (b * b - 1.0) / 6.0;
  }
  const double* t1 = spl + j * SPL_STRIDE;
  const double* t2 = t1 + SPL_STRIDE;
  ro = a * __ldg(t1) + b * __ldg(t2) + cc * __ldg(t1 + 1) + dd * __ldg(t2 + 1);
#pragma unroll
  for (int c = 0; c < 7; ++c)
    if (MASK & (1u << c)) {
      double2 e1 = __ldg(reinterpret_cast<const double2*>(t1 + 2 + 2 * c));
      double2 e2 = __ldg(reinterpret_cast<const double2*>(t2 + 2 + 2 * c));
      double2 s1 = __ldg(reinterpret_cast<const double2*>(t1 + 16 + 2 * c));
      double2 s2 = __ldg(reinterpret_cast<const double2*>(t2 + 16 + 2 * c));
      el[c] = a * dz{e1.x, e1.y} + b * dz{e2.x, e2.y} + cc * dz{s1.x, s1.y} + dd * dz{s2.x, s2.y};
    }
}

#if GEM_FAST
// The environment of one Bulirsch-Stoer step (fast build): the knot range of
// the step's layer is looked up once per step instead of at every sub-step.
// The interval and t = r - rk(j) are the ones eval_spline finds.
struct EnvF : Env {
  int sj1, sjhi;       // first and last knot interval of the layer
  int sflat;           // layer 1: the homogeneous sphere, evaluated at its knot (t = 0)
  int sequi;           // equidistant knots: direct index; else the search of eval_spline
  double srk1, srdrk;  // rk(j1) and 1/drk of the layer
};
// Lanes without a step (active false) may hold no layer yet (a lane that never
// took an item): they read the tables of layer 1 and evaluate nothing.
__device__ __forceinline__ EnvF make_envf(const FKStatic& P, const Env& e, bool active) {
  EnvF f;
  static_cast<Env&>(f) = e;
  const Tab* __restrict__ T = e.tab;
  const int nl = (active && e.nl >= 1 && e.nl <= P.nlay) ? e.nl : 1;
  f.sflat = nl == 1;
  f.sequi = P.equidis == 1;
  if (nl == 1) {
    f.sj1 = f.sjhi = T->iktop[1];
    f.srk1 = 0.0; f.srdrk = 0.0;
  } else {
    const int j1 = T->iktop[nl - 1] + 1, j2 = T->iktop[nl];
    f.sj1 = j1; f.sjhi = j2 - 1;
    f.srk1 = T->rk[j1]; f.srdrk = T->rdrk[nl];
  }
  return f;
}
template <unsigned MASK>
__device__ __forceinline__ void eval_spline(const FKStatic& P, const EnvF& e, double r, double& ro, dz* el) {
  if (!e.sequi) { eval_spline<MASK>(P, static_cast<const Env&>(e), r, e.nl, ro, el); return; }
  const Tab* __restrict__ T = e.tab;
  int j = e.sj1;
  double t = 0.0;
  if (!e.sflat) {
    if (e.sjhi > e.sj1) {
      j = (int)((r - e.srk1) * e.srdrk) + e.sj1;
      j = j < e.sj1 ? e.sj1 : (j > e.sjhi ? e.sjhi : j);
    }
    j = j < 1 ? 1 : (j > P.nk - 1 ? P.nk - 1 : j);
    t = r - T->rk[j];
  }
  const double* __restrict__ q = e.poly + (long long)j * POLY_STRIDE;
  auto horner = [&](int v) {
    double2 c32 = __ldg(reinterpret_cast<const double2*>(q + 4 * v));
    double2 c10 = __ldg(reinterpret_cast<const double2*>(q + 4 * v + 2));
    return fma(fma(fma(c32.x, t, c32.y), t, c10.x), t, c10.y);
  };
  ro = horner(0);
#pragma unroll
  for (int c = 0; c < 7; ++c)
    if (MASK & (1u << c)) el[c] = dz{horner(1 + 2 * c), horner(2 + 2 * c)};
}
#endif

// ------------------------------------------------------------------------
//  ODE systems: y = A(x) z, nonzero entries only, column order as matmul
// ------------------------------------------------------------------------
enum { SYS_MINORS = 0, SYS_FLUID = 1, SYS_RADIAL = 2, SYS_TOROIDAL = 3, SYS_SOLIDT = 4 };
template <int SYS> struct SysNV;
template <> struct SysNV<SYS_MINORS> { static constexpr int NV = 5; };
template <> struct SysNV<SYS_FLUID> { static constexpr int NV = 2; };
template <> struct SysNV<SYS_RADIAL> { static constexpr int NV = 2; };
template <> struct SysNV<SYS_TOROIDAL> { static constexpr int NV = 2; };
template <> struct SysNV<SYS_SOLIDT> { static constexpr int NV = 4; };

// 1/z: Smith's division on the parity path, one reciprocal on the fast path
__device__ __forceinline__ dz zinv(dz z) {
#if GEM_FAST
  return zinv_fast(z);
#else
  return 1.0 / z;
#endif
}
__device__ __forceinline__ double rinv(double x) {
#if GEM_FAST
  return __drcp_rn(x);
#else
  return 1.0 / x;
#endif
}

#if GEM_FAST
// Fast build: the system matrix at x in a compact form -- the quantities
// that depend on x, from which the entries follow with a few products -- so
// that a Bulirsch-Stoer step evaluates the positions all its attempts share
// (x0, x0 + h/2, x0 + h) once.  Entries as in the plain build below.
template <int SYS> struct SysM;
template <> struct SysM<SYS_MINORS> { dz a, b, c, m23, m24; double rr, ro; };   // a = z2/r, b = 4 z1/r^2, c = N/r^2
template <> struct SysM<SYS_FLUID> { dz m12; double m11, ro; };
template <> struct SysM<SYS_RADIAL> { dz m11, m12, m21, m22; };
template <> struct SysM<SYS_TOROIDAL> { dz m12, m21; double rr; };
template <> struct SysM<SYS_SOLIDT> { dz z2, zrpc, w, c, a43; double rr, ro; };  // w = z1/r^2, c = N/r^2

template <int SYS>
__device__ __forceinline__ void sys_eval(const FKStatic& P, const EnvF& e, double x, SysM<SYS>& M) {
  double ro;
  dz el[7];
  const dz zom{e.omre, e.omim};
  const double dll1 = e.dll1;
  if constexpr (SYS == SYS_MINORS) {          // minorsOdeSystem.f90:77-126
    eval_spline<0x1Fu>(P, e, x, ro, el);
    const double rr = rinv(x), rr2 = rr * rr;
    const dz zrpc = zinv(el[1]);
    const dz z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
    M.a = ((2.0 * el[2]) * zrpc) * rr;
    M.b = (4.0 * z1) * rr2;
    M.c = el[4] * rr2;
    M.m23 = zinv(el[3]);
    M.m24 = zrpc;
    M.rr = rr;
    M.ro = ro;
  } else if constexpr (SYS == SYS_FLUID) {   // fluidOdeSystem.f90:78-95
    eval_spline<0x02u>(P, e, x, ro, el);
    const dz zomro = zom * zom * ro;
    M.m11 = -2.0 * rinv(x);
    M.m12 = zinv(el[1]) - dll1 * zinv((zomro * x) * x);
    M.ro = ro;
  } else if constexpr (SYS == SYS_RADIAL) {  // radialOdeSystem.f90:78-99
    eval_spline<0x17u>(P, e, x, ro, el);
    const dz zomro = zom * zom * ro;
    const double rr = rinv(x), rr2 = rr * rr;
    const dz rc = zinv(el[1]);
    M.m11 = ((-2.0 * el[2]) * rr) * rc;
    M.m12 = rc;
    M.m21 = (-zomro) + (4.0 * rr2) * ((el[0] - (el[2] * el[2]) * rc) - el[4]);
    M.m22 = (2.0 * rr) * (el[2] * rc - 1.0);
  } else if constexpr (SYS == SYS_TOROIDAL) {  // toroidalOdeSystem.f90:81-102
    eval_spline<0x18u>(P, e, x, ro, el);
    const dz zomro = zom * zom * ro;
    const double rr = rinv(x), rr2 = rr * rr;
    M.m12 = zinv(el[3]);
    M.m21 = (-zomro) - (el[4] * rr2) * (2.0 - dll1);
    M.rr = rr;
  } else {                                    // solidtOdeSystem.f90:77-114
    eval_spline<0x1Fu>(P, e, x, ro, el);
    const double rr = rinv(x), rr2 = rr * rr;
    const dz zrpc = zinv(el[1]);
    M.z2 = (el[2] * rr) * zrpc;
    M.zrpc = zrpc;
    M.w = (el[0] - (el[2] * el[2]) * zrpc - el[4]) * rr2;
    M.c = el[4] * rr2;
    M.a43 = -zinv(el[3]);
    M.rr = rr;
    M.ro = ro;
  }
}

template <int SYS>
__device__ __forceinline__ void sys_apply(const SysM<SYS>& M, const Env& e, const dz* z, dz* y) {
  const dz zom{e.omre, e.omim};
  const double dll1 = e.dll1;
  if constexpr (SYS == SYS_MINORS) {
    const dz zomro = zom * zom * M.ro;
    const double rr = M.rr, m11 = -2.0 * rr, m13 = dll1 * rr;
    const dz m12 = (-0.5 * dll1) * M.b;
    const dz m14 = (-0.5 * dll1) * M.a;
    const dz m22 = rr - M.a;
    const dz m32 = (-zomro) + (0.25 * dll1) * M.b + (dll1 - 2.0) * M.c;
    const dz m33 = (-3.0 * rr) - M.a;
    const dz m42 = (-zomro) + M.b;
    const dz m55 = M.a - 5.0 * rr;
    y[0] = m11 * z[0] + m12 * z[1] + m13 * z[2] + m14 * z[3];
    y[1] = m22 * z[1] + M.m23 * z[2] + M.m24 * z[3];
    y[2] = (-M.a) * z[0] + m32 * z[1] + m33 * z[2] + M.m24 * z[4];
    y[3] = (-m11) * z[0] + m42 * z[1] + (-m22) * z[3] + M.m23 * z[4];
    y[4] = M.b * z[0] + m42 * z[2] + m32 * z[3] + m55 * z[4];
  } else if constexpr (SYS == SYS_FLUID) {
    const dz zomro = zom * zom * M.ro;
    y[0] = M.m11 * z[0] + M.m12 * z[1];
    y[1] = (-zomro) * z[0];
  } else if constexpr (SYS == SYS_RADIAL) {
    y[0] = M.m11 * z[0] + M.m12 * z[1];
    y[1] = M.m21 * z[0] + M.m22 * z[1];
  } else if constexpr (SYS == SYS_TOROIDAL) {
    y[0] = M.rr * z[0] + M.m12 * z[1];
    y[1] = M.m21 * z[0] + (-3.0 * M.rr) * z[1];
  } else {
    const dz zomro = zom * zom * M.ro;
    const double rr = M.rr, rr2 = rr * rr;
    const dz a11 = 2.0 * M.z2;
    const dz a12 = zomro - 4.0 * M.w;
    const dz a22 = (-a11) + 2.0 * rr;
    const dz a32 = (2.0 * dll1) * M.w;
    const dz a34 = zomro - (dll1 * M.w + (dll1 - 2.0) * M.c);
    (void)rr2;
    y[0] = a11 * z[0] + a12 * z[1] + rr * z[2] + (2.0 * M.w) * z[3];
    y[1] = (-M.zrpc) * z[0] + a22 * z[1] + M.z2 * z[3];
    y[2] = ((-dll1) * M.z2) * z[0] + a32 * z[1] + (-rr) * z[2] + a34 * z[3];
    y[3] = ((-dll1) * rr) * z[1] + M.a43 * z[2] + (3.0 * rr) * z[3];
  }
}

template <int SYS>
__device__ __forceinline__ void apply_sys(const FKStatic& P, const EnvF& e, double x, const dz* z, dz* y) {
  SysM<SYS> M;
  sys_eval<SYS>(P, e, x, M);
  sys_apply<SYS>(M, e, z, y);
}
#else
template <int SYS>
__device__ __forceinline__ void apply_sys(const FKStatic& P, const Env& e, double x, const dz* z, dz* y) {
  double ro;
  dz el[7];
  dz zom{e.omre, e.omim};
  double dll1 = e.dll1;
  if (SYS == SYS_MINORS) {          // minorsOdeSystem.f90:77-126
    eval_spline<0x1Fu>(P, e, x, e.nl, ro, el);
    dz zomro = zom * zom * ro;
    double rr = rinv(x), rr2 = rr * rr;
    dz zrpc = zinv(el[1]);
    dz z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
    dz z2 = (2.0 * el[2]) * zrpc;
    dz z3 = (4.0 * z1) * rr2;
    double m11 = -2.0 * rr;
    dz m12 = ((-2.0 * dll1) * z1) * rr2;
    double m13 = dll1 * rr;
    dz m14 = (((-dll1) * el[2]) * zrpc) * rr;
    dz m22 = (1.0 - z2) * rr;
    dz m23 = zinv(el[3]);
    dz m24 = zrpc;
    dz m31 = (-z2) * rr;
    dz m32 = (-zomro) + ((dll1 * (z1 + el[4])) - 2.0 * el[4]) * rr2;
    dz m33 = (-(3.0 + z2)) * rr;
    double m41 = -m11;
    dz m42 = (-zomro) + z3;
    dz m55 = (z2 - 5.0) * rr;
    y[0] = m11 * z[0] + m12 * z[1] + m13 * z[2] + m14 * z[3];
    y[1] = m22 * z[1] + m23 * z[2] + m24 * z[3];
    y[2] = m31 * z[0] + m32 * z[1] + m33 * z[2] + m24 * z[4];
    y[3] = m41 * z[0] + m42 * z[1] + (-m22) * z[3] + m23 * z[4];
    y[4] = z3 * z[0] + m42 * z[2] + m32 * z[3] + m55 * z[4];
  } else if (SYS == SYS_FLUID) {    // fluidOdeSystem.f90:78-95
    eval_spline<0x02u>(P, e, x, e.nl, ro, el);
    dz zomro = zom * zom * ro;
    double m11 = -2.0 / x;
    dz m12 = 1.0 / el[1] - dll1 / ((zomro * x) * x);
    y[0] = m11 * z[0] + m12 * z[1];
    y[1] = (-zomro) * z[0];
  } else if (SYS == SYS_RADIAL) {   // radialOdeSystem.f90:78-99
    eval_spline<0x17u>(P, e, x, e.nl, ro, el);
    dz zomro = zom * zom * ro;
    double rr = rinv(x), rr2 = rr * rr;
    dz m11 = ((-2.0 * el[2]) * rr) / el[1];
    dz m12 = 1.0 / el[1];
    dz m21 = (-zomro) + (4.0 * rr2) * ((el[0] - (el[2] * el[2]) / el[1]) - el[4]);
    dz m22 = (2.0 * rr) * (el[2] / el[1] - 1.0);
    y[0] = m11 * z[0] + m12 * z[1];
    y[1] = m21 * z[0] + m22 * z[1];
  } else if (SYS == SYS_TOROIDAL) { // toroidalOdeSystem.f90:81-102
    eval_spline<0x18u>(P, e, x, e.nl, ro, el);
    dz zomro = zom * zom * ro;
    double rr = rinv(x), rr2 = rr * rr;
    dz m12 = zinv(el[3]);
    dz m21 = (-zomro) - (el[4] * rr2) * (2.0 - dll1);
    y[0] = rr * z[0] + m12 * z[1];
    y[1] = m21 * z[0] + (-3.0 * rr) * z[1];
  } else {                          // solidtOdeSystem.f90:77-114
    eval_spline<0x1Fu>(P, e, x, e.nl, ro, el);
    dz zomro = zom * zom * ro;
    double rr = rinv(x), rr2 = rr * rr;
    dz zrpc = zinv(el[1]);
    dz z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
    dz z2 = (el[2] * rr) * zrpc;
    dz zdlz1 = dll1 * z1;
    dz a11 = 2.0 * z2;
    dz a21 = -zrpc;
    dz a31 = (-dll1) * z2;
    dz a12 = zomro - (4.0 * z1) * rr2;
    dz a22 = (-a11) + 2.0 * rr;
    dz a32 = (2.0 * rr2) * zdlz1;
    double a42 = (-dll1) * rr;
    dz a43 = -zinv(el[3]);
    dz a14 = (2.0 * z1) * rr2;
    dz a34 = zomro - (zdlz1 + (dll1 - 2.0) * el[4]) * rr2;
    y[0] = a11 * z[0] + a12 * z[1] + rr * z[2] + a14 * z[3];
    y[1] = a21 * z[0] + a22 * z[1] + z2 * z[3];
    y[2] = a31 * z[0] + a32 * z[1] + (-rr) * z[2] + a34 * z[3];
    y[3] = a42 * z[1] + a43 * z[2] + (3.0 * rr) * z[3];
  }
}
#endif

// ------------------------------------------------------------------------
//  Bulirsch-Stoer full step (complexBulirschStep.f90:111-240,297-340)
// ------------------------------------------------------------------------
#if GEM_FAST
// The 2-variable systems keep the matrices at x0 + h/2 and x0 + h across the
// attempts of a step; the 5- and 4-variable systems do when BIG is set (a
// schedule choice: at 384-512 threads per block the held matrices cost more in
// spilled registers than evaluating them again, at 256 they do not).
template <int SYS, bool BIG> struct SysCache {
  static constexpr bool value = BIG || SYS == SYS_TOROIDAL || SYS == SYS_FLUID || SYS == SYS_RADIAL;
};

// Neville coefficients of the fast build.  With x_k = h / n_k, the update of
// level m of diagonal p, u = (c - d) / (x_{p-m} - x_p), c' = x_{p-m} u,
// d' = x_p u, is c' = a (c - d), d' = b (c - d) with a = n_p / (n_p - n_{p-m})
// and b = n_{p-m} / (n_p - n_{p-m}): h cancels, so no division is left.
struct NevTab {
  double a[7][7], b[7][7];
};
constexpr NevTab make_nev() {
  const int n[7] = {2, 4, 6, 8, 12, 16, 24};
  NevTab t{};
  for (int p = 1; p < 7; ++p)
    for (int m = 1; m <= p; ++m) {
      t.a[p][m] = (double)n[p] / (double)(n[p] - n[p - m]);
      t.b[p][m] = (double)n[p - m] / (double)(n[p] - n[p - m]);
    }
  return t;
}
__device__ __constant__ const NevTab NEV = make_nev();

// Modified midpoint of attempt jtry with t0 = A(xstart) y0 given (in memory), and with
// CACHE the matrices at xstart + h/2 (Mh) and xstart + h (Me): the parts every
// attempt of a step shares.  The grid point g (in 48ths of the step) sits at
// xstart + g h48, h48 = h / 48 rounded once per step.
template <int SYS, bool CACHE>
__device__ __forceinline__ void midpoint(const FKStatic& P, const EnvF& e, int jtry, double h48, double xstart,
                                         const dz* y0, const Slot& t0, const SysM<SYS>& Mh, const SysM<SYS>& Me,
                                         dz* out) {
  constexpr int NV = SysNV<SYS>::NV;
  const int nstep = SEQDIV[jtry - 1];
  const int dix = 48 / nstep;
  const double hdiv = (double)dix * h48;
  dz z0[NV], z1[NV], t[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { z0[v] = y0[v]; z1[v] = y0[v] + hdiv * t0.get(v); }
  const double h2 = 2.0 * hdiv;
  for (int m = 1; m <= nstep - 1; ++m) {
    if (CACHE && m * dix == 24) {
      sys_apply<SYS>(Mh, e, z1, t);
    } else {
      const double x = xstart + (double)(m * dix) * h48;
      apply_sys<SYS>(P, e, x, z1, t);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      dz z2 = z0[v] + h2 * t[v];
      z0[v] = z1[v];
      z1[v] = z2;
    }
  }
  if constexpr (CACHE) sys_apply<SYS>(Me, e, z1, t);
  else apply_sys<SYS>(P, e, xstart + 48.0 * h48, z1, t);
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = 0.5 * ((z1[v] + z0[v]) + hdiv * t[v]);
}
#else
template <int SYS>
__device__ __forceinline__ void midpoint(const FKStatic& P, const Env& e, int jtry, double h, double xstart,
                                         const dz* y0, dz* out) {
  constexpr int NV = SysNV<SYS>::NV;
  const int nstep = SEQDIV[jtry - 1];
  const double hdiv = h / (double)nstep;
  const int dix = 48 / nstep;
  dz z0[NV], z1[NV], t[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) z0[v] = y0[v];
  apply_sys<SYS>(P, e, xstart + (0.0 * h) / 48.0, z0, t);
#pragma unroll
  for (int v = 0; v < NV; ++v) z1[v] = z0[v] + hdiv * t[v];
  const double h2 = 2.0 * hdiv;
  for (int m = 1; m <= nstep - 1; ++m) {
    double x = xstart + ((double)(m * dix) * h) / 48.0;
    apply_sys<SYS>(P, e, x, z1, t);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      dz z2 = z0[v] + h2 * t[v];
      z0[v] = z1[v];
      z1[v] = z2;
    }
  }
  apply_sys<SYS>(P, e, xstart + (48.0 * h) / 48.0, z1, t);
#pragma unroll
  for (int v = 0; v < NV; ++v) out[v] = 0.5 * ((z1[v] + z0[v]) + hdiv * t[v]);
}
#endif

// ------------------------------------------------------------------------
//  Nodes and discontinuities inside an integration range
//  (geminiIntegrationEnvironment.f90:96-203); returns index bounds only.
// ------------------------------------------------------------------------
__device__ __forceinline__ void disco_range(const FKStatic& P, double x1, double x2, int& jl, int& jr) {
  double xl = x1, xr = x2;
  if (x1 > x2) { xl = x2; xr = x1; }
  int n = P.nlay;
  jl = locate(xl, n, P.rb) + 1;
  if (jl > n) { jr = jl - 1; return; }
  if (fabs(1.0 - xl / P.rb[jl]) < EPS_D) jl = jl + 1;
  if (jl >= n) { jr = jl - 1; return; }
  jr = locate(xr, n, P.rb);
  if (jr == 0) { jr = 0; jl = 1; }
}

__device__ __forceinline__ void node_range(const FKStatic& P, double x1, double x2, int& jl, int& jr) {
  double xl = x1, xr = x2;
  if (x1 > x2) { xl = x2; xr = x1; }
  int n = P.nnod;
  jl = locate(xl, n, P.rnod) + 1;
  if (jl > n) { jr = jl - 1; return; }
  jr = locate(xr, n, P.rnod);
  if (jr < n) { if (fabs(1.0 - xr / P.rnod[jr + 1]) < EPS_D) jr = jr + 1; }
  if (jr == 0) { jr = 0; jl = 1; }
}

// ------------------------------------------------------------------------
//  Start radius (initialValues.f90:71-192)
// ------------------------------------------------------------------------
__device__ __forceinline__ double velocity_at(const FKStatic& P, const Env& e, double r, int nl) {
  double ro; dz el[7];
  eval_spline<0x60u>(P, e, r, nl, ro, el);
  double v = sqrt(el[6].re / ro);
  if (P.iflso[nl] == 1) v = sqrt(el[5].re / ro);
  return v;
}
__device__ __forceinline__ double vslow(double om, double dll1, double r, double v) {
  return dll1 / (r * r) - (om / v) * (om / v);
}
__device__ double integrate_slowness(const FKStatic& P, const Env& e, double rturn, double dr, bool tor) {
  double q = 0.0, r = rturn;
  double rbot = (tor && P.hascore) ? P.roc : P.rhs - TENTH_F * dr;
  const double qmax = -log(1.e-5);
  while (q < qmax) {
    if (r - dr < rbot) { r = rbot; break; }
    r = r - dr;
    int nl, top;
    layer_index(P, r, nl, top);
    double v = velocity_at(P, e, r, nl);
    q = q + dr * sqrt(vslow(e.omre, e.dll1, r, v));
  }
  return r;
}
__device__ double start_radius(const FKStatic& P, const Env& e, bool tor) {
  double r; int nl;
  if (tor && P.hascore) { r = P.roc; nl = P.noc + 1; } else { r = P.rhs; nl = 1; }
  double dr = (P.rearth - r) / 400.0;
  double v = velocity_at(P, e, r, nl);
  double p = vslow(e.omre, e.dll1, r, v), pold = p;
  if (p <= 0.0) {
    if (tor && P.hascore) return P.roc;
    return P.rhs - TENTH_F * dr;
  }
  double rmax = (tor && P.hasocean) ? P.ruc : P.rearth;
  while (p > 0.0) {
    pold = p;
    if (fabs(1.0 - r / rmax) < EPS_D) return integrate_slowness(P, e, rmax, dr, tor);
    r = fmin(r + dr, rmax);
    int top;
    layer_index(P, r, nl, top);
    v = velocity_at(P, e, r, nl);
    p = vslow(e.omre, e.dll1, r, v);
  }
  double rturn = r - dr * p / (p - pold);
  return integrate_slowness(P, e, rturn, dr, tor);
}

// ------------------------------------------------------------------------
//  Continued fractions (initialValues.f90:487-574)
// ------------------------------------------------------------------------
__device__ int sphancf(dz zx, double el, int kindhf, dz& zf) {
  const double tiny = 1.e-30, eps = 1.e-6;
  zf = dz{tiny, 0.0};
  dz zc = zf, zd{0.0, 0.0};
  double elph2 = (el + 0.5) * (el + 0.5);
  int j;
  for (j = 1; j <= 10000; ++j) {
    dz zb = 2.0 * (zx + dz{0.0, (double)j});
    double za = ((double)j - 0.5) * ((double)j - 0.5) - elph2;
    zd = zb + za * zd;
    if (zabs(zd) < tiny) zd = dz{tiny, 0.0};
    zc = zb + za / zc;
    if (zabs(zc) < tiny) zc = dz{tiny, 0.0};
    zd = 1.0 / zd;
    dz zdelta = zc * zd;
    zf = zf * zdelta;
    if (zabs(zdelta - 1.0) < eps) break;
  }
  if (j > 10000) return ST_CF;
  const dz ci{0.0, 1.0};
  if (kindhf == 1) zf = ((el + 1.0) - ci * zx) - ci * zf;
  else zf = ((el + 1.0) + ci * zx) + ci * zf;
  return ST_OK;
}

__device__ int zetl(dz zx2, double el, dz& z) {
  const double tiny = 1.e-30, eps = 1.e-6;
  z = dz{tiny, 0.0};
  dz zd{2.0 * el + 3.0, 0.0};
  dz zc = zd + zx2 / z;
  zd = 1.0 / zd;
  dz zdelta = zc * zd;
  z = z * zdelta;
  for (int i = 2; i <= 10000; ++i) {
    zd = (2.0 * (el + (double)i) + 1.0) - zx2 * zd;
    if (zd.re == 0.0 && zd.im == 0.0) zd = dz{tiny, 0.0};
    zc = (2.0 * (el + (double)i) + 1.0) - zx2 / zc;
    if (zc.re == 0.0 && zc.im == 0.0) zc = dz{tiny, 0.0};
    zd = 1.0 / zd;
    zdelta = zc * zd;
    z = z * zdelta;
    if (fabs(zabs(zdelta) - 1.0) < eps) return ST_OK;
  }
  return ST_CF;
}

// minors start vector from the ratio functions (initialValues.f90:258-274, 329-346)
__device__ __forceinline__ void minors_from_ratios(bool liquid, double el, double elp1, double r, double ro,
                                                   dz zom, const dz* el7, dz zeta, dz zetb, dz zxb2, dz* ys) {
  if (el < EPS_D) {
    ys[0] = -zeta;
    ys[1] = (((-ro) * r) * zom) * zom + ((4.0 * el7[6]) / r) * zeta;
  } else if (liquid) {
    ys[0] = (-(1.0 - zeta / el)) / (((zom * zom) * ro) * r);
    ys[1] = dz{1.0 / el, 0.0};
  } else {
    dz za = zeta / el;
    dz zb = zetb / (el + 1.0);
    ys[1] = ((-za) + zb * (za - 1.0)) / el;
    dz mr = el7[6] / r;
    ys[0] = mr * (zxb2 / el + (2.0 * elp1) * ys[1]);
    ys[2] = mr * ((-2.0) * ys[1] + (zxb2 / elp1) * (za - 1.0));
    ys[3] = (-mr) * ((zxb2 / (el * el)) * (1.0 - zb) + 4.0 * ys[1]);
    ys[4] = ((el7[6] * el7[6]) / (r * r)) *
            ((((-4.0) * (el - 1.0)) * (el + 2.0)) * ys[1] +
             (zxb2 / el) * ((((zxb2 / elp1) - ((2.0 * (el - 1.0)) * (2.0 * el + 1.0)) / elp1) -
                             (4.0 / (el + 1.0)) * za) - (2.0 / el) * zb));
  }
}

// minorsBottomInitialValues (initialValues.f90:202-275)
__device__ int minors_bottom_iv(const FKStatic& P, const Env& e, double rstart, dz* ys, double& htry) {
  double ro; dz el7[7];
  eval_spline<0x7Fu>(P, e, rstart, e.nl, ro, el7);
  bool liquid = P.iflso[e.nl] == 1;
  double el = -0.5 + sqrt(0.25 + e.dll1);
  double elp1 = e.dll1;
  dz zom{e.omre, e.omim};
  double rsq = rstart * rstart;
  double v = sqrt(el7[6].re / ro);
  if (liquid) v = sqrt(el7[5].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  dz zxa2 = (((ro * zom) * zom) * rsq) / (el7[5] + (4.0 * el7[6]) / 3.0);
  dz zeta{0, 0}, zetb{0, 0}, zxb2{0, 0};
  int rc;
  if (el < EPS_D) {
    rc = zetl(zxa2, el, zeta); if (rc) return rc;
  } else {
    if (zabs(zxa2 / elp1) <= 1.0) rc = zetl(zxa2, el, zeta);
    else rc = sphancf(zsqrt(zxa2), el, 1, zeta);
    if (rc) return rc;
    if (!liquid) {
      zxb2 = (((ro * zom) * zom) * rsq) / el7[6];
      if (zabs(zxb2 / elp1) <= 1.0) rc = zetl(zxb2, el, zetb);
      else rc = sphancf(zsqrt(zxb2), el, 1, zetb);
      if (rc) return rc;
    }
  }
  minors_from_ratios(liquid, el, elp1, rstart, ro, zom, el7, zeta, zetb, zxb2, ys);
  return ST_OK;
}

// minorsSurfaceInitialValues (initialValues.f90:287-367)
__device__ int minors_surface_iv(const FKStatic& P, const Env& e, dz* ys, double& htry) {
  int nlay = P.nlay;
  double elp1 = e.dll1;
  double el = -0.5 + sqrt(0.25 + elp1);
  double rearth = P.rearth;
  dz zom{e.omre, e.omim};
  bool liquid = P.iflso[nlay] == 1;
  double ro; dz el7[7];
  eval_spline<0x7Fu>(P, e, rearth, nlay, ro, el7);
  double v = sqrt(el7[6].re / ro);
  if (liquid) v = sqrt(el7[5].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (P.fsflag == 1) {
    double rsq = rearth * rearth;
    dz zxa2 = (((ro * zom) * zom) * rsq) / (el7[5] + (4.0 * el7[6]) / 3.0);
    dz zeta, zetb{0, 0}, zxb2{0, 0};
    int rc = sphancf(zsqrt(zxa2), el, 2, zeta); if (rc) return rc;
    if (!liquid) {
      zxb2 = (((ro * zom) * zom) * rsq) / el7[6];
      rc = sphancf(zsqrt(zxb2), el, 2, zetb); if (rc) return rc;
    }
    minors_from_ratios(liquid, el, elp1, rearth, ro, zom, el7, zeta, zetb, zxb2, ys);
  } else {
    if (el < EPS_F || liquid) { ys[0] = dz{1.0, 0.0}; ys[1] = dz{0.0, 0.0}; }
    else { ys[0] = dz{0, 0}; ys[1] = dz{1.0, 0.0}; ys[2] = dz{0, 0}; ys[3] = dz{0, 0}; ys[4] = dz{0, 0}; }
  }
  return ST_OK;
}

// toroidalBottomInitialValues (initialValues.f90:376-418)
__device__ int toroidal_bottom_iv(const FKStatic& P, const Env& e, double rstart, dz* ys, double& htry) {
  double ro; dz el7[7];
  eval_spline<0x40u>(P, e, rstart, e.nl, ro, el7);
  double el = -0.5 + sqrt(0.25 + e.dll1);
  double elp1 = e.dll1;
  dz zom{e.omre, e.omim};
  double rsq = rstart * rstart;
  double v = sqrt(el7[6].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (rstart > P.roc) {
    dz zxb2 = (((ro * zom) * zom) * rsq) / el7[6], zetb;
    int rc;
    if (zabs(zxb2 / elp1) < 1.0) rc = zetl(zxb2, el, zetb);
    else rc = sphancf(zsqrt(zxb2), el, 1, zetb);
    if (rc) return rc;
    ys[0] = dz{1.0 / el, 0.0};
    ys[1] = (el7[6] / (rstart * el)) * ((el - 1.0) - zetb);
  } else {
    ys[0] = dz{1.0 / el, 0.0};
    ys[1] = dz{0.0, 0.0};
  }
  return ST_OK;
}

// toroidalSurfaceInitialValues (initialValues.f90:434-469)
__device__ int toroidal_surface_iv(const FKStatic& P, const Env& e, dz* ys, double& htry, double& rsurf,
                                   int& nl) {
  if (P.hasocean) { nl = P.nlay - 1; rsurf = P.ruc; } else { nl = P.nlay; rsurf = P.rearth; }
  double el = -0.5 + sqrt(0.25 + e.dll1);
  dz zom{e.omre, e.omim};
  double ro; dz el7[7];
  eval_spline<0x40u>(P, e, rsurf, nl, ro, el7);
  double v = sqrt(el7[6].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (P.fsflag == 1) {
    double rsq = rsurf * rsurf;
    dz zxb2 = (((ro * zom) * zom) * rsq) / el7[6], zetb;
    int rc = sphancf(zsqrt(zxb2), el, 2, zetb); if (rc) return rc;
    ys[0] = dz{1.0 / el, 0.0};
    ys[1] = (el7[6] / (rsurf * el)) * ((el - 1.0) - zetb);
  } else {
    ys[0] = dz{1.0, 0.0}; ys[1] = dz{0.0, 0.0};
  }
  return ST_OK;
}

}  // namespace GEM_NS
