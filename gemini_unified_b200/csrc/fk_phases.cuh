// FK solver as three warp-lockstep phase kernels (K1 + K2 fused per phase).
//
// The reference runs, for every (omega, l), the toroidal minors, the
// spheroidal minors and the unit-jump Green functions back to back
// (computeGreenFKSpectraForSynthetics.f90:424-494).  Here each of the three
// becomes its own persistent kernel over all items of a frequency slab:
//
//   fk_setup_kernel   start radii of both motion types (initialValues.f90:71-192)
//   PH_TOR            toroidal minors (toroidalMinors.f90:71-268), toroidal
//                     unit-jump Green functions (unitJumpGreenFunctions.f90:147-175)
//                     and the toroidal spectra of every node;
//   PH_SPH            spheroidal minors up and down (spheroidalMinors.f90:72-585);
//                     minors below/above the receiver and the determinant go to
//                     per-item storage in HBM;
//   PH_ADJ            spheroidal adjoint integrations (spheroidalAdjoint.f90),
//                     unit-jump Green functions (unitJumpGreenFunctions.f90:201-372),
//                     reciprocity and source terms, spheroidal spectra.
//
// Inside a phase every lane of a warp integrates the same kind of ODE system,
// so the lockstep Bulirsch-Stoer step keeps the whole warp busy: lanes refill
// from the phase's work queue as soon as their item is done.  Each lane walks
// its item as a small state machine (bookkeeping runs divergently between two
// lockstep steps).  The Neville tableau is built incrementally, one new
// diagonal per attempt (the exact values the reference recomputes from
// scratch), and kept in shared memory, lane-interleaved.
#pragma once
#include "fk_kernel.h"
#include "fk_solver.cuh"

namespace GEM_NS {

enum : int { PH_TOR = 0, PH_SPH = 1, PH_ADJ = 2 };
template <int PH> struct PhaseNV { static constexpr int NV = PH == PH_TOR ? 2 : (PH == PH_SPH ? 5 : 4); };
// levels 0..5 of the per-lane Neville diagonal feed the last attempt; the
// levels below PhaseDiag::L live in shared memory, the rest (read only by the
// seventh attempt) in the lane's registers or stack
template <int PH, int BLK> struct PhaseDiag { static constexpr int L = (PH == PH_SPH && BLK > 384) ? 5 : 6; };

// lane states
enum : int {
  S_FETCH = 0, S_IDLE, S_ITEM_INIT, S_TOR_UP, S_TOR_DONE, S_SPH_GROUP, S_SPH_GROUP_END, S_ADJ_PLAN,
  S_ADJ_NEXT, S_ADJ_END, S_OUTPUT, S_ITEM_END, S_PROP_NEXT, S_SUB_END, S_INTEG
};
// node sinks
enum : int { K_DT = 0, K_UT, K_UM, K_DM, K_ADJIC, K_ADJ_UP, K_ADJ_DN };

// per-lane scratch slot (element-major across the lanes of the grid)
struct LaneLayout {
  int NN;
  __device__ __forceinline__ int ut(int n, int c) const { return n * 2 + c; }
  __device__ __forceinline__ int dt(int n, int c) const { return 2 * NN + n * 2 + c; }
  __device__ __forceinline__ int lg(int n) const { return n; }                       // spheroidal phase
  __device__ __forceinline__ int sph(int n, int j, int c) const { return n * 16 + j * 4 + c; }   // adjoint phase
  __device__ __forceinline__ int adjic(int n, int c) const { return 16 * NN + n * 4 + c; }
  static constexpr int PER_NODE = 20;
};

struct Lane {
  int st, status;
  int k;                // item index = output index k of the slab
  int iwn;
  Env e;
  double rstart_t, rstart_s;
  dz det;
  // spheroidal groups
  int up, liq, liq_old;
  double rbeg, rend, rlim, lgnorm_g, lgnormend, htry_g;
  dz yend[5];
  // adjoints
  int stage, core_below, ocean_above, lowest, highest;
  double re_dn;
  // current propagation
  int sys, nv, sink, after, do_norm;
  int jl, jr, dl, dr, nnodp, ndp, jnod, jd, kmin, nstep;
  double x1, x2, xa, xe, x, h, hdid, lgnorm, s0, s1, idir;
  int kopt;   // target attempt of the step-size control
  double hs;  // multiplier of the initial steps given by the initial-value formulas
  dz y[5];
  unsigned qnext, qend;   // queue positions reserved by the lane and not yet taken
};

// ------------------------------------------------------------------------
//  Per-item storage between the phases (HBM, element-major over items)
// ------------------------------------------------------------------------
struct ItemStore {
  const FKLaunch* LL;
  __device__ __forceinline__ dz um(int k, int n, int c) const {   // n = 1..jre
    double2 v = LL->um[((long long)(n - 1) * 6 + c) * LL->nkf + k];
    return dz{v.x, v.y};
  }
  __device__ __forceinline__ void put_um(int k, int n, int c, dz v) const {
    LL->um[((long long)(n - 1) * 6 + c) * LL->nkf + k] = make_double2(v.re, v.im);
  }
  __device__ __forceinline__ dz dm(int k, int n, int c, int jre) const {   // n = jre..nnod (jre: P.jsl)
    double2 v = LL->dm[((long long)(n - jre) * 6 + c) * LL->nkf + k];
    return dz{v.x, v.y};
  }
  __device__ __forceinline__ void put_dm(int k, int n, int c, int jre, dz v) const {
    LL->dm[((long long)(n - jre) * 6 + c) * LL->nkf + k] = make_double2(v.re, v.im);
  }
};

// Reference-algorithm work of a step whose lane made attempts 1..j: sub-step
// matrix-vector products (mv), system matrices on the 1/48 grid (sm), and the
// extrapolation flops from the third attempt on for NV variables (ext) -- the
// oracle's accounting, summed once per step from these tables.
struct StepWork {
  int mv[8], sm[8], ext[6][8];
};
constexpr StepWork make_stepwork() {
  const int seq[7] = {2, 4, 6, 8, 12, 16, 24}, nx[7] = {3, 2, 4, 4, 4, 8, 8};
  StepWork w{};
  for (int j = 1; j <= 7; ++j) {
    w.mv[j] = w.mv[j - 1] + seq[j - 1] + 1;
    w.sm[j] = w.sm[j - 1] + nx[j - 1];
    for (int nv = 0; nv < 6; ++nv)
      w.ext[nv][j] = w.ext[nv][j - 1] + (j >= 3 ? (j * (j - 1) / 2) * 8 * nv + (j - 1) * 2 * nv + 8 * nv + 3 : 0);
  }
  return w;
}
__device__ __constant__ const StepWork STEPWORK = make_stepwork();

// ------------------------------------------------------------------------
//  Lockstep Bulirsch-Stoer step of all lanes with `active` set
//  (complexBulirschStep.f90:111-170,180-238,297-340)
// ------------------------------------------------------------------------
template <int SYS, int NVD, int DL, bool BIG>
__device__ __noinline__ void bs_step(const FKStatic& P, const Env& e_in, bool active, double h, double x,
                                     const dz* y0, dz* yext, int& result, double2* D, int lane, const Slot& xs,
                                     Counters& cnt_out) {
  constexpr int NV = SysNV<SYS>::NV;
  // the lane state lives in local memory: work on a register copy of the
  // environment; the counters follow from the attempts made (added at the end)
#if GEM_FAST
  const EnvF e = make_envf(P, e_in, active);
#else
  const Env e = e_in;
#endif
  int lane_att = 0, warp_att = 0, jdone = 0;
  bool need = active;
  int res = 0;   // 0: failed; > 0: number of attempts of a successful step
#if GEM_FAST
  // What every attempt shares: y0 (read from the lane state), A(x) y0 and the
  // matrices at x + h/2 and x + h.  y0 and A(x) y0 are read once per attempt,
  // so they stay in memory (A(x) y0 in the lane's scratch elements 0..4)
  // instead of holding 20 registers each through the sub-step loop.
  constexpr bool CACHE = SysCache<SYS, BIG>::value;
  SysM<SYS> Mh, Me;
  const double h48 = h / 48.0;   // grid spacing of the step's sub-steps
  if (need) {
    dz ys[NV], t0[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ys[v] = y0[v];
    apply_sys<SYS>(P, e, x, ys, t0);
#pragma unroll
    for (int v = 0; v < NV; ++v) xs.put(v, t0[v]);
    if constexpr (CACHE) {
      sys_eval<SYS>(P, e, x + 24.0 * h48, Mh);
      sys_eval<SYS>(P, e, x + 48.0 * h48, Me);
    }
  }
#else
  (void)xs;
  dz ys[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) ys[v] = y0[v];
#endif
  dz dlast[NV];   // diagonal level DL when DL < 6 (fast build: scratch elements 5..9)
  for (int j = 1; j <= 7; ++j) {
    unsigned needm = __ballot_sync(0xffffffffu, need);
    if (!needm) break;
    lane_att += __popc(needm);
    warp_att += 1;
    if (!need) continue;
    dz Y[NV];
#if GEM_FAST
    midpoint<SYS, CACHE>(P, e, j, h48, x, y0, xs, Mh, Me, Y);
#else
    midpoint<SYS>(P, e, j, h, x, ys, Y);
#endif
    jdone = j;
    // new diagonal of the Neville tableau for point p = j-1 (0-based)
    const int p = j - 1;
    dz yy[NV], dy[NV], c[NV], pend[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { yy[v] = Y[v]; c[v] = Y[v]; pend[v] = Y[v]; dy[v] = dz{0.0, 0.0}; }
#if GEM_FAST
    for (int m = 1; m <= p; ++m) {
      const double na = NEV.a[p][m], nb = NEV.b[p][m];
#else
    const double xp = h / (double)SEQDIV[p];
    for (int m = 1; m <= p; ++m) {
      const double xi = h / (double)SEQDIV[p - m];
      const double hh = xi - xp;
#endif
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const bool shared_level = DL == 6 || m - 1 < DL;
        double2* slot = D + ((m - 1) * NVD + v) * 32 + lane;
#if GEM_FAST
        dz pv = shared_level ? dz{0.0, 0.0} : xs.get(5 + v);
#else
        dz pv = dlast[v];
#endif
        if (shared_level) { double2 q = *slot; pv = dz{q.x, q.y}; }
#if GEM_FAST
        const dz u = c[v] - pv;
        c[v] = na * u;
        dz nd = nb * u;
#else
        dz u = (c[v] - pv) / hh;
        c[v] = xi * u;
        dz nd = xp * u;
#endif
        if (shared_level) *slot = make_double2(pend[v].re, pend[v].im);   // level m-1 of the new diagonal
#if GEM_FAST
        else xs.put(5 + v, pend[v]);
#else
        else dlast[v] = pend[v];
#endif
        pend[v] = nd;
        yy[v] = yy[v] + nd;
        dy[v] = nd;
      }
    }
    if (p < DL) {
#pragma unroll
      for (int v = 0; v < NV; ++v) D[(p * NVD + v) * 32 + lane] = make_double2(pend[v].re, pend[v].im);
    } else if (p < 6) {
#if GEM_FAST
#pragma unroll
      for (int v = 0; v < NV; ++v) xs.put(5 + v, pend[v]);
#else
#pragma unroll
      for (int v = 0; v < NV; ++v) dlast[v] = pend[v];
#endif
    }
    if (j >= 3) {
      double s1 = 0.0, s2 = 0.0;
#if GEM_FAST
#pragma unroll
      for (int v = 0; v < NV; ++v) s1 += dy[v].re * dy[v].re + dy[v].im * dy[v].im;
#pragma unroll
      for (int v = 0; v < NV; ++v) s2 += yy[v].re * yy[v].re + yy[v].im * yy[v].im;
      const bool conv = s1 < (P.eps * P.eps) * s2;
#else
#pragma unroll
      for (int v = 0; v < NV; ++v) { double a = zabs(dy[v]); s1 += a * a; }
#pragma unroll
      for (int v = 0; v < NV; ++v) { double a = zabs(yy[v]); s2 += a * a; }
      double errmax = sqrt(s1 / s2);
      const bool conv = errmax / P.eps < 1.0;
#endif
      if (conv) {
#pragma unroll
        for (int v = 0; v < NV; ++v) yext[v] = yy[v];
        res = j;
        need = false;
      } else if (j == 7) {
        need = false;
      }
    }
  }
  result = res;
  const int mv = STEPWORK.mv[jdone], sm = STEPWORK.sm[jdone];
  cnt_out.lane_attempts += lane_att;
  cnt_out.warp_attempts += warp_att;
  cnt_out.attempts += jdone;
  cnt_out.matvecs += mv;
  cnt_out.sysmats += sm;
  cnt_out.flops += (long long)sm * FLOP_SYSMAT[SYS] + (long long)mv * FLOP_MV[SYS] + STEPWORK.ext[NV][jdone];
}

// ------------------------------------------------------------------------
//  Helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ double above_pc(const FKStatic& P, int nl) {   // nodeEarthmodel.f90:616-636
  int npc;
  if (P.iflso[nl] == 1) npc = nl;
  else if (nl < P.noc) npc = P.noc - 1;
  else if (nl > P.noc) npc = P.iflso[P.nlay] == 1 ? P.nlay - 1 : P.nlay;
  else npc = P.nlay;
  return P.rb[npc];
}
__device__ __forceinline__ double below_pc(const FKStatic& P, int nl) {   // nodeEarthmodel.f90:645-663
  int npc;
  if (P.iflso[nl] == 1) npc = nl;
  else if (nl < P.noc) npc = 1;
  else if (nl > P.noc) npc = P.noc + 1;
  else npc = nl;
  return P.rb[npc - 1];
}

// 4x4 minor matrices from the six minors (spheroidalMinors.f90:306-323):
// mtil = [[0,m1,m2,m3],[-m1,0,m4,m5],[-m2,-m4,0,m6],[-m3,-m5,-m6,0]]
__device__ __forceinline__ void mtil_times(const dz* m, const dz* a, dz* out) {
  out[0] = m[0] * a[1] + m[1] * a[2] + m[2] * a[3];
  out[1] = (-m[0]) * a[0] + m[3] * a[2] + m[4] * a[3];
  out[2] = (-m[1]) * a[0] + (-m[3]) * a[1] + m[5] * a[3];
  out[3] = (-m[2]) * a[0] + (-m[4]) * a[1] + (-m[5]) * a[2];
}
// column j of meps = [[0,m6,-m5,m4],[-m6,0,m3,-m2],[m5,-m3,0,m1],[-m4,m2,-m1,0]]
__device__ __forceinline__ void meps_col(const dz* m, int j, dz* col) {
  dz z{0.0, 0.0};
  switch (j) {
    case 0: col[0] = z; col[1] = -m[5]; col[2] = m[4]; col[3] = -m[3]; break;
    case 1: col[0] = m[5]; col[1] = z; col[2] = -m[2]; col[3] = m[1]; break;
    case 2: col[0] = -m[4]; col[1] = m[2]; col[2] = z; col[3] = -m[0]; break;
    default: col[0] = m[3]; col[1] = -m[1]; col[2] = m[0]; col[3] = z; break;
  }
}

__device__ __forceinline__ void set_env(const FKStatic& P, const FKLaunch& LL, int slot, int iwn, Env& e) {
  const int jf = LL.jf[slot];
  const double f = (double)(jf - 1) * P.df;
  e.spl = LL.spl + (long long)slot * (P.nk + 1) * SPL_STRIDE;
  e.poly = LL.poly + (long long)slot * (P.nk + 1) * POLY_STRIDE;
  e.nl = 1;
  e.omre = 2.0 * PI_F * f;
  e.omim = -P.sigma;
  double wn = (double)(iwn - 1) * P.dwn;
  if (P.global_ == 1) wn = sqrt((double)((long long)(iwn - 1) * iwn)) / P.rearth;
  e.dll1 = (wn * P.rearth) * (wn * P.rearth);
}

// htry of the spheroidal adjoint (spheroidalAdjoint.f90:126-129)
__device__ double adjoint_htry(const FKStatic& P, Env& e, double ra, double re) {
  int nl, top;
  layer_index(P, ra, nl, top);
  if (top == 1 && ra < re) nl = min(nl + 1, P.nlay);
  e.nl = nl;
  double ro; dz el7[7];
  eval_spline<0x60u>(P, e, ra, nl, ro, el7);
  double v = sqrt(el7[6].re / ro);
  if (v < EPS_D) v = sqrt((el7[5] + (4.0 / 3.0) * el7[6]).re / ro);
  return ((0.25 * v) * TWO_PI_F) / e.omre;
}

// moment (istyp 1) / force (0) source terms at node n (sourceTerms.f90:59-118)
__device__ void source_terms_of(const FKStatic& P, const Env& e, int n, int istyp, dz zsph[4][4], dz ztor[2][2]) {
  const double r = P.rnod[n];
  const bool fluid = P.state[n] == 1;
  const double rr2 = 1.0 / (r * r), rr3 = rr2 / r, elp1 = e.dll1, om = e.omre;
  double ro; dz el[7];
  eval_spline<0x0Eu>(P, e, r, P.layer[n], ro, el);
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) zsph[i][j] = dz{0, 0};
  for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) ztor[i][j] = dz{0, 0};
  if (istyp == 1) {
    if (fluid) {
      zsph[0][0] = rr2 * (1.0 / el[1] - (elp1 * rr2) / ((om * om) * ro));
      zsph[1][0] = dz{rr3 * 2.0, 0};
      zsph[0][1] = dz{(((0.5 * elp1) * rr2) * rr2) / ((om * om) * ro), 0};
      zsph[1][1] = dz{-rr3, 0};
    } else {
      zsph[0][0] = rr2 / el[1];
      zsph[1][0] = ((rr3 * 2.0) * el[2]) / el[1];
      zsph[3][0] = ((-rr3) * el[2]) / el[1];
      zsph[1][1] = dz{-rr3, 0};
      zsph[3][1] = dz{0.5 * rr3, 0};
      zsph[2][2] = (0.5 * rr2) / el[3];
      zsph[3][3] = dz{0.25 * rr3, 0};
      ztor[0][0] = (0.5 * rr2) / el[3];
      ztor[1][1] = dz{0.25 * rr3, 0};
    }
  } else {
    if (fluid) {
      zsph[1][0] = dz{-rr2, 0};
      zsph[0][1] = dz{(elp1 * rr3) / ((om * om) * ro), 0};
    } else {
      zsph[1][0] = dz{-rr2, 0};
      zsph[3][1] = dz{0.5 * rr2, 0};
      ztor[1][0] = dz{0.5 * rr2, 0};
    }
  }
}

__device__ __forceinline__ void source_terms(const FKStatic& P, const Env& e, int n, dz zsph[4][4], dz ztor[2][2]) {
  source_terms_of(P, e, n, P.istyp, zsph, ztor);
}

__device__ __forceinline__ void put_out(const FKStatic& P, const FKLaunch& LL, int k, int isp, int n, dz v) {
  long long o = (long long)k + LL.nkf * ((long long)isp + (long long)P.nsp * (n - 1));
  if (LL.gf64) LL.gf64[o] = make_double2(v.re, v.im);
  if (LL.gfre) LL.gfre[o] = (float)v.re;
  if (LL.gfim) LL.gfim[o] = (float)v.im;
}

// ------------------------------------------------------------------------
//  DSV spectra with radial derivatives (computeGreenFKSpectraForASKI.f90:
//  471-541): the source sits at node P.jre, the unit-jump Green functions of
//  node n times the source terms give the field at n (no reciprocity), and
//  its radial derivative is A(r) times the field (dsvDerivatives.f90:39-72),
//  A the solid (solidOdeSystem.f90:77-114) or toroidal
//  (toroidalOdeSystem.f90:81-102) system matrix of the layer in which
//  getLayerIndexNodeEarthmodel places r.  Every node is solid (the host
//  rejects fluid nodes in this mode).
// ------------------------------------------------------------------------
__device__ void dsv_sph_derivative(const FKStatic& P, const Env& e, double r, int nj, const dz g[4][4],
                                   dz d[4][4]) {
  int nl, top;
  layer_index(P, r, nl, top);
  Env el_env = e;
  el_env.nl = nl;
  double ro; dz el[7];
  eval_spline<0x1Fu>(P, el_env, r, nl, ro, el);
  const dz zom{e.omre, e.omim};
  const double dll1 = e.dll1, rr = 1.0 / r, rr2 = rr * rr;
  const dz zrpc = 1.0 / el[1];
  const dz z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
  const dz z2 = (el[2] * rr) * zrpc;
  const dz zdlz1 = dll1 * z1;
  const dz zomro = zom * zom * ro;
  dz a[4][4];
  a[0][0] = -(2.0 * z2); a[0][1] = zrpc; a[0][2] = dll1 * z2; a[0][3] = dz{-0.0, 0.0};
  a[1][0] = (-zomro) + (4.0 * z1) * rr2; a[1][1] = 2.0 * z2 - 2.0 * rr; a[1][2] = -((2.0 * rr2) * zdlz1);
  a[1][3] = dz{dll1 * rr, 0.0};
  a[2][0] = dz{-rr, 0.0}; a[2][1] = dz{-0.0, 0.0}; a[2][2] = dz{rr, 0.0}; a[2][3] = 1.0 / el[3];
  a[3][0] = -((2.0 * z1) * rr2); a[3][1] = -z2; a[3][2] = (-zomro) + (zdlz1 + (dll1 - 2.0) * el[4]) * rr2;
  a[3][3] = dz{-3.0 * rr, 0.0};
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < 4; ++i) {
      dz v{0.0, 0.0};
      for (int kk = 0; kk < 4; ++kk) v = v + a[i][kk] * g[kk][j];
      d[i][j] = v;
    }
}

__device__ void dsv_tor_derivative(const FKStatic& P, const Env& e, double r, int nj, const dz g[2][2],
                                   dz d[2][2]) {
  int nl, top;
  layer_index(P, r, nl, top);
  Env el_env = e;
  el_env.nl = nl;
  double ro; dz el[7];
  eval_spline<0x18u>(P, el_env, r, nl, ro, el);
  const dz zom{e.omre, e.omim};
  const double rr = 1.0 / r, rr2 = rr * rr;
  const dz zomro = zom * zom * ro;
  dz a[2][2];
  a[0][0] = dz{rr, 0.0}; a[0][1] = 1.0 / el[3];
  a[1][0] = (-zomro) - (el[4] * rr2) * (2.0 - e.dll1); a[1][1] = dz{-3.0 * rr, 0.0};
  for (int j = 0; j < nj; ++j)
    for (int i = 0; i < 2; ++i) {
      dz v{0.0, 0.0};
      for (int kk = 0; kk < 2; ++kk) v = v + a[i][kk] * g[kk][j];
      d[i][j] = v;
    }
}

// spheroidal part of node n: U, V for every jump, then dU/dr, dV/dr
__device__ void output_dsv_sph_node(const FKStatic& P, const Env& e, const Slot& s, const LaneLayout& lay, int n,
                                    const FKLaunch& LL, int k) {
  dz zsph[4][4], ztor[2][2];
  source_terms(P, e, P.jre, zsph, ztor);
  dz g[4][4], d[4][4];
  for (int j = 0; j < P.njsph; ++j)
    for (int i = 0; i < 4; ++i) {
      dz v{0.0, 0.0};
      for (int kk = 0; kk < 4; ++kk) v = v + s.get(lay.sph(n, kk, i)) * zsph[kk][j];
      g[i][j] = v;
    }
  dsv_sph_derivative(P, e, P.rnod[n], P.njsph, g, d);
  int isp = 0;
  for (int i = 0; i < 4; i += 2)
    for (int j = 0; j < P.njsph; ++j) put_out(P, LL, k, isp++, n, g[i][j]);
  for (int i = 0; i < 4; i += 2)
    for (int j = 0; j < P.njsph; ++j) put_out(P, LL, k, isp++, n, d[i][j]);
}

// toroidal part of node n: W for every jump, then dW/dr
__device__ void output_dsv_tor_node(const FKStatic& P, const Env& e, const dz ti[2][2], int n, const FKLaunch& LL,
                                    int k) {
  dz zsph[4][4], ztor[2][2];
  source_terms(P, e, P.jre, zsph, ztor);
  dz g[2][2], d[2][2];
  for (int j = 0; j < P.njtor; ++j)
    for (int i = 0; i < 2; ++i) g[i][j] = (dz{0.0, 0.0} + ti[i][0] * ztor[0][j]) + ti[i][1] * ztor[1][j];
  dsv_tor_derivative(P, e, P.rnod[n], P.njtor, g, d);
  int isp = 4 * P.njsph;
  for (int j = 0; j < P.njtor; ++j) put_out(P, LL, k, isp++, n, g[0][j]);
  for (int j = 0; j < P.njtor; ++j) put_out(P, LL, k, isp++, n, d[0][j]);
}

// toroidal part of node n for one source of a set (node jsh, type ty) into that
// source's output block at element offset off
__device__ void output_dsv_tor_src(const FKStatic& P, const Env& e, const dz ti[2][2], int n, const FKLaunch& LL,
                                   int k, int jsh, int ty, long long off) {
  dz zsph[4][4], ztor[2][2];
  source_terms_of(P, e, jsh, ty, zsph, ztor);
  const int njsph = ty == 0 ? 2 : 4, njtor = ty == 0 ? 1 : 2, nsp = 4 * njsph + 2 * njtor;
  dz g[2][2], d[2][2];
  for (int j = 0; j < njtor; ++j)
    for (int i = 0; i < 2; ++i) g[i][j] = (dz{0.0, 0.0} + ti[i][0] * ztor[0][j]) + ti[i][1] * ztor[1][j];
  dsv_tor_derivative(P, e, P.rnod[n], njtor, g, d);
  for (int q = 0; q < 2 * njtor; ++q) {
    const dz v = q < njtor ? g[0][q] : d[0][q - njtor];
    const long long o = off + k + LL.nkf * ((long long)(4 * njsph + q) + (long long)nsp * (n - 1));
    if (LL.gf64) LL.gf64[o] = make_double2(v.re, v.im);
    if (LL.gfre) LL.gfre[o] = (float)v.re;
    if (LL.gfim) LL.gfim[o] = (float)v.im;
  }
}

// spheroidal spectra of node n: reciprocity (reciprocity.f90:82-153) and
// gfsph = bgsph * zsph (computeGreenFKSpectraForSynthetics.f90:445-494)
__device__ void output_sph_node(const FKStatic& P, const Env& e, const Slot& s, const LaneLayout& lay, int n,
                                const FKLaunch& LL, int k) {
  if (P.dsv) { output_dsv_sph_node(P, e, s, lay, n, LL, k); return; }
  const double re = P.rnod[P.jre], r = P.rnod[n];
  const double elp1 = e.dll1, rlp1 = 1.0 / elp1, f = (r / re) * (r / re);
  const bool fluid = P.state[n] == 1;
  dz zsph[4][4], ztor[2][2];
  source_terms(P, e, n, zsph, ztor);
  dz bi[4][4];
  for (int j = 0; j < 4; ++j) for (int c = 0; c < 4; ++c) bi[c][j] = s.get(lay.sph(n, j, c));
  dz bo[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) bo[i][j] = dz{0, 0};
  bo[0][0] = (-f) * bi[1][1]; bo[1][0] = f * bi[1][0];
  bo[0][1] = f * bi[0][1]; bo[1][1] = (-f) * bi[0][0];
  if (!fluid) {
    bo[2][0] = ((-f) * bi[1][3]) * rlp1; bo[3][0] = (f * bi[1][2]) * rlp1;
    bo[2][1] = (f * bi[0][3]) * rlp1; bo[3][1] = ((-f) * bi[0][2]) * rlp1;
    bo[0][2] = ((-f) * bi[3][1]) * elp1; bo[1][2] = (f * bi[3][0]) * elp1;
    bo[2][2] = (-f) * bi[3][3]; bo[3][2] = f * bi[3][2];
    bo[0][3] = (f * bi[2][1]) * elp1; bo[1][3] = ((-f) * bi[2][0]) * elp1;
    bo[2][3] = f * bi[2][3]; bo[3][3] = (-f) * bi[2][2];
  } else if (elp1 > EPS_D) {
    bo[2][0] = ((-f) * bi[1][3]) * rlp1; bo[3][0] = (f * bi[1][2]) * rlp1;
    bo[2][1] = (f * bi[0][3]) * rlp1; bo[3][1] = ((-f) * bi[0][2]) * rlp1;
  }
  const int nk = fluid ? 2 : 4;
  int isp = 0;
  for (int i = 0; i < P.ncsph; i += P.dsvstep)
    for (int l = 0; l < P.njsph; ++l) {
      dz g{0.0, 0.0};
      if (!fluid || l < 2) {
        g = bo[i][0] * zsph[0][l];
        for (int kk = 1; kk < nk; ++kk) g = g + bo[i][kk] * zsph[kk][l];
      }
      put_out(P, LL, k, isp++, n, g);
    }
}

// toroidal spectra of node n (reciprocity.f90:169-180, :485-490)
__device__ void output_tor_node(const FKStatic& P, const Env& e, const dz ti[2][2], int n, const FKLaunch& LL,
                                int k) {
  if (P.dsv) { output_dsv_tor_node(P, e, ti, n, LL, k); return; }
  const double re = P.rnod[P.jre], r = P.rnod[n], f = (r / re) * (r / re);
  const bool fluid = P.state[n] == 1;
  dz zsph[4][4], ztor[2][2];
  source_terms(P, e, n, zsph, ztor);
  dz bt[2][2];
  bt[0][0] = (-f) * ti[1][1]; bt[1][0] = f * ti[1][0];
  bt[0][1] = f * ti[0][1]; bt[1][1] = (-f) * ti[0][0];
  int isp = (P.ncsph + P.dsvstep - 1) / P.dsvstep * P.njsph;
  for (int i = 0; i < P.nctor; i += P.dsvstep)
    for (int l = 0; l < P.njtor; ++l) {
      dz g{0.0, 0.0};
      if (!fluid) g = bt[i][0] * ztor[0][l] + bt[i][1] * ztor[1][l];
      put_out(P, LL, k, isp++, n, g);
    }
}

// store the solution at node n
template <int PH>
__device__ void sink_node(const FKStatic& P, const FKLaunch& LL, const Slot& s, const LaneLayout& lay, Lane& L,
                          int n) {
  const ItemStore IS{&LL};
  switch (L.sink) {
    case K_DT: case K_UT:
      for (int c = 0; c < 2; ++c) s.put(L.sink == K_UT ? lay.ut(n, c) : lay.dt(n, c), L.y[c]);
      break;
    case K_UM:
      for (int c = 0; c < L.nv; ++c) IS.put_um(L.k, n, c, L.y[c]);
      IS.put_um(L.k, n, 5, (-L.y[0]) / L.e.dll1);
      s.put(lay.lg(n), dz{L.lgnorm, 0.0});
      break;
    case K_DM:
      for (int c = 0; c < L.nv; ++c) IS.put_dm(L.k, n, c, P.jsl, L.y[c]);
      IS.put_dm(L.k, n, 5, P.jsl, (-L.y[0]) / L.e.dll1);
      s.put(lay.lg(n), dz{L.lgnorm, 0.0});
      break;
    case K_ADJIC:
      for (int c = 0; c < 4; ++c) s.put(lay.adjic(n, c), L.y[c]);
      break;
    default: {   // K_ADJ_UP / K_ADJ_DN: UJGF = mtil * adjoint (unitJumpGreenFunctions.f90:359-372)
      const bool up = L.sink == K_ADJ_UP;
      bool use;
      if (up) use = n >= P.jre && P.state[n] == 0 && P.rnod[n] < P.ruc;
      else use = n < P.jre && P.state[n] == 0 && P.rnod[n] >= L.rstart_s && P.rnod[n] > P.roc;
      if (!use) return;
      dz m[6], out[4];
      for (int c = 0; c < 6; ++c) m[c] = up ? IS.dm(L.k, n, c, P.jsl) : IS.um(L.k, n, c);
      mtil_times(m, L.y, out);
      for (int c = 0; c < 4; ++c) s.put(lay.sph(n, L.stage >> 1, c), out[c]);
    }
  }
}

// start a propagation (propagateOde.f90:132-216); the lane continues in S_PROP_NEXT
template <int PH>
__device__ void prop_begin(const FKStatic& P, const FKLaunch& LL, const Slot& s, const LaneLayout& lay, Lane& L,
                           int sys, double x1, double x2, double htry, const dz* ys, bool do_norm, double lgnorm,
                           int sink, int after) {
  L.sys = sys;
  L.nv = sys == SYS_MINORS ? 5 : (sys == SYS_SOLIDT ? 4 : 2);
  L.sink = sink; L.after = after; L.do_norm = do_norm; L.lgnorm = lgnorm;
  for (int v = 0; v < 5; ++v) L.y[v] = v < L.nv ? ys[v] : dz{0.0, 0.0};
  L.x1 = x1; L.x2 = x2;
  node_range(P, x1, x2, L.jl, L.jr);
  L.nnodp = L.jr - L.jl + 1; if (L.nnodp < 0) L.nnodp = 0;
  disco_range(P, x1, x2, L.dl, L.dr);
  L.ndp = L.dr - L.dl + 1; if (L.ndp < 0) L.ndp = 0;
  L.idir = copysign(1.0, x2 - x1);
  const bool asc = x2 >= x1;
  auto xn = [&](int kk) { return asc ? P.rnod[L.jl + kk - 1] : P.rnod[L.jr - kk + 1]; };
  auto xd = [&](int kk) { return asc ? P.rb[L.dl + kk - 1] : P.rb[L.dr - kk + 1]; };
  if ((L.ndp > 0 && ((x1 - xd(1)) * L.idir > 0 || (xd(L.ndp) - x2) * L.idir > 0)) ||
      (L.nnodp > 0 && ((x1 - xn(1)) * L.idir > 0 || (xn(L.nnodp) - x2) * L.idir > 0))) {
    L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; return;
  }
  if (fabs(x2 - x1) < MINSIZE_IS) {
    if (L.nnodp == 0) { L.st = after; return; }
    if (L.nnodp > 1) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; return; }
    sink_node<PH>(P, LL, s, lay, L, asc ? L.jl : L.jr);
    L.st = after;
    return;
  }
  L.hdid = htry;
  L.jnod = 1; L.jd = 1;
  L.xa = x1;
  L.st = S_PROP_NEXT;
}

#define FAIL(code) do { L.status = (code); L.st = S_ITEM_END; } while (0)

// ------------------------------------------------------------------------
//  Per-lane bookkeeping of one phase
// ------------------------------------------------------------------------
template <int PH>
__device__ __noinline__ void advance(const FKStatic& P, const FKLaunch& LL, const Slot& s, const LaneLayout& lay,
                                     Lane& L) {
  const int jre = P.jre, nnod = P.nnod;
  const ItemStore IS{&LL};
  for (int guard = 0; guard < 100000; ++guard) {
    switch (L.st) {
      case S_FETCH: case S_IDLE: case S_INTEG:
        return;

      case S_ITEM_INIT: {
        const int2 w = LL.items[L.k];
        set_env(P, LL, w.x, w.y, L.e);
        L.iwn = w.y;
        L.status = ST_OK;
        L.kopt = LL.prop_kopt ? (int)LL.prop_kopt[(long long)PH * LL.nkf + L.k] : P.kopt;
        L.hs = LL.prop_hs ? (double)LL.prop_hs[(long long)PH * LL.nkf + L.k] : 1.0;
        L.det = dz{0, 0};
        if (LL.status && LL.status[L.k] != ST_OK) { L.st = S_FETCH; break; }   // failed in an earlier phase
        if (P.global_ == 0 && L.iwn == 1) { L.st = S_FETCH; break; }           // wn = 0 stays zero
        L.rstart_t = LL.rstart[L.k];
        L.rstart_s = LL.rstart[LL.nkf + L.k];
        if (PH == PH_TOR) {   // toroidalMinors.f90:150-199
          for (int el = 0; el < 4 * lay.NN; ++el) s.put(el, dz{0.0, 0.0});
          L.up = 0;
          L.st = S_TOR_DONE;
          // minors over the source-node range jsl..jsr (toroidalMinors.f90:129-160)
          if (L.e.dll1 < EPS_D || L.rstart_t >= P.rnod[P.jsr]) { L.st = S_ITEM_END; break; }
          double rmin = fmax(L.rstart_t, P.rnod[P.jsl]);
          dz ys[5]; double htry, rsurf; int nl;
          int rc = toroidal_surface_iv(P, L.e, ys, htry, rsurf, nl);
          if (rc) { FAIL(rc); break; }
          if (rsurf < rmin) { L.st = S_ITEM_END; break; }
          L.e.nl = nl;
          L.rend = rsurf;
          prop_begin<PH>(P, LL, s, lay, L, SYS_TOROIDAL, rsurf, rmin, htry * L.hs, ys, false, 0.0, K_DT, S_TOR_UP);
        } else if (PH == PH_SPH) {   // spheroidalMinors.f90:155-182
          for (int el = 0; el < lay.NN; ++el) s.put(lay.lg(el), dz{0.0, 0.0});
          if (L.rstart_s >= P.rnod[P.jsr]) { L.st = S_ITEM_END; break; }
          L.up = 1;
          L.rbeg = L.rstart_s; L.rend = L.rstart_s; L.rlim = P.rnod[P.jsr];
          L.lgnorm_g = 0.0; L.lgnormend = 0.0; L.htry_g = 0.0; L.liq_old = 0;
          L.st = S_SPH_GROUP;
        } else {   // unitJumpGreenFunctions.f90:194-372
          for (int el = 0; el < LaneLayout::PER_NODE * lay.NN; ++el) s.put(el, dz{0.0, 0.0});
          double2 d = LL.dets[L.k];
          L.det = dz{d.x, d.y};
          if (!(zabs(L.det) > TINY_D)) { L.st = L.e.dll1 < EPS_D ? S_OUTPUT : S_ITEM_END; break; }
          if (L.e.dll1 < EPS_D) {   // l = 0 (:201-220)
            for (int j = 0; j < 2; ++j) {
              double u1 = j == 0 ? 1.0 : 0.0, u2 = j == 1 ? 1.0 : 0.0;
              dz dd = (u2 * IS.dm(L.k, jre, 0, P.jsl) - u1 * IS.dm(L.k, jre, 1, P.jsl)) / L.det;
              dz ee = (u2 * IS.um(L.k, jre, 0) - u1 * IS.um(L.k, jre, 1)) / L.det;
              for (int n = jre; n <= nnod; ++n)
                for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), ee * IS.dm(L.k, n, c, P.jsl));
              for (int n = jre - 1; n >= 1; --n)
                for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), dd * IS.um(L.k, n, c));
            }
            L.st = S_OUTPUT;
            break;
          }
          if (P.state[jre] == 1 && P.layer[jre] == P.nlay) { FAIL(ST_UNSUPPORTED); break; }   // source in the ocean
          double re_ic = fmax(L.rstart_s, P.rnod[1]);
          if (re_ic < P.ric) {   // inner-core propagator P_4m (:227-238)
            dz ys[5] = {{0, 0}, {0, 0}, {0, 0}, {1.0, 0}, {0, 0}};
            double htry = adjoint_htry(P, L.e, P.ric, re_ic) * L.hs;
            prop_begin<PH>(P, LL, s, lay, L, SYS_SOLIDT, P.ric, re_ic, htry, ys, false, 0.0, K_ADJIC, S_ADJ_PLAN);
            L.up = 1;
          } else {
            L.up = 0;
            L.st = S_ADJ_PLAN;
          }
        }
        break;
      }

      // ---------------- toroidal phase
      case S_TOR_UP: {   // toroidalMinors.f90:206-240
        if (L.jr - L.jl < 0) { FAIL(ST_BOOKKEEPING); break; }
        double rmax = fmin(P.rnod[P.jsr], L.rend);
        int nl, top;
        layer_index(P, L.rstart_t, nl, top);
        if (top == 1) nl = nl + 1;
        L.e.nl = nl;
        dz ys[5]; double htry;
        int rc = toroidal_bottom_iv(P, L.e, L.rstart_t, ys, htry);
        if (rc) { FAIL(rc); break; }
        prop_begin<PH>(P, LL, s, lay, L, SYS_TOROIDAL, L.rstart_t, rmax, htry * L.hs, ys, false, 0.0, K_UT, S_TOR_DONE);
        L.up = 1;
        break;
      }
      case S_TOR_DONE: {   // determinant and toroidal UJGF (unitJumpGreenFunctions.f90:147-175)
        if (L.jr - L.jl < 0) { FAIL(ST_BOOKKEEPING); break; }
        if constexpr (PH == PH_TOR) {
          if (LL.nsrc > 0) {   // every source node of a set, each into its own output block
            for (int b = 0; b < LL.nsrc; ++b) {
              const int jsh = LL.src_node[b], ty = LL.src_type[b];
              const dz det =
                  s.get(lay.ut(jsh, 0)) * s.get(lay.dt(jsh, 1)) - s.get(lay.dt(jsh, 0)) * s.get(lay.ut(jsh, 1));
              if (!(zabs(det) > TINY_D)) continue;
              const int mask = ty == 1 ? 3 : 2;
              dz dcoef[2], ecoef[2];
              for (int j = 0; j < 2; ++j) {
                double u1 = j == 0 ? 1.0 : 0.0, u2 = j == 1 ? 1.0 : 0.0;
                dcoef[j] = (u2 * s.get(lay.dt(jsh, 0)) - u1 * s.get(lay.dt(jsh, 1))) / det;
                ecoef[j] = (u2 * s.get(lay.ut(jsh, 0)) - u1 * s.get(lay.ut(jsh, 1))) / det;
              }
              for (int n = 1; n <= nnod; ++n) {
                dz ti[2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};   // [comp][jump]
                for (int j = 0; j < 2; ++j) {
                  if (!(mask & (1 << j))) continue;
                  if (n < jsh) {
                    if (P.state[n] == 0 && P.rnod[n] > L.rstart_t)
                      for (int c = 0; c < 2; ++c) ti[c][j] = dcoef[j] * s.get(lay.ut(n, c));
                  } else if (P.state[n] == 0) {
                    for (int c = 0; c < 2; ++c) ti[c][j] = ecoef[j] * s.get(lay.dt(n, c));
                  }
                }
                output_dsv_tor_src(P, L.e, ti, n, LL, L.k, jsh, ty, (long long)b * LL.src_blk);
              }
            }
            L.st = S_ITEM_END;
            break;
          }
        }
        L.det = s.get(lay.ut(jre, 0)) * s.get(lay.dt(jre, 1)) - s.get(lay.dt(jre, 0)) * s.get(lay.ut(jre, 1));
        if (!(zabs(L.det) > TINY_D)) { L.st = S_ITEM_END; break; }
        // jumps whose Green functions are stored: the DSV spectra of a moment
        // source use both, those of a force only the second
        const int tor_mask = (P.dsv ? P.istyp == 1 : P.stressflag) ? 3 : 2;
        dz dcoef[2], ecoef[2];
        for (int j = 0; j < 2; ++j) {
          double u1 = j == 0 ? 1.0 : 0.0, u2 = j == 1 ? 1.0 : 0.0;
          dcoef[j] = (u2 * s.get(lay.dt(jre, 0)) - u1 * s.get(lay.dt(jre, 1))) / L.det;
          ecoef[j] = (u2 * s.get(lay.ut(jre, 0)) - u1 * s.get(lay.ut(jre, 1))) / L.det;
        }
        for (int n = 1; n <= nnod; ++n) {
          dz ti[2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};   // [comp][jump]
          for (int j = 0; j < 2; ++j) {
            if (!(tor_mask & (1 << j))) continue;
            if (n < jre) {
              if (P.state[n] == 0 && P.rnod[n] > L.rstart_t)
                for (int c = 0; c < 2; ++c) ti[c][j] = dcoef[j] * s.get(lay.ut(n, c));
            } else if (P.state[n] == 0) {
              for (int c = 0; c < 2; ++c) ti[c][j] = ecoef[j] * s.get(lay.dt(n, c));
            }
          }
          output_tor_node(P, L.e, ti, n, LL, L.k);
        }
        L.st = S_ITEM_END;
        break;
      }

      // ---------------- spheroidal phase
      case S_SPH_GROUP: {
        const bool up = L.up == 1;
        if (!(up ? L.rend < L.rlim : L.rend > L.rlim)) {
          // normalise to the final normalisation factor (spheroidalMinors.f90:360-365,552-557)
          int n0 = up ? 1 : P.jsl, n1 = up ? P.jsr : nnod;
          for (int n = n0; n <= n1; ++n) {
            double fct = pow(10.0, s.get(lay.lg(n)).re - L.lgnormend);
            for (int c = 0; c < 6; ++c) {
              if (up) IS.put_um(L.k, n, c, IS.um(L.k, n, c) * fct);
              else IS.put_dm(L.k, n, c, P.jsl, IS.dm(L.k, n, c, P.jsl) * fct);
            }
          }
          if (up) {
            for (int el = 0; el < lay.NN; ++el) s.put(lay.lg(el), dz{0.0, 0.0});
            L.up = 0;
            L.rbeg = P.rearth; L.rend = P.rearth; L.rlim = fmax(L.rstart_s, P.rnod[P.jsl]);
            L.lgnorm_g = 0.0; L.lgnormend = 0.0; L.liq_old = 0;
            break;
          }
          // determinants at the source nodes jsl..jsr (spheroidalMinors.f90:566-575)
          for (int js = P.jsl; js <= P.jsr; ++js) {
            dz u[6], d[6];
            for (int c = 0; c < 6; ++c) { u[c] = IS.um(L.k, js, c); d[c] = IS.dm(L.k, js, c, P.jsl); }
            if (P.state[js] == 1 || L.e.dll1 < EPS_D) L.det = u[0] * d[1] - d[0] * u[1];
            else L.det = ((((u[0] * d[5] + u[5] * d[0]) - u[1] * d[4]) + u[2] * d[3]) + u[3] * d[2]) - u[4] * d[1];
            LL.dets[(long long)(js - P.jsl) * LL.nkf + L.k] = make_double2(L.det.re, L.det.im);
          }
          L.st = S_ITEM_END;
          break;
        }
        int nl, top;
        layer_index(P, L.rbeg, nl, top);
        if (up && top == 1) nl = nl + 1;
        L.liq = P.iflso[nl] == 1;
        L.e.nl = nl;
        L.rend = up ? fmin(above_pc(P, nl), L.rlim) : fmax(below_pc(P, nl), L.rlim);
        const bool l0 = L.e.dll1 < EPS_D;
        const int sys = L.liq ? SYS_FLUID : (l0 ? SYS_RADIAL : SYS_MINORS);
        dz ys[5] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
        if (L.rbeg == (up ? L.rstart_s : P.rearth)) {
          int rc = up ? minors_bottom_iv(P, L.e, L.rbeg, ys, L.htry_g) : minors_surface_iv(P, L.e, ys, L.htry_g);
          if (rc) { FAIL(rc); break; }
          L.htry_g *= L.hs;
        } else if (L.liq && !L.liq_old) {
          if (l0) { ys[0] = L.yend[0]; ys[1] = L.yend[1]; } else { ys[0] = L.yend[2]; ys[1] = L.yend[4]; }
        } else if (!L.liq && L.liq_old) {
          if (l0) { ys[0] = L.yend[0]; ys[1] = L.yend[1]; }
          else { ys[3] = L.yend[1]; ys[1] = L.yend[0]; }
        } else {
          FAIL(ST_BOOKKEEPING); break;
        }
        prop_begin<PH>(P, LL, s, lay, L, sys, L.rbeg, L.rend, L.htry_g, ys, true, L.lgnorm_g, up ? K_UM : K_DM,
                       S_SPH_GROUP_END);
        break;
      }
      case S_SPH_GROUP_END: {
        if (L.up == 0 && L.jr - L.jl < 0) { FAIL(ST_BOOKKEEPING); break; }
        L.liq_old = L.liq;
        L.rbeg = L.rend;
        for (int v = 0; v < 5; ++v) L.yend[v] = L.y[v];
        L.lgnormend = L.lgnorm;
        L.lgnorm_g = L.lgnormend;
        L.st = S_SPH_GROUP;
        break;
      }

      // ---------------- adjoint phase
      case S_ADJ_PLAN: {
        if (L.up == 1 && L.jr - L.jl < 0) { FAIL(ST_BOOKKEEPING); break; }
        L.core_below = 0; L.lowest = 0;
        L.re_dn = fmax(fmax(L.rstart_s, P.roc), P.rnod[1]);
        for (int n = jre - 1; n >= 1; --n) {
          if (P.rnod[n] < L.rstart_s) continue;
          if (P.state[n] == 1 || P.rnod[n] < P.ric) L.core_below = 1;
          else if (P.rnod[n] > P.roc && P.rnod[n] >= L.re_dn) L.lowest = n;
        }
        L.ocean_above = 0; L.highest = jre;
        for (int n = jre; n <= nnod; ++n) {
          if (P.state[n] == 0 && P.rnod[n] < P.ruc) L.highest = n;
          else if (P.state[n] == 1 && P.rnod[n] > P.ruc) L.ocean_above = 1;
        }
        L.stage = -1;
        L.st = S_ADJ_NEXT;
        break;
      }
      case S_ADJ_NEXT: {   // stage = 2*jump + (0 up, 1 down)  (:303-372)
        // jumps 2 and 4 only without stresses, and for the DSV spectra of a force
        const int sph_mask = (P.dsv ? P.istyp == 1 : P.stressflag) ? 15 : 10;
        int stg = L.stage + 1;
        for (; stg < 8; ++stg) {
          int j = stg >> 1;
          if (!(sph_mask & (1 << j))) continue;
          if ((stg & 1) && L.lowest == 0 && !L.core_below) continue;
          break;
        }
        if (stg >= 8) { L.st = S_OUTPUT; break; }
        L.stage = stg;
        const int j = stg >> 1;
        const bool upd = (stg & 1) == 0;
        dz m[6], col[4], ys[5];
        for (int c = 0; c < 6; ++c) m[c] = upd ? IS.um(L.k, jre, c) : IS.dm(L.k, jre, c, P.jsl);
        meps_col(m, j, col);
        for (int c = 0; c < 4; ++c) ys[c] = upd ? dz{0.0, 0.0} - col[c] / L.det : dz{0.0, 0.0} + col[c] / L.det;
        ys[4] = dz{0, 0};
        const double ra = P.rnod[jre];
        const double xe = upd ? (L.ocean_above ? P.ruc : P.rnod[L.highest]) : (L.core_below ? L.re_dn : P.rnod[L.lowest]);
        double htry = adjoint_htry(P, L.e, ra, upd ? P.ruc : L.re_dn) * L.hs;
        prop_begin<PH>(P, LL, s, lay, L, SYS_SOLIDT, ra, xe, htry, ys, false, 0.0, upd ? K_ADJ_UP : K_ADJ_DN, S_ADJ_END);
        break;
      }
      case S_ADJ_END: {
        if (L.jr - L.jl < 0) { FAIL(ST_BOOKKEEPING); break; }
        const int j = L.stage >> 1;
        if ((L.stage & 1) == 0) {
          if (L.ocean_above)
            for (int n = jre; n <= nnod; ++n)
              if (P.state[n] == 1 && P.rnod[n] > P.ruc)
                for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), L.y[2] * IS.dm(L.k, n, c, P.jsl));
        } else if (L.core_below) {
          dz a3 = L.y[2];
          for (int n = jre - 1; n >= 1; --n) {
            if (P.rnod[n] < L.rstart_s) continue;
            if (P.state[n] == 0 && P.rnod[n] < P.ric) {
              dz mm[6], a[4], out[4];
              for (int c = 0; c < 6; ++c) mm[c] = IS.um(L.k, n, c);
              for (int c = 0; c < 4; ++c) a[c] = s.get(lay.adjic(n, c));
              mtil_times(mm, a, out);
              for (int c = 0; c < 4; ++c) s.put(lay.sph(n, j, c), a3 * out[c]);
            } else if (P.state[n] == 1) {
              for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), a3 * IS.um(L.k, n, c));
            }
          }
        }
        L.st = S_ADJ_NEXT;
        break;
      }
      case S_OUTPUT:
        for (int n = 1; n <= nnod; ++n) output_sph_node(P, L.e, s, lay, n, LL, L.k);
        L.st = S_ITEM_END;
        break;

      case S_ITEM_END:
        if (L.status != ST_OK && LL.status) LL.status[L.k] = L.status;
        L.st = S_FETCH;
        return;

      // ---------------- propagator: next sub-interval (propagateOde.f90:218-246)
      case S_PROP_NEXT: {
        if (!(fabs(L.x2 - L.xa) > MINSIZE_IS)) {
          if (L.jnod - 1 != L.nnodp || L.jd - 1 != L.ndp) { FAIL(ST_BOOKKEEPING); break; }
          L.st = L.after;
          break;
        }
        const bool asc = L.x2 >= L.x1;
        double s0 = 2.0 * fabs(L.x2 - L.x1), s1 = 3.0 * fabs(L.x2 - L.x1), s2 = fabs(L.x2 - L.xa);
        if (L.jnod <= L.nnodp) s0 = fabs((asc ? P.rnod[L.jl + L.jnod - 1] : P.rnod[L.jr - L.jnod + 1]) - L.xa);
        if (L.jd <= L.ndp) s1 = fabs((asc ? P.rb[L.dl + L.jd - 1] : P.rb[L.dr - L.jd + 1]) - L.xa);
        int kmin = 0; double smin = s0;
        if (s1 < smin) { kmin = 1; smin = s1; }
        if (s2 < smin) { kmin = 2; smin = s2; }
        L.s0 = s0; L.s1 = s1; L.kmin = kmin;
        L.xe = L.xa + L.idir * smin;
        // doIntegrationStep (integrationStep.f90:98-134)
        if (fabs(L.xe - L.xa) < MINSIZE_IS) { L.st = S_SUB_END; break; }
        L.x = L.xa;
        L.h = copysign(L.hdid, L.xe - L.xa);
        L.nstep = 0;
        L.st = S_INTEG;
        return;
      }
      // ---------------- propagator: sub-interval end (propagateOde.f90:255-311)
      case S_SUB_END: {
        if (L.do_norm) {
          double sm = 0.0;
          for (int v = 0; v < L.nv; ++v) sm += fabs(L.y[v].re) + fabs(L.y[v].im);
          double ynorm = sm / L.nv;
          if (ynorm > MAXY_PROP) {
            for (int v = 0; v < L.nv; ++v) { L.y[v].re = L.y[v].re / ynorm; L.y[v].im = L.y[v].im / ynorm; }
            L.lgnorm = L.lgnorm + log10(ynorm);
          }
        }
        const bool asc = L.x2 >= L.x1;
        if (L.kmin == 0) {
          sink_node<PH>(P, LL, s, lay, L, asc ? L.jl + L.jnod - 1 : L.jr - L.jnod + 1);
          L.jnod++;
          if (fabs(L.s0 - L.s1) < MINSIZE_IS) { L.e.nl += (int)L.idir; L.jd++; }
        } else if (L.kmin == 1) {
          L.jd++;
          L.e.nl += (int)L.idir;
          if (fabs(L.s0 - L.s1) < MINSIZE_IS) {
            sink_node<PH>(P, LL, s, lay, L, asc ? L.jl + L.jnod - 1 : L.jr - L.jnod + 1);
            L.jnod++;
          }
        }
        L.xa = L.xe;
        L.st = S_PROP_NEXT;
        break;
      }
      default:
        FAIL(ST_BOOKKEEPING);
        break;
    }
  }
  FAIL(ST_BOOKKEEPING);
}
#undef FAIL

// ------------------------------------------------------------------------
//  Start radii of all items (one thread per item)
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(128) fk_setup_kernel(const __grid_constant__ FKStatic P, FKLaunch LL) {
  __shared__ Tab tab;
  for (int i = threadIdx.x; i <= MAXKNOT; i += blockDim.x) tab.rk[i] = P.rk[i];
  for (int i = threadIdx.x; i <= MAXLAY; i += blockDim.x) {
    tab.drk[i] = P.drk[i]; tab.iktop[i] = P.iktop[i]; tab.rdrk[i] = 1.0 / P.drk[i];
  }
  __syncthreads();
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < LL.nitems; k += (long long)gridDim.x * blockDim.x) {
    int2 w = LL.items[k];
    Env e;
    e.tab = &tab;
    set_env(P, LL, w.x, w.y, e);
    LL.rstart[k] = start_radius(P, e, true);
    LL.rstart[LL.nkf + k] = start_radius(P, e, false);
  }
}

// ------------------------------------------------------------------------
//  Lockstep phase kernel
// ------------------------------------------------------------------------
template <int PH, int BLK, bool BIG>
__global__ void __launch_bounds__(BLK, 1) fk_phase_kernel(const __grid_constant__ FKStatic P, FKLaunch LL) {
  constexpr int NVD = PhaseNV<PH>::NV;
  extern __shared__ double2 smem_diag[];
  __shared__ Tab tab;
  // block-shared run of queue positions (LL.qchunk > 0): (end << 32) | next,
  // refilled from the phase's queue under blk_lock
  __shared__ unsigned long long blk_q;
  __shared__ int blk_lock;
  for (int i = threadIdx.x; i <= MAXKNOT; i += blockDim.x) tab.rk[i] = P.rk[i];
  for (int i = threadIdx.x; i <= MAXLAY; i += blockDim.x) {
    tab.drk[i] = P.drk[i]; tab.iktop[i] = P.iktop[i]; tab.rdrk[i] = 1.0 / P.drk[i];
  }
  if (threadIdx.x == 0) { blk_q = 0ull; blk_lock = 0; }
  __syncthreads();
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  constexpr int DL = PhaseDiag<PH, BLK>::L;
  double2* D = smem_diag + (threadIdx.x >> 5) * (DL * NVD * 32);
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  Slot s{LL.scratch + tid, LL.nthreads};
  LaneLayout lay{P.nnod + 1};
  // the step's own scratch elements follow the node storage
  const Slot xs{LL.scratch + tid + (long long)LaneLayout::PER_NODE * lay.NN * LL.nthreads, LL.nthreads};
  Counters cnt{0, 0, 0, 0, 0, 0, 0, 0};
  unsigned long long trips = 0, integ_lanes = 0, t_start = 0;
  if (LL.warp_ns) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_start));
  unsigned* queue = LL.queue + PH;
  Lane L;
  L.e.tab = &tab;
  L.st = S_FETCH;
  L.qnext = 0; L.qend = 0;
  const unsigned qg = LL.qgran > 1 ? (unsigned)LL.qgran : 1u;
  unsigned long long cyc_adv = 0, cyc_step = 0, mixed_trips = 0, cyc_minor_sys = 0;
  int waited = 0;   // trips this lane has waited for its bookkeeping
  for (;;) {
    unsigned long long c0 = clock64();
    // The bookkeeping of lanes between integrations runs divergently, so its
    // cost per pass hardly depends on how many lanes take part: it is deferred
    // until adv_min lanes wait, one has waited adv_wait trips, or none integrates.
    const bool pend = L.st != S_INTEG && L.st != S_IDLE;
    const unsigned pm = __ballot_sync(FULL, pend);
    waited = pend ? waited + 1 : 0;
    const bool go = pm && (__popc(pm) >= LL.adv_min || __any_sync(FULL, waited > LL.adv_wait) ||
                           !__any_sync(FULL, L.st == S_INTEG));
    // A lane at a sub-interval end inside its integration has a short pass
    // (renormalisation, node store, next sub-interval) and takes it at once;
    // waiting for it cost more than it saved at every threshold measured.
    if (!go && pm) {
      const bool pshort = L.st == S_SUB_END && fabs(L.x2 - L.xe) > MINSIZE_IS;
      if (__any_sync(FULL, pshort) && pshort) advance<PH>(P, LL, s, lay, L);
    }
    for (int round = 0; go && round < 64; ++round) {
      // the next position of the lane's reserved run, without the queue
      if (L.st == S_FETCH && L.qnext < L.qend) {
        if (L.qnext < (unsigned)LL.nitems) { L.k = LL.order[L.qnext++]; L.st = S_ITEM_INIT; }
        else L.qnext = L.qend;
      }
      unsigned fm = __ballot_sync(FULL, L.st == S_FETCH);
      if (fm && LL.qchunk > 0) {
        // the block's warps share runs of qchunk consecutive positions (one
        // frequency's adjacent degrees), so their spline tables stay in L1.  The
        // positions of a run go out by an atomic add on its next position; the
        // warp that finds the run used up and takes the lock installs the next
        // run from the queue.  Lanes left without a position retry.
        const int leader = __ffs(fm) - 1;
        unsigned base = 0, got = 0;
        if (lane == leader) {
          const unsigned n = (unsigned)__popc(fm);
          const unsigned long long q = atomicAdd(&blk_q, (unsigned long long)n);
          const unsigned next = (unsigned)q, end = (unsigned)(q >> 32);
          if (next < end) { base = next; got = min(n, end - next); }
          if (got < n && atomicCAS(&blk_lock, 0, 1) == 0) {
            const unsigned long long cur = atomicAdd(&blk_q, 0ull);
            if ((unsigned)cur >= (unsigned)(cur >> 32)) {
              const unsigned nb = atomicAdd(queue, (unsigned)LL.qchunk);
              atomicExch(&blk_q, ((unsigned long long)(nb + (unsigned)LL.qchunk) << 32) | nb);
            }
            atomicExch(&blk_lock, 0);
          }
        }
        base = __shfl_sync(FULL, base, leader);
        got = __shfl_sync(FULL, got, leader);
        if (L.st == S_FETCH) {
          const unsigned r = (unsigned)__popc(fm & ((1u << lane) - 1u));
          if (r < got) {
            const unsigned my = base + r;
            if (my < (unsigned)LL.nitems) { L.k = LL.order[my]; L.st = S_ITEM_INIT; }
            else L.st = S_IDLE;
          }
        }
      } else if (fm) {
        int leader = __ffs(fm) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(queue, (unsigned)__popc(fm) * qg);
        base = __shfl_sync(FULL, base, leader);
        if (L.st == S_FETCH) {
          const unsigned my = base + (unsigned)__popc(fm & ((1u << lane) - 1u)) * qg;
          if (my < (unsigned)LL.nitems) { L.k = LL.order[my]; L.st = S_ITEM_INIT; L.qnext = my + 1; L.qend = my + qg; }
          else L.st = S_IDLE;
        }
      }
      advance<PH>(P, LL, s, lay, L);
      if (!__any_sync(FULL, L.st == S_FETCH)) break;
    }
    const bool integ = L.st == S_INTEG;
    unsigned long long c1 = clock64();
    cyc_adv += c1 - c0;
    ++trips;
    integ_lanes += __popc(__ballot_sync(FULL, integ));
    if (!__any_sync(FULL, integ)) {
      if (__all_sync(FULL, L.st == S_IDLE)) break;
      continue;
    }
    // overshoot clamp (integrationStep.f90:136-139) and one lockstep step per system
    if (integ && (L.x + L.h - L.xe) * (L.x + L.h - L.xa) > 0.0) L.h = L.xe - L.x;
    dz yext[5];
    int result = 0;
    if (PH == PH_TOR) {
      bs_step<SYS_TOROIDAL, NVD, DL, BIG>(P, L.e, integ, L.h, L.x, L.y, yext, result, D, lane, xs, cnt);
    } else if (PH == PH_ADJ) {
      bs_step<SYS_SOLIDT, NVD, DL, BIG>(P, L.e, integ, L.h, L.x, L.y, yext, result, D, lane, xs, cnt);
    } else {
      unsigned sysmask = __reduce_or_sync(FULL, integ ? (1u << L.sys) : 0u);
      mixed_trips += __popc(sysmask) > 1;
      if (sysmask & (1u << SYS_MINORS))
        bs_step<SYS_MINORS, NVD, DL, BIG>(P, L.e, integ && L.sys == SYS_MINORS, L.h, L.x, L.y, yext, result, D, lane, xs,
                                          cnt);
      const unsigned long long c2 = clock64();
      if (sysmask & (1u << SYS_FLUID)) {
        int r = 0;
        bs_step<SYS_FLUID, NVD, DL, BIG>(P, L.e, integ && L.sys == SYS_FLUID, L.h, L.x, L.y, yext, r, D, lane, xs,
                                          cnt);
        if (integ && L.sys == SYS_FLUID) result = r;
      }
      if (sysmask & (1u << SYS_RADIAL)) {
        int r = 0;
        bs_step<SYS_RADIAL, NVD, DL, BIG>(P, L.e, integ && L.sys == SYS_RADIAL, L.h, L.x, L.y, yext, r, D, lane, xs,
                                          cnt);
        if (integ && L.sys == SYS_RADIAL) result = r;
      }
      cyc_minor_sys += clock64() - c2;
    }
    cyc_step += clock64() - c1;
    if (LL.steplog) {
      // one warp-aggregated slot reservation per lockstep step
      const unsigned lm = __ballot_sync(FULL, integ);
      const int first = __ffs(lm) - 1;
      unsigned long long base = 0;
      if (lane == first) base = atomicAdd(LL.steplog_n, (unsigned long long)__popc(lm));
      base = __shfl_sync(FULL, base, first);
      const unsigned long long slot = base + __popc(lm & ((1u << lane) - 1u));
      if (integ && slot < LL.steplog_cap) {
        double sm = 0.0;
        for (int v = 0; v < L.nv; ++v) sm += fabs(L.y[v].re) + fabs(L.y[v].im);
        StepRec rec;
        rec.x = L.x; rec.h = L.h; rec.k = L.k;
        rec.lgy = (float)(log10(sm / L.nv + 1e-300) + L.lgnorm);
        rec.nl = (short)L.e.nl; rec.sys = (signed char)L.sys; rec.result = (signed char)(result > 0 ? result : 0);
        rec.phase = (short)PH; rec.nstep = (short)(L.nstep < 32767 ? L.nstep : 32767);
        LL.steplog[slot] = rec;
      }
    }
    // step-size control (integrationStep.f90:140-185)
    if (integ) {
      L.nstep++;
      if (result > 0) {
        cnt.steps_ok++;
        L.x = L.x + L.h;
        for (int v = 0; v < L.nv; ++v) L.y[v] = yext[v];
        if (fabs(L.x - L.xe) < MINSIZE_IS) {
          L.st = S_SUB_END;
        } else {
          if (result > L.kopt) L.h = L.h * SHRINK_BS;
          else if (result < L.kopt) L.h = L.h * GROW_BS;
          L.hdid = L.h;
        }
      } else {
        cnt.steps_rej++;
        L.h = 0.5 * L.h / 1.0;
        if (fabs(L.h) < MINSIZE_IS) { L.status = ST_MINSTEP; L.st = S_ITEM_END; }
      }
      if (L.st == S_INTEG && L.nstep >= MAXNUM_IS) { L.status = ST_MAXSTEPS; L.st = S_ITEM_END; }
    }
  }
  if (LL.prof && lane == 0) {
    atomicAdd(LL.prof + 0, trips);
    atomicAdd(LL.prof + 1, integ_lanes);
    atomicAdd(LL.prof + 2, (unsigned long long)cnt.warp_attempts);
    atomicAdd(LL.prof + 3, (unsigned long long)cnt.lane_attempts);
    atomicAdd(LL.prof + 4, cyc_adv);
    atomicAdd(LL.prof + 5, cyc_step);
    atomicAdd(LL.prof + 6, mixed_trips);     // spheroidal: trips with lanes in two systems
    atomicAdd(LL.prof + 7, cyc_minor_sys);   // spheroidal: cycles in the fluid and l = 0 steps
  }
  if (LL.warp_ns && lane == 0) {
    unsigned long long t_end;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t_end));
    long long w = (long long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    LL.warp_ns[2 * w] = t_start;
    LL.warp_ns[2 * w + 1] = t_end;
  }
  long long v[6] = {cnt.steps_ok, cnt.steps_rej, cnt.attempts, cnt.sysmats, cnt.matvecs, cnt.flops};
  for (int kk = 0; kk < 6; ++kk) {
    long long x = v[kk];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
    if (lane == 0) atomicAdd(LL.stats + kk, (unsigned long long)x);
  }
}

}  // namespace GEM_NS
