// Warp-lockstep FK solver (K1 + K2 fused).
//
// Each lane of a warp owns one (omega, l) item and walks the reference's
// pipeline for it (toroidalMinors.f90:71-268, spheroidalMinors.f90:72-585,
// unitJumpGreenFunctions.f90:62-380, reciprocity + source terms +
// packing computeGreenFKSpectraForSynthetics.f90:445-494).  The pipeline is
// written as a per-lane state machine, so the lanes never wait inside a
// divergent call: every trip of the warp loop
//   1. lets each lane advance its bookkeeping (initial values, node and
//      discontinuity handling, phase changes) until it needs an integration
//      step,
//   2. runs one Bulirsch-Stoer step for all lanes that integrate the same ODE
//      system, in lockstep: attempt j is computed for every lane that has
//      not converged yet, so the warp issues one instruction stream,
//   3. applies the step-size control of each lane.
// The Neville tableau is built incrementally (one new diagonal per attempt,
// the exact values the reference recomputes from scratch) and kept in
// shared memory, lane-interleaved so accesses do not conflict.
#pragma once
#include "fk_kernel.h"
#include "fk_solver.cuh"

namespace gem {

constexpr int NV_MAX = 5;
constexpr int FK_WARPS = FK_BLOCK / 32;
constexpr int DIAG_PER_WARP = 7 * NV_MAX * 32;   // double2 per warp

// lane states
enum : int {
  S_FETCH = 0, S_IDLE, S_ITEM_INIT, S_TOR_UP, S_TOR_DONE, S_SPH_GROUP, S_SPH_GROUP_END, S_SPH_DONE,
  S_ADJ_PLAN, S_ADJ_NEXT, S_ADJ_END, S_OUTPUT, S_ITEM_END, S_PROP_NEXT, S_SUB_END, S_INTEG
};
// node sinks
enum : int { K_DT = 0, K_UT, K_UM, K_DM, K_ADJIC, K_ADJ_UP, K_ADJ_DN };

struct Lane {
  int st, status;
  int slot, iwn;
  long long kidx;
  Env e;
  double rstart_t, rstart_s;
  dz det_t, det_s;
  // spheroidal minors groups
  int up, liq, liq_old;
  double rbeg, rend, rlim, lgnorm_g, lgnormend, htry_g;
  dz yend[NV_MAX];
  // adjoints
  int stage, core_below, ocean_above, lowest, highest;
  double re_dn;
  // current propagation
  int sys, nv, sink, after, do_norm;
  int jl, jr, dl, dr, nnodp, ndp, jnod, jd, kmin, nstep;
  double x1, x2, xa, xe, x, h, hdid, lgnorm, s0, s1, idir;
  dz y[NV_MAX];
};

// ------------------------------------------------------------------------
//  Lockstep Bulirsch-Stoer step of all lanes with `active` set
//  (complexBulirschStep.f90:111-170,180-238,297-340)
// ------------------------------------------------------------------------
template <int SYS>
__device__ __noinline__ void bs_step(const FKStatic& P, const Env& e, bool active, double h, double x,
                                     const dz* y0, dz* yext, int& result, double2* D, int lane, Counters& cnt) {
  constexpr int NV = SysNV<SYS>::NV;
  bool need = active;
  result = 0;   // 0 failed, >0: donetry of a successful step
  dz ys[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) ys[v] = y0[v];
  for (int j = 1; j <= 7; ++j) {
    if (!__any_sync(0xffffffffu, need)) break;
    if (!need) continue;
    dz Y[NV];
    midpoint<SYS>(P, e, j, h, x, ys, Y);
    cnt.attempts++;
    cnt.matvecs += SEQDIV[j - 1] + 1;
    cnt.sysmats += NXDIV[j - 1];
    cnt.flops += (long long)NXDIV[j - 1] * FLOP_SYSMAT[SYS] + (long long)(SEQDIV[j - 1] + 1) * FLOP_MV[SYS];
    // new diagonal of the Neville tableau for point p = j-1 (0-based)
    const int p = j - 1;
    dz yy[NV], dy[NV], c[NV], pend[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { yy[v] = Y[v]; c[v] = Y[v]; pend[v] = Y[v]; dy[v] = dz{0.0, 0.0}; }
    const double xp = h / (double)SEQDIV[p];
    for (int m = 1; m <= p; ++m) {
      const double xi = h / (double)SEQDIV[p - m];
      const double hh = xi - xp;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double2* slot = D + ((m - 1) * NV_MAX + v) * 32 + lane;
        double2 pv = *slot;
        dz u = (c[v] - dz{pv.x, pv.y}) / hh;
        c[v] = xi * u;
        dz nd = xp * u;
        *slot = make_double2(pend[v].re, pend[v].im);   // level m-1 of the new diagonal
        pend[v] = nd;
        yy[v] = yy[v] + nd;
        dy[v] = nd;
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) D[(p * NV_MAX + v) * 32 + lane] = make_double2(pend[v].re, pend[v].im);
    if (j >= 3) {
      cnt.flops += (long long)(j * (j - 1) / 2) * 8 * NV + (long long)(j - 1) * 2 * NV + 8 * NV + 3;
      double s1 = 0.0, s2 = 0.0;
#pragma unroll
      for (int v = 0; v < NV; ++v) { double a = zabs(dy[v]); s1 += a * a; }
#pragma unroll
      for (int v = 0; v < NV; ++v) { double a = zabs(yy[v]); s2 += a * a; }
      double errmax = sqrt(s1 / s2);
      if (errmax / P.eps < 1.0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) yext[v] = yy[v];
        result = j;
        need = false;
      } else if (j == 7) {
        need = false;
      }
    }
  }
}

// ------------------------------------------------------------------------
//  Helpers of the bookkeeping
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

// store the solution at node n (the propagator's node handling, plus the
// consumers: minors, toroidal solutions, adjoint * minor matrix)
__device__ void sink_node(const FKStatic& P, const Slot& s, const Layout& lay, Lane& L, int n) {
  switch (L.sink) {
    case K_DT: case K_UT:
      for (int c = 0; c < 2; ++c) s.put(L.sink == K_UT ? lay.ut(n, c) : lay.dt(n, c), L.y[c]);
      break;
    case K_UM: case K_DM: {
      bool up = L.sink == K_UM;
      for (int c = 0; c < L.nv; ++c) s.put(up ? lay.um(n, c) : lay.dm(n, c), L.y[c]);
      s.put(up ? lay.um(n, 5) : lay.dm(n, 5), (-L.y[0]) / L.e.dll1);
      s.put(up ? lay.ulg(n) : lay.dlg(n), dz{L.lgnorm, 0.0});
      break;
    }
    case K_ADJIC:
      for (int c = 0; c < 4; ++c) s.put(lay.adjic(n, c), L.y[c]);
      break;
    default: {   // K_ADJ_UP / K_ADJ_DN: UJGF = mtil * adjoint (unitJumpGreenFunctions.f90:359-372)
      bool up = L.sink == K_ADJ_UP;
      bool use;
      if (up) use = n >= P.jre && P.state[n] == 0 && P.rnod[n] < P.ruc;
      else use = n < P.jre && P.state[n] == 0 && P.rnod[n] >= L.rstart_s && P.rnod[n] > P.roc;
      if (!use) return;
      dz m[6], out[4];
      for (int c = 0; c < 6; ++c) m[c] = s.get(up ? lay.dm(n, c) : lay.um(n, c));
      mtil_times(m, L.y, out);
      for (int c = 0; c < 4; ++c) s.put(lay.sph(n, L.stage >> 1, c), out[c]);
    }
  }
}

// start a propagation (propagateOde.f90:132-216); the lane continues in S_PROP_NEXT
__device__ void prop_begin(const FKStatic& P, const Slot& s, const Layout& lay, Lane& L, int sys, double x1,
                           double x2, double htry, const dz* ys, bool do_norm, double lgnorm, int sink, int after) {
  L.sys = sys;
  L.nv = sys == SYS_MINORS ? 5 : (sys == SYS_SOLIDT ? 4 : 2);
  L.sink = sink; L.after = after; L.do_norm = do_norm; L.lgnorm = lgnorm;
  for (int v = 0; v < NV_MAX; ++v) L.y[v] = v < L.nv ? ys[v] : dz{0.0, 0.0};
  L.x1 = x1; L.x2 = x2;
  node_range(P, x1, x2, L.jl, L.jr);
  L.nnodp = L.jr - L.jl + 1; if (L.nnodp < 0) L.nnodp = 0;
  disco_range(P, x1, x2, L.dl, L.dr);
  L.ndp = L.dr - L.dl + 1; if (L.ndp < 0) L.ndp = 0;
  L.idir = copysign(1.0, x2 - x1);
  const bool asc = x2 >= x1;
  auto xn = [&](int k) { return asc ? P.rnod[L.jl + k - 1] : P.rnod[L.jr - k + 1]; };
  auto xd = [&](int k) { return asc ? P.rb[L.dl + k - 1] : P.rb[L.dr - k + 1]; };
  if ((L.ndp > 0 && ((x1 - xd(1)) * L.idir > 0 || (xd(L.ndp) - x2) * L.idir > 0)) ||
      (L.nnodp > 0 && ((x1 - xn(1)) * L.idir > 0 || (xn(L.nnodp) - x2) * L.idir > 0))) {
    L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; return;
  }
  if (fabs(x2 - x1) < MINSIZE_IS) {
    if (L.nnodp == 0) { L.st = after; return; }
    if (L.nnodp > 1) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; return; }
    sink_node(P, s, lay, L, asc ? L.jl : L.jr);
    L.st = after;
    return;
  }
  L.hdid = htry;
  L.jnod = 1; L.jd = 1;
  L.xa = x1;
  L.st = S_PROP_NEXT;
}

// htry of the spheroidal adjoint (spheroidalAdjoint.f90:126-129)
__device__ double adjoint_htry(const FKStatic& P, Env& e, double ra, double re) {
  int nl, top;
  layer_index(P, ra, nl, top);
  if (top == 1 && ra < re) nl = min(nl + 1, P.nlay);
  e.nl = nl;
  double ro; dz el7[7];
  eval_spline<0x60u>(P, e.spl, ra, nl, ro, el7);
  double v = sqrt(el7[6].re / ro);
  if (v < EPS_D) v = sqrt((el7[5] + (4.0 / 3.0) * el7[6]).re / ro);
  return ((0.25 * v) * TWO_PI_F) / e.omre;
}

// reciprocity (reciprocity.f90:82-180), source terms (sourceTerms.f90:59-118)
// and gfsph = bgsph * zsph, packed into the output (:445-494)
__device__ void output_node(const FKStatic& P, const Env& e, const Slot& s, const Layout& lay, int n,
                            const FKLaunch& LL, long long kidx) {
  const double re = P.rnod[P.jre], r = P.rnod[n];
  const double elp1 = e.dll1, rlp1 = 1.0 / elp1, f = (r / re) * (r / re);
  const bool fluid = P.state[n] == 1;
  const double rr2 = 1.0 / (r * r), rr3 = rr2 / r;
  double ro; dz el[7];
  eval_spline<0x0Eu>(P, e.spl, r, P.layer[n], ro, el);
  dz zsph[4][4], ztor[2][2];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) zsph[i][j] = dz{0, 0};
  for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) ztor[i][j] = dz{0, 0};
  const double om = e.omre;
  if (P.istyp == 1) {
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
  auto put = [&](dz v) {
    long long o = kidx + LL.nkf * ((long long)isp + (long long)P.nsp * (n - 1));
    if (LL.gf64) LL.gf64[o] = make_double2(v.re, v.im);
    if (LL.gfre) LL.gfre[o] = (float)v.re;
    if (LL.gfim) LL.gfim[o] = (float)v.im;
    isp++;
  };
  for (int i = 0; i < P.ncsph; i += P.dsvstep)
    for (int l = 0; l < P.njsph; ++l) {
      dz g{0.0, 0.0};
      if (!fluid || l < 2) {
        g = bo[i][0] * zsph[0][l];
        for (int k = 1; k < nk; ++k) g = g + bo[i][k] * zsph[k][l];
      }
      put(g);
    }
  if (P.nctor > 0) {
    dz ti[2][2];
    for (int j = 0; j < 2; ++j) for (int c = 0; c < 2; ++c) ti[c][j] = s.get(lay.tor(n, j, c));
    dz bt[2][2];
    bt[0][0] = (-f) * ti[1][1]; bt[1][0] = f * ti[1][0];
    bt[0][1] = f * ti[0][1]; bt[1][1] = (-f) * ti[0][0];
    for (int i = 0; i < P.nctor; i += P.dsvstep)
      for (int l = 0; l < P.njtor; ++l) {
        dz g{0.0, 0.0};
        if (!fluid) g = bt[i][0] * ztor[0][l] + bt[i][1] * ztor[1][l];
        put(g);
      }
  }
}

// ------------------------------------------------------------------------
//  Per-lane bookkeeping: advance the item's state machine until the lane
//  needs an integration step (S_INTEG), a new item (S_FETCH) or is idle.
// ------------------------------------------------------------------------
__device__ __noinline__ void advance(const FKStatic& P, const FKLaunch& LL, const Slot& s, const Layout& lay,
                                     Lane& L) {
  const int jre = P.jre, nnod = P.nnod;
  for (int guard = 0; guard < 100000; ++guard) {
    switch (L.st) {
      case S_FETCH: case S_IDLE: case S_INTEG:
        return;

      case S_ITEM_INIT: {
        const int jf = LL.jf[L.slot];
        const double f = (double)(jf - 1) * P.df;
        L.e.spl = LL.spl + (long long)L.slot * (P.nk + 1) * SPL_STRIDE;
        L.e.nl = 1;
        L.e.omre = 2.0 * PI_F * f;
        L.e.omim = -P.sigma;
        double wn = (double)(L.iwn - 1) * P.dwn;
        if (P.global_ == 1) wn = sqrt((double)((long long)(L.iwn - 1) * L.iwn)) / P.rearth;
        L.e.dll1 = (wn * P.rearth) * (wn * P.rearth);
        L.status = ST_OK;
        L.det_t = dz{0, 0}; L.det_s = dz{0, 0};
        if (P.global_ == 0 && L.iwn == 1) { L.st = S_ITEM_END; break; }   // wn = 0 stays zero
        if (P.state[jre] == 1) { L.status = ST_UNSUPPORTED; L.st = S_ITEM_END; break; }
        for (int el = 0; el < lay.NN * Layout::PER_NODE; ++el) s.put(el, dz{0.0, 0.0});
        L.rstart_t = start_radius(P, L.e, true);
        L.rstart_s = start_radius(P, L.e, false);
        // ---- toroidal minors, downward from the surface (toroidalMinors.f90:150-199)
        L.st = S_TOR_DONE;
        if (L.e.dll1 < EPS_D || L.rstart_t >= P.rnod[jre]) break;
        double rmin = fmax(L.rstart_t, P.rnod[jre]);
        dz ys[5]; double htry, rsurf; int nl;
        int rc = toroidal_surface_iv(P, L.e, ys, htry, rsurf, nl);
        if (rc) { L.status = rc; L.st = S_ITEM_END; break; }
        if (rsurf < rmin) break;
        L.e.nl = nl;
        L.rend = rsurf;   // remembered for the upward limit
        prop_begin(P, s, lay, L, SYS_TOROIDAL, rsurf, rmin, htry, ys, false, 0.0, K_DT, S_TOR_UP);
        break;
      }

      case S_TOR_UP: {   // toroidalMinors.f90:206-240
        if (L.jr - L.jl < 0) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
        double rmax = fmin(P.rnod[jre], L.rend);
        int nl, top;
        layer_index(P, L.rstart_t, nl, top);
        if (top == 1) nl = nl + 1;
        L.e.nl = nl;
        dz ys[5]; double htry;
        int rc = toroidal_bottom_iv(P, L.e, L.rstart_t, ys, htry);
        if (rc) { L.status = rc; L.st = S_ITEM_END; break; }
        prop_begin(P, s, lay, L, SYS_TOROIDAL, L.rstart_t, rmax, htry, ys, false, 0.0, K_UT, S_TOR_DONE);
        L.up = 1;      // marks that the upward toroidal integration ran
        break;
      }

      case S_TOR_DONE: {
        if (L.up == 1) {
          if (L.jr - L.jl < 0) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
          L.det_t = s.get(lay.ut(jre, 0)) * s.get(lay.dt(jre, 1)) - s.get(lay.dt(jre, 0)) * s.get(lay.ut(jre, 1));
        }
        // ---- spheroidal minors (spheroidalMinors.f90:155-575)
        if (L.rstart_s >= P.rnod[jre]) { L.st = S_SPH_DONE; break; }
        L.up = 1;
        L.rbeg = L.rstart_s; L.rend = L.rstart_s; L.rlim = P.rnod[jre];
        L.lgnorm_g = 0.0; L.lgnormend = 0.0; L.htry_g = 0.0; L.liq_old = 0;
        L.st = S_SPH_GROUP;
        break;
      }

      case S_SPH_GROUP: {
        const bool up = L.up == 1;
        if (!(up ? L.rend < L.rlim : L.rend > L.rlim)) {
          // normalise to the final normalisation factor (spheroidalMinors.f90:360-365,552-557)
          for (int n = 1; n <= nnod; ++n) {
            double lgn = s.get(up ? lay.ulg(n) : lay.dlg(n)).re - L.lgnormend;
            double fct = pow(10.0, lgn);
            for (int c = 0; c < 6; ++c) {
              int el = up ? lay.um(n, c) : lay.dm(n, c);
              s.put(el, s.get(el) * fct);
            }
          }
          if (up) {
            L.up = 0;
            L.rbeg = P.rearth; L.rend = P.rearth; L.rlim = fmax(L.rstart_s, P.rnod[jre]);
            L.lgnorm_g = 0.0; L.lgnormend = 0.0; L.liq_old = 0;
            break;   // stay in S_SPH_GROUP for the downward sequence
          }
          dz u[6], d[6];
          for (int c = 0; c < 6; ++c) { u[c] = s.get(lay.um(jre, c)); d[c] = s.get(lay.dm(jre, c)); }
          if (P.state[jre] == 1 || L.e.dll1 < EPS_D) L.det_s = u[0] * d[1] - d[0] * u[1];
          else L.det_s = ((((u[0] * d[5] + u[5] * d[0]) - u[1] * d[4]) + u[2] * d[3]) + u[3] * d[2]) - u[4] * d[1];
          L.st = S_SPH_DONE;
          break;
        }
        int nl, top;
        layer_index(P, L.rbeg, nl, top);
        if (up && top == 1) nl = nl + 1;
        L.liq = P.iflso[nl] == 1;
        L.e.nl = nl;
        L.rend = up ? fmin(above_pc(P, nl), L.rlim) : fmax(below_pc(P, nl), L.rlim);
        const bool l0 = L.e.dll1 < EPS_D;
        int sys = L.liq ? SYS_FLUID : (l0 ? SYS_RADIAL : SYS_MINORS);
        dz ys[5] = {{0, 0}, {0, 0}, {0, 0}, {0, 0}, {0, 0}};
        if (L.rbeg == (up ? L.rstart_s : P.rearth)) {
          int rc = up ? minors_bottom_iv(P, L.e, L.rbeg, ys, L.htry_g) : minors_surface_iv(P, L.e, ys, L.htry_g);
          if (rc) { L.status = rc; L.st = S_ITEM_END; break; }
        } else if (L.liq && !L.liq_old) {
          if (l0) { ys[0] = L.yend[0]; ys[1] = L.yend[1]; } else { ys[0] = L.yend[2]; ys[1] = L.yend[4]; }
        } else if (!L.liq && L.liq_old) {
          if (l0) { ys[0] = L.yend[0]; ys[1] = L.yend[1]; }
          else { ys[3] = L.yend[1]; ys[1] = L.yend[0]; }
        } else {
          L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break;
        }
        prop_begin(P, s, lay, L, sys, L.rbeg, L.rend, L.htry_g, ys, true, L.lgnorm_g, up ? K_UM : K_DM,
                   S_SPH_GROUP_END);
        break;
      }

      case S_SPH_GROUP_END: {
        if (L.up == 0 && L.jr - L.jl < 0) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
        L.liq_old = L.liq;
        L.rbeg = L.rend;
        for (int v = 0; v < NV_MAX; ++v) L.yend[v] = L.y[v];
        L.lgnormend = L.lgnorm;
        L.lgnorm_g = L.lgnormend;
        L.st = S_SPH_GROUP;
        break;
      }

      case S_SPH_DONE: {
        // ---- toroidal unit jump Green functions (unitJumpGreenFunctions.f90:147-175)
        const int tor_mask = P.stressflag ? 3 : 2;
        if (zabs(L.det_t) > TINY_D) {
          for (int j = 0; j < 2; ++j) {
            if (!(tor_mask & (1 << j))) continue;
            double u1 = j == 0 ? 1.0 : 0.0, u2 = j == 1 ? 1.0 : 0.0;
            dz d = (u2 * s.get(lay.dt(jre, 0)) - u1 * s.get(lay.dt(jre, 1))) / L.det_t;
            for (int n = 1; n <= jre - 1; ++n)
              if (P.state[n] == 0 && P.rnod[n] > L.rstart_t)
                for (int c = 0; c < 2; ++c) s.put(lay.tor(n, j, c), d * s.get(lay.ut(n, c)));
            dz ee = (u2 * s.get(lay.ut(jre, 0)) - u1 * s.get(lay.ut(jre, 1))) / L.det_t;
            for (int n = jre; n <= nnod; ++n)
              if (P.state[n] == 0)
                for (int c = 0; c < 2; ++c) s.put(lay.tor(n, j, c), ee * s.get(lay.dt(n, c)));
          }
        }
        if (!(zabs(L.det_s) > TINY_D)) { L.st = S_OUTPUT; break; }
        if (L.e.dll1 < EPS_D) {   // l = 0 (:201-220)
          for (int j = 0; j < 2; ++j) {
            double u1 = j == 0 ? 1.0 : 0.0, u2 = j == 1 ? 1.0 : 0.0;
            dz d = (u2 * s.get(lay.dm(jre, 0)) - u1 * s.get(lay.dm(jre, 1))) / L.det_s;
            dz ee = (u2 * s.get(lay.um(jre, 0)) - u1 * s.get(lay.um(jre, 1))) / L.det_s;
            for (int n = jre; n <= nnod; ++n)
              for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), ee * s.get(lay.dm(n, c)));
            for (int n = jre - 1; n >= 1; --n)
              for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), d * s.get(lay.um(n, c)));
          }
          L.st = S_OUTPUT;
          break;
        }
        if (P.state[jre] == 1 && P.layer[jre] == P.nlay) { L.status = ST_UNSUPPORTED; L.st = S_ITEM_END; break; }
        // inner-core propagator P_4m (:227-238)
        double re_ic = fmax(L.rstart_s, P.rnod[1]);
        if (re_ic < P.ric) {
          dz ys[5] = {{0, 0}, {0, 0}, {0, 0}, {1.0, 0}, {0, 0}};
          double htry = adjoint_htry(P, L.e, P.ric, re_ic);
          prop_begin(P, s, lay, L, SYS_SOLIDT, P.ric, re_ic, htry, ys, false, 0.0, K_ADJIC, S_ADJ_PLAN);
        } else {
          L.st = S_ADJ_PLAN;
        }
        break;
      }

      case S_ADJ_PLAN: {
        if (L.sink == K_ADJIC && L.jr - L.jl < 0) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
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
        const int sph_mask = P.stressflag ? 15 : 10;
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
        for (int c = 0; c < 6; ++c) m[c] = s.get(upd ? lay.um(jre, c) : lay.dm(jre, c));
        meps_col(m, j, col);
        for (int c = 0; c < 4; ++c) ys[c] = upd ? dz{0.0, 0.0} - col[c] / L.det_s : dz{0.0, 0.0} + col[c] / L.det_s;
        ys[4] = dz{0, 0};
        const double ra = P.rnod[jre];
        const double xe = upd ? (L.ocean_above ? P.ruc : P.rnod[L.highest]) : (L.core_below ? L.re_dn : P.rnod[L.lowest]);
        double htry = adjoint_htry(P, L.e, ra, upd ? P.ruc : L.re_dn);
        prop_begin(P, s, lay, L, SYS_SOLIDT, ra, xe, htry, ys, false, 0.0, upd ? K_ADJ_UP : K_ADJ_DN, S_ADJ_END);
        break;
      }

      case S_ADJ_END: {
        if (L.jr - L.jl < 0) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
        const int j = L.stage >> 1;
        if ((L.stage & 1) == 0) {
          if (L.ocean_above)
            for (int n = jre; n <= nnod; ++n)
              if (P.state[n] == 1 && P.rnod[n] > P.ruc)
                for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), L.y[2] * s.get(lay.dm(n, c)));
        } else if (L.core_below) {
          dz a3 = L.y[2];
          for (int n = jre - 1; n >= 1; --n) {
            if (P.rnod[n] < L.rstart_s) continue;
            if (P.state[n] == 0 && P.rnod[n] < P.ric) {
              dz mm[6], a[4], out[4];
              for (int c = 0; c < 6; ++c) mm[c] = s.get(lay.um(n, c));
              for (int c = 0; c < 4; ++c) a[c] = s.get(lay.adjic(n, c));
              mtil_times(mm, a, out);
              for (int c = 0; c < 4; ++c) s.put(lay.sph(n, j, c), a3 * out[c]);
            } else if (P.state[n] == 1) {
              for (int c = 0; c < 2; ++c) s.put(lay.sph(n, j, c), a3 * s.get(lay.um(n, c)));
            }
          }
        }
        L.st = S_ADJ_NEXT;
        break;
      }

      case S_OUTPUT:
        for (int n = 1; n <= nnod; ++n) output_node(P, L.e, s, lay, n, LL, L.kidx);
        L.st = S_ITEM_END;
        break;

      case S_ITEM_END:
        if (LL.status) LL.status[L.kidx] = L.status;
        L.st = S_FETCH;
        return;

      // ---------------- propagator: next sub-interval (propagateOde.f90:218-246)
      case S_PROP_NEXT: {
        if (!(fabs(L.x2 - L.xa) > MINSIZE_IS)) {
          if (L.jnod - 1 != L.nnodp || L.jd - 1 != L.ndp) { L.status = ST_BOOKKEEPING; L.st = S_ITEM_END; break; }
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
          sink_node(P, s, lay, L, asc ? L.jl + L.jnod - 1 : L.jr - L.jnod + 1);
          L.jnod++;
          if (fabs(L.s0 - L.s1) < MINSIZE_IS) { L.e.nl += (int)L.idir; L.jd++; }
        } else if (L.kmin == 1) {
          L.jd++;
          L.e.nl += (int)L.idir;
          if (fabs(L.s0 - L.s1) < MINSIZE_IS) {
            sink_node(P, s, lay, L, asc ? L.jl + L.jnod - 1 : L.jr - L.jnod + 1);
            L.jnod++;
          }
        }
        L.xa = L.xe;
        L.st = S_PROP_NEXT;
        break;
      }
      default:
        L.status = ST_BOOKKEEPING; L.st = S_ITEM_END;
        break;
    }
  }
  L.status = ST_BOOKKEEPING;
  L.st = S_ITEM_END;
}

// ------------------------------------------------------------------------
//  The persistent kernel
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(FK_BLOCK, 1) fk_solve_kernel(const __grid_constant__ FKStatic P, FKLaunch LL) {
  extern __shared__ double2 smem_diag[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  double2* D = smem_diag + warp * DIAG_PER_WARP;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  Slot s{LL.scratch + tid, LL.nthreads};
  Layout lay{P.nnod + 1};
  Counters cnt{0, 0, 0, 0, 0, 0};
  Lane L;
  L.st = S_FETCH;
  L.up = 0;
  const unsigned FULL = 0xffffffffu;
  for (long long trip = 0;; ++trip) {
    // ---- refill lanes that finished their item, then advance bookkeeping
    for (int round = 0; round < 64; ++round) {
      unsigned fm = __ballot_sync(FULL, L.st == S_FETCH);
      if (fm) {
        int leader = __ffs(fm) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(LL.queue, (unsigned)__popc(fm));
        base = __shfl_sync(FULL, base, leader);
        if (L.st == S_FETCH) {
          unsigned my = base + __popc(fm & ((1u << lane) - 1u));
          if (my < (unsigned)LL.nitems) {
            int2 w = LL.items[my];
            L.slot = w.x; L.iwn = w.y;
            L.kidx = (long long)LL.koff[L.slot] + L.iwn - 1;
            L.up = 0;
            L.st = S_ITEM_INIT;
          } else {
            L.st = S_IDLE;
          }
        }
      }
      advance(P, LL, s, lay, L);
      if (!__any_sync(FULL, L.st == S_FETCH)) break;
    }
    const bool integ = L.st == S_INTEG;
    if (!__any_sync(FULL, integ)) {
      if (__all_sync(FULL, L.st == S_IDLE)) break;
      continue;
    }
    // ---- overshoot clamp (integrationStep.f90:136-139) and one lockstep BS step per system
    if (integ && (L.x + L.h - L.xe) * (L.x + L.h - L.xa) > 0.0) L.h = L.xe - L.x;
    unsigned sysmask = __reduce_or_sync(FULL, integ ? (1u << L.sys) : 0u);
    dz yext[NV_MAX];
    int result = 0;
    if (sysmask & (1u << SYS_MINORS))
      bs_step<SYS_MINORS>(P, L.e, integ && L.sys == SYS_MINORS, L.h, L.x, L.y, yext, result, D, lane, cnt);
    if (sysmask & (1u << SYS_SOLIDT)) {
      int r = 0;
      bs_step<SYS_SOLIDT>(P, L.e, integ && L.sys == SYS_SOLIDT, L.h, L.x, L.y, yext, r, D, lane, cnt);
      if (integ && L.sys == SYS_SOLIDT) result = r;
    }
    if (sysmask & (1u << SYS_TOROIDAL)) {
      int r = 0;
      bs_step<SYS_TOROIDAL>(P, L.e, integ && L.sys == SYS_TOROIDAL, L.h, L.x, L.y, yext, r, D, lane, cnt);
      if (integ && L.sys == SYS_TOROIDAL) result = r;
    }
    if (sysmask & (1u << SYS_FLUID)) {
      int r = 0;
      bs_step<SYS_FLUID>(P, L.e, integ && L.sys == SYS_FLUID, L.h, L.x, L.y, yext, r, D, lane, cnt);
      if (integ && L.sys == SYS_FLUID) result = r;
    }
    if (sysmask & (1u << SYS_RADIAL)) {
      int r = 0;
      bs_step<SYS_RADIAL>(P, L.e, integ && L.sys == SYS_RADIAL, L.h, L.x, L.y, yext, r, D, lane, cnt);
      if (integ && L.sys == SYS_RADIAL) result = r;
    }
    // ---- step-size control (integrationStep.f90:140-185)
    if (integ) {
      L.nstep++;
      if (result > 0) {
        cnt.steps_ok++;
        L.x = L.x + L.h;
        for (int v = 0; v < L.nv; ++v) L.y[v] = yext[v];
        if (fabs(L.x - L.xe) < MINSIZE_IS) {
          L.st = S_SUB_END;
        } else {
          if (result > 6) L.h = L.h * SHRINK_BS;
          else if (result < 6) L.h = L.h * GROW_BS;
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
  long long v[6] = {cnt.steps_ok, cnt.steps_rej, cnt.attempts, cnt.sysmats, cnt.matvecs, cnt.flops};
  for (int k = 0; k < 6; ++k) {
    long long x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(FULL, x, o);
    if (lane == 0) atomicAdd(LL.stats + k, (unsigned long long)x);
  }
}

}  // namespace gem
