// Travel-time table by ray tracing (computeTravelTimeTable.f90:160-226) on the GPU.
//
// One thread per turning radius integrates Delta(r) and T(r) of its ray from the
// turning point up to the top node: the real Bulirsch-Stoer step
// (episode/realBulirschStep.f90:130-307) on the ray system (rayOdeSystem.f90:151-170),
// with sub-intervals at the nodes and discontinuities as propagateOde.f90:132-331
// makes them, and the solution stored at every node it passes.  The spline
// tables are the model's at the reference frequency.  The file is built without
// FMA contraction, so the arithmetic repeats the reference's operation by operation.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "../../include/gemini_fk.h"

#define GEM_NS gem_ray
#define GEM_FAST 0
#include "fk_kernel.h"
#include "fk_solver.cuh"

namespace gem_ray {

struct RayLane {
  Env e;        // spline table and layer index
  int stype;    // 0 P, 1 S
  double p;     // angular slowness r/v at the turning point
};

// getPVelocitySplineEarthmodel / getSVelocitySplineEarthmodel (splineEarthmodelCoefficients.f90:192-210)
__device__ double ray_velocity(const FKStatic& P, const RayLane& R, int nl, double r) {
  double ro;
  dz el[7];
  eval_spline<0x60u>(P, R.e, r, nl, ro, el);
  if (R.stype == 0) return sqrt((el[5].re + (4.0 / 3.0) * el[6].re) / ro);
  return sqrt(el[6].re / ro);
}

// derivativeRealRayOdeSystem (rayOdeSystem.f90:151-170)
__device__ void ray_derivative(const FKStatic& P, const RayLane& R, double x, double* dy) {
  const double v = ray_velocity(P, R, R.e.nl, x);
  const double t = x / v;
  const double ur2 = t * t;
  const double q = sqrt(ur2 - R.p * R.p);
  dy[0] = R.p / (q * x);
  dy[1] = ur2 / (q * x);
}

// doFullStepRealBulirsch (realBulirschStep.f90:130-176) with the non-linear
// modified midpoint (:222-252) and the full-tableau extrapolation (:258-290);
// returns the number of attempts when it converged, 0 otherwise.
__device__ int ray_full_step(const FKStatic& P, const RayLane& R, double eps, double h, double xstart,
                             const double* y, double* yext) {
  double ysol[7][2];
  int ntry = 3, nfirst = 1;
  for (;;) {
    for (int j = nfirst; j <= ntry; ++j) {
      const int nstep = SEQDIV[j - 1];
      const double hdiv = h / (double)nstep;
      double z0[2] = {y[0], y[1]}, z1[2], z2[2], d[2];
      ray_derivative(P, R, xstart, d);
      for (int i = 0; i < 2; ++i) z1[i] = z0[i] + hdiv * d[i];
      for (int m = 1; m <= nstep - 1; ++m) {
        ray_derivative(P, R, xstart + (double)m * hdiv, d);
        for (int i = 0; i < 2; ++i) z2[i] = z0[i] + (2.0 * hdiv) * d[i];
        for (int i = 0; i < 2; ++i) { z0[i] = z1[i]; z1[i] = z2[i]; }
      }
      ray_derivative(P, R, xstart + h, d);
      for (int i = 0; i < 2; ++i) ysol[j - 1][i] = 0.5 * ((z1[i] + z0[i]) + hdiv * d[i]);
    }
    // extrapolation to h -> 0 over the ntry solutions
    const int n = ntry;
    double x[7], c[7][2], dd[7][2], yy[2], dy[2] = {0.0, 0.0};
    for (int j = 0; j < n; ++j) {
      x[j] = h / (double)SEQDIV[j];
      for (int i = 0; i < 2; ++i) { c[j][i] = ysol[j][i]; dd[j][i] = ysol[j][i]; }
    }
    int js = n;
    for (int i = 0; i < 2; ++i) yy[i] = ysol[js - 1][i];
    for (int m = 1; m <= n - 1; ++m) {
      for (int i = 1; i <= n - m; ++i) {
        const double hh = x[i - 1] - x[i + m - 1];
        for (int v = 0; v < 2; ++v) {
          const double u = (c[i][v] - dd[i - 1][v]) / hh;
          c[i - 1][v] = x[i - 1] * u;
          dd[i - 1][v] = x[i + m - 1] * u;
        }
      }
      for (int v = 0; v < 2; ++v) { yy[v] = yy[v] + dd[js - 2][v]; dy[v] = dd[js - 2][v]; }
      js = js - 1;
    }
    const double errmax = sqrt((dy[0] * dy[0] + dy[1] * dy[1]) / (yy[0] * yy[0] + yy[1] * yy[1]));
    if (errmax / eps < 1.0) {
      yext[0] = yy[0]; yext[1] = yy[1];
      return ntry;
    }
    if (ntry < 7) { ntry = ntry + 1; nfirst = ntry; }
    else return 0;
  }
}

// doIntegrationStep (integrationStep.f90:98-190) with adjustStepSizeRealBulirsch (:295-307)
__device__ int ray_integration_step(const FKStatic& P, const RayLane& R, double eps, double& hdid, double x1,
                                    double x2, double* y) {
  if (fabs(x2 - x1) < MINSIZE_IS) return 0;
  double x = x1;
  double h = copysign(hdid, x2 - x1);
  double ys[2] = {y[0], y[1]}, yext[2];
  for (int nstep = 0; nstep < MAXNUM_IS;) {
    if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
    const int done = ray_full_step(P, R, eps, h, x, ys, yext);
    nstep++;
    if (done > 0) {
      x = x + h;
      ys[0] = yext[0]; ys[1] = yext[1];
      if (fabs(x - x2) < MINSIZE_IS) { y[0] = ys[0]; y[1] = ys[1]; return 0; }
      if (done > 6) h = h * SHRINK_BS;
      else if (done < 6) h = h * GROW_BS;
      hdid = h;
    } else {
      h = 0.5 * h / 1.0;
      if (fabs(h) < MINSIZE_IS) return ST_MINSTEP;
    }
  }
  return ST_MAXSTEPS;
}

// table[(n*nnod + j-1)*2 + {0, 1}] = (Delta, T) at node j; status[n]: 0 ok, else the
// integrator's or the bookkeeping's status (the row then stays zero)
__global__ void __launch_bounds__(128) ray_table_kernel(const __grid_constant__ FKStatic P, const double* spl,
                                                        int ntp, int stype, double eps, double drtp, double a0,
                                                        double* rtp_out, double* slowness, float* table,
                                                        int* status) {
  __shared__ Tab tab;
  for (int i = threadIdx.x; i <= MAXKNOT; i += blockDim.x) tab.rk[i] = P.rk[i];
  for (int i = threadIdx.x; i <= MAXLAY; i += blockDim.x) {
    tab.drk[i] = P.drk[i]; tab.iktop[i] = P.iktop[i]; tab.rdrk[i] = 1.0 / P.drk[i];
  }
  __syncthreads();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= ntp) return;
  const int nnod = P.nnod;
  for (int j = 0; j < nnod; ++j) {
    table[((long long)n * nnod + j) * 2] = 0.0f;
    table[((long long)n * nnod + j) * 2 + 1] = 0.0f;
  }
  const double rtp = P.roc + (double)n * drtp;
  rtp_out[n] = rtp;
  RayLane R;
  R.e.tab = &tab; R.e.spl = spl; R.e.poly = nullptr; R.e.omre = R.e.omim = R.e.dll1 = 0.0;
  R.stype = stype;
  int nl, top;
  layer_index(P, rtp, nl, top);
  if (top == 1) nl = nl + 1;
  R.e.nl = nl;
  R.p = rtp / ray_velocity(P, R, nl, rtp);
  slowness[n] = R.p;
  double y[2] = {a0, R.p * a0};
  // propagateOde.f90:132-331 from rtp*(1+eps) to the top node
  const double x1 = rtp * (1.0 + eps), x2 = P.rnod[nnod];
  int nl0, nr0, dl0, dr0;
  node_range(P, x1, x2, nl0, nr0);
  disco_range(P, x1, x2, dl0, dr0);
  const int nn = nr0 - nl0 + 1 > 0 ? nr0 - nl0 + 1 : 0, nd = dr0 - dl0 + 1 > 0 ? dr0 - dl0 + 1 : 0;
  const double idir = copysign(1.0, x2 - x1);
  const bool asc = x2 >= x1;
  auto xn = [&](int k) { return asc ? P.rnod[nl0 + k - 1] : P.rnod[nr0 - k + 1]; };   // k = 1..nn
  auto xd = [&](int k) { return asc ? P.rb[dl0 + k - 1] : P.rb[dr0 - k + 1]; };
  auto sink = [&](int k) {
    const int j = asc ? nl0 + k - 1 : nr0 - k + 1;
    table[((long long)n * nnod + (j - 1)) * 2] = (float)y[0];
    table[((long long)n * nnod + (j - 1)) * 2 + 1] = (float)y[1];
  };
  int rc = 0;
  if (nn < 1) rc = ST_BOOKKEEPING;
  if (!rc && nd > 0 && ((x1 - xd(1)) * idir > 0 || (xd(nd) - x2) * idir > 0)) rc = ST_BOOKKEEPING;
  if (!rc && nn > 0 && ((x1 - xn(1)) * idir > 0 || (xn(nn) - x2) * idir > 0)) rc = ST_BOOKKEEPING;
  int jnod = 1, jd = 1;
  if (!rc) {
    if (fabs(x2 - x1) < MINSIZE_IS) {
      if (nn == 1) { sink(1); jnod = 2; }
      else rc = ST_BOOKKEEPING;
    } else {
      double hdid = drtp, xa = x1;
      while (!rc && fabs(x2 - xa) > MINSIZE_IS) {
        double s0 = 2.0 * fabs(x2 - x1), s1 = 3.0 * fabs(x2 - x1);
        const double s2 = fabs(x2 - xa);
        if (jnod <= nn) s0 = fabs(xn(jnod) - xa);
        if (jd <= nd) s1 = fabs(xd(jd) - xa);
        int kmin = 0;
        double smin = s0;
        if (s1 < smin) { kmin = 1; smin = s1; }
        if (s2 < smin) { kmin = 2; smin = s2; }
        const double xe = xa + idir * smin;
        rc = ray_integration_step(P, R, eps, hdid, xa, xe, y);
        if (rc) break;
        if (kmin == 0) {
          sink(jnod);
          jnod++;
          if (fabs(s0 - s1) < MINSIZE_IS) { R.e.nl += (int)idir; jd++; }
        } else if (kmin == 1) {
          jd++;
          R.e.nl += (int)idir;
          if (fabs(s0 - s1) < MINSIZE_IS) { sink(jnod); jnod++; }
        }
        xa = xe;
      }
    }
  }
  if (!rc && (jnod - 1 != nn || jd - 1 != nd)) rc = ST_BOOKKEEPING;
  if (rc) {
    for (int j = 0; j < nnod; ++j) {
      table[((long long)n * nnod + j) * 2] = 0.0f;
      table[((long long)n * nnod + j) * 2 + 1] = 0.0f;
    }
  }
  status[n] = rc;
}

cudaError_t launch_ray_table(const FKStatic& P, const double* spl, int ntp, int stype, double eps, double drtp,
                             double a0, double* rtp, double* slowness, float* table, int* status, cudaStream_t st) {
  ray_table_kernel<<<(ntp + 127) / 128, 128, 0, st>>>(P, spl, ntp, stype, eps, drtp, a0, rtp, slowness, table,
                                                      status);
  return cudaGetLastError();
}

}  // namespace gem_ray

// ---------------------------------------------------------------------------
//  Travel-time lookup (travelTimes.f90: setSourceInfoTravelTimes,
//  getReceiverTravelTimes, getTravelTimes), host code on the table as the
//  reference reads it back: float32 radii, slownesses and (Delta, T).
// ---------------------------------------------------------------------------
namespace {
// locate (locatePoint.f90:72-101) on a 1-based view x[1..n]
template <class T, class U>
int locate_h(U xx, int n, const T* x) {
  int lidx = 0, ridx = n + 1;
  const bool asc = x[n] > x[1];
  while (ridx - lidx > 1) {
    const int midx = (lidx + ridx) >> 1;
    const bool gt = xx > x[midx];
    if (asc) { if (gt) lidx = midx; else ridx = midx; }
    else { if (gt) ridx = midx; else lidx = midx; }
  }
  return lidx;
}

// findZeroPassTravelTimes (travelTimes.f90:385-414), mode 'end', a[1..n]
int zero_pass_end(double x, int n, const double* a) {
  double amax = a[1], amin = a[1];
  for (int j = 2; j <= n; ++j) { amax = a[j] > amax ? a[j] : amax; amin = a[j] < amin ? a[j] : amin; }
  if (x > amax || x < amin) return -1;
  int j = n;
  double prod = 1.0;
  while (prod > 0.0 && j > 1) {
    prod = (x - a[j - 1]) * (x - a[j]);
    j = j - 1;
  }
  return j;
}
}  // namespace

int gem_set_error(gem_ctx* ctx, const char* msg);

namespace {
int travel_times(int nnod, int ntp, const float* rnod0, const float* rtp0, const float* slow0, const float* table,
                 int istele, double rs, int n, const double* re, const double* delta, double* tt, const char** why) {
  const float* rnod = rnod0 - 1;   // 1-based views as in the reference
  const float* rtp = rtp0 - 1;
  const float* slow = slow0 - 1;
  auto D = [&](int j, int i) { return table[((long long)(i - 1) * nnod + (j - 1)) * 2]; };       // delta(j, i)
  auto TT = [&](int j, int i) { return table[((long long)(i - 1) * nnod + (j - 1)) * 2 + 1]; };  // ttime(j, i)
  const double tol = 1.0e-5;
  // setSourceInfoTravelTimes (:105-140)
  int js = locate_h((float)rs, nnod, rnod);
  if (js == 0) {
    if (std::fabs(rnod[js + 1] - rs) > tol * rs) { *why = "source radius below ray table range"; return GEM_ERROR; }
    js = 1;
  } else if (js == nnod) {
    if (std::fabs(rnod[js] - rs) > tol * rs) { *why = "source radius above ray table range"; return GEM_ERROR; }
    js = nnod - 1;
  }
  const int jtps = locate_h((float)rs, ntp, rtp);
  if (jtps == 0) { *why = "no turning point below source"; return GEM_ERROR; }
  double h = rnod[js + 1] - rnod[js];
  const double as = (rnod[js + 1] - rs) / h;
  const double bs = 1.0 - as;
  std::vector<double> delv((size_t)ntp + 1), tauv((size_t)ntp + 1);
  for (int s = 0; s < n; ++s) {
    // getReceiverTravelTimes (:141-247)
    tt[s] = -1.0;
    const double r = re[s], din = delta[s];
    const int jtpr = locate_h((float)r, ntp, rtp);
    if (jtpr == 0) { *why = "no turning point below receiver"; return GEM_ERROR; }
    int je = locate_h((float)r, nnod, rnod);
    if (je == 0) {
      if (std::fabs(rnod[je + 1] - r) > tol * r) { *why = "receiver radius below ray table range"; return GEM_ERROR; }
      je = 1;
    } else if (je == nnod) {
      if (std::fabs(rnod[je] - r) > tol * r) { *why = "receiver radius above ray table range"; return GEM_ERROR; }
      je = nnod - 1;
    }
    h = rnod[je + 1] - rnod[je];
    const double ae = (rnod[je + 1] - r) / h;
    const double be = 1.0 - ae;
    const int jtpmax = jtps < jtpr ? jtps : jtpr;
    double dmax = 0.0, dmin = 0.0;
    for (int i = 1; i <= jtpmax; ++i) {
      delv[i] = as * D(js, i) + bs * D(js + 1, i) + ae * D(je, i) + be * D(je + 1, i);
      if (i == 1 || delv[i] > dmax) dmax = delv[i];
      if (i == 1 || delv[i] < dmin) dmin = delv[i];
    }
    double ad, bd;
    int jd;
    if (din >= dmin) {
      for (int i = 1; i <= jtpmax; ++i)
        tauv[i] = as * TT(js, i) + bs * TT(js + 1, i) + ae * TT(je, i) + be * TT(je + 1, i) - slow[i] * delv[i];
      if (din > dmax) {
        tt[s] = tauv[1] + slow[1] * din;
        continue;
      }
      jd = istele ? locate_h(din, jtpmax, delv.data()) : zero_pass_end(din, jtpmax, delv.data());
      if (jd < 0) { *why = "zero not found, this should not happen as range was checked"; return GEM_ERROR; }
      h = delv[jd + 1] - delv[jd];
      ad = (delv[jd + 1] - din) / h;
      bd = 1.0 - ad;
    } else {
      if (istele) { *why = "Delta out of turning point range"; return GEM_ERROR; }
      for (int i = 1; i <= jtpmax; ++i) {
        delv[i] = as * D(js, i) + bs * D(js + 1, i) - ae * D(je, i) - be * D(je + 1, i);
        tauv[i] = as * TT(js, i) + bs * TT(js + 1, i) - ae * TT(je, i) - be * TT(je + 1, i) - slow[i] * delv[i];
      }
      jd = locate_h(din, jtpmax, delv.data());
      if (jd == 0) {
        jd = 1;
        h = delv[jd + 1] - delv[jd];
        if (std::fabs(h) < 1.0e-4) { ad = 1.0; bd = 0.0; }
        else { ad = (delv[jd + 1] - din) / h; bd = 1.0 - ad; }
      } else if (jd == jtpmax) {
        jd = jtpmax - 1;
        h = delv[jd + 1] - delv[jd];
        if (std::fabs(h) < 1.0e-4) { ad = 0.0; bd = 1.0; }
        else { ad = (delv[jd + 1] - din) / h; bd = 1.0 - ad; }
      } else {
        h = delv[jd + 1] - delv[jd];
        ad = (delv[jd + 1] - din) / h;
        bd = 1.0 - ad;
      }
    }
    const double tau = ad * tauv[jd] + bd * tauv[jd + 1];
    const double p = ad * slow[jd] + bd * slow[jd + 1];
    tt[s] = tau + p * din;
  }
  return GEM_OK;
}
}  // namespace

extern "C" int gem_travel_times(gem_ctx* ctx, int nnod, int ntp, const float* rnod, const float* rtp,
                                const float* slowness, const float* table, int istele, double rs, int n,
                                const double* re, const double* delta, double* tt) {
  if (!ctx) return GEM_ERROR;
  if (!rnod || !rtp || !slowness || !table || !re || !delta || !tt || nnod < 2 || ntp < 2 || n < 0)
    return gem_set_error(ctx, "travel times: invalid arguments");
  const char* why = nullptr;
  const int rc = travel_times(nnod, ntp, rnod, rtp, slowness, table, istele, rs, n, re, delta, tt, &why);
  if (rc != GEM_OK) return gem_set_error(ctx, why);
  return GEM_OK;
}
