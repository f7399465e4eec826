// =============================================================================
//  GEMINI FK hot path -- CPU FP64 ORACLE, phase 1 (FK spectra).
//  Test infrastructure only; see oracle_core.h for the conventions.
//
//  Restates, in order:
//    nodeEarthmodel.f90:98-330,599-663      (model, layer lookup)
//    complexElasticConstants.f90:48-106      (complex VTI constants)
//    cubicSpline.f90:74-109,176-221          (natural spline, LAPACK dgtsv)
//    splineEarthmodelCoefficients.f90:46-188 (spline coefficients, evaluation)
//    externalRadialNodes.f90:82-156,337-418  (external nodes)
//    geminiIntegrationEnvironment.f90:59-203 (nodes / discontinuities)
//    minors/fluid/radial/toroidal/solidtOdeSystem.f90 (system matrices)
//    episode/complexBulirschStep.f90:111-359, integrationStep.f90:98-190,
//    propagateOde.f90:132-331                (integrator)
//    initialValues.f90:71-574                (start radius, initial values)
//    toroidalMinors.f90:71-268, spheroidalMinors.f90:72-585,
//    spheroidalAdjoint.f90:53-159, unitJumpGreenFunctions.f90:62-380,
//    reciprocity.f90:82-180, sourceTerms.f90:59-118,
//    computeGreenFKSpectraForSynthetics.f90:186-236,380-501 (FK driver)
//    computeGreenFKSpectraForASKI.f90:196-233,451-541, dsvDerivatives.f90:39-72,
//    solidOdeSystem.f90:77-114               (DSV spectra with derivatives)
// =============================================================================
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oracle_core.h"

using namespace orc;

// ---------------------------------------------------------------------------
//  Flat input descriptions shared with the Python test harness (ctypes).
// ---------------------------------------------------------------------------
extern "C" {
typedef struct {
  double fref, rearth, ric, roc;
  int aniflag, fsflag, equidis, nlay, nk, nic, noc;
  const int* iflso;   // [nlay]
  const int* iktop;   // [nlay], 1-based knot index of layer top
  const double* rb;   // [nlay], radius of layer top
  const double* depth;  // [nk]
  const double* ro;
  const double* vpv;
  const double* vph;
  const double* vsv;
  const double* vsh;
  const double* eta;
  const double* qk;   // Qkappa
  const double* qm;   // Qmu
} or_model_desc;

typedef struct {
  double tlen, fmax, fmin, p1lim, p2lim, frac, xlen, eps;
  int global;      // 1 global (Legendre), 0 regional (Bessel)
  int attmode;     // 0 ELASTIC 1 ATTENUATION_ONLY 2 DISPERSION_ONLY 3 ATTENUATION_AND_DISPERSION
  int istyp;       // 0 FORCE 1 MOMENT
  int stressflag;  // 0/1
  int jre;         // receiver node (1-based)
} or_fk_params;
}

// ===========================================================================
//  Earth model (nodeEarthmodel.f90)
// ===========================================================================
struct Model {
  double fref, rearth, ric, roc;
  int aniflag, fsflag, equidis, nlay, nk, nic, noc;
  std::vector<int> iflso, iktop, ikbot;    // 1-based storage [0] unused
  std::vector<double> rb, drk;             // 1-based
  std::vector<double> rk, ro, vpv, vph, vsv, vsh, eta, qkinv, qminv;  // 1-based
};

static void buildModel(const or_model_desc* d, Model& m) {
  m.fref = d->fref; m.rearth = d->rearth; m.ric = d->ric; m.roc = d->roc;
  m.aniflag = d->aniflag; m.fsflag = d->fsflag; m.equidis = d->equidis;
  m.nlay = d->nlay; m.nk = d->nk; m.nic = d->nic; m.noc = d->noc;
  int L = m.nlay, K = m.nk;
  m.iflso.assign(L + 1, 0); m.iktop.assign(L + 1, 0); m.ikbot.assign(L + 1, 0);
  m.rb.assign(L + 1, 0.0); m.drk.assign(L + 1, 0.0);
  for (int i = 1; i <= L; ++i) {
    m.iflso[i] = d->iflso[i - 1]; m.iktop[i] = d->iktop[i - 1]; m.rb[i] = d->rb[i - 1];
  }
  m.ikbot[1] = 0;                                   // nodeEarthmodel.f90:165-166
  for (int i = 2; i <= L; ++i) m.ikbot[i] = m.iktop[i - 1] + 1;
  auto cp = [&](std::vector<double>& v, const double* s) {
    v.assign(K + 1, 0.0); for (int i = 1; i <= K; ++i) v[i] = s[i - 1]; };
  m.rk.assign(K + 1, 0.0);
  for (int i = 1; i <= K; ++i) m.rk[i] = m.rearth - d->depth[i - 1];   // :175
  // nodeEarthmodel.f90:184-190 drk per layer
  if (m.equidis == 1) {
    m.drk[1] = -1.0;
    for (int nl = 2; nl <= L; ++nl)
      m.drk[nl] = (m.rk[m.iktop[nl]] - m.rk[m.ikbot[nl]]) / (double)(m.iktop[nl] - m.ikbot[nl]);
  } else {
    for (int nl = 1; nl <= L; ++nl) m.drk[nl] = -1.0;
  }
  cp(m.ro, d->ro);
  m.qkinv.assign(K + 1, 0.0); m.qminv.assign(K + 1, 0.0);
  for (int i = 1; i <= K; ++i) {
    m.qkinv[i] = 1.0 / d->qk[i - 1];                 // :206
    m.qminv[i] = 1.0 / d->qm[i - 1];                 // :213
    if (m.qminv[i] < 0.0) m.qminv[i] = 0.0;          // :214
  }
  if (m.aniflag == 0) {                              // :217-238
    cp(m.vpv, d->vpv); cp(m.vph, d->vpv); cp(m.vsv, d->vsv); cp(m.vsh, d->vsv);
    m.eta.assign(K + 1, 1.0);
  } else {
    cp(m.vpv, d->vpv); cp(m.vph, d->vph); cp(m.vsv, d->vsv); cp(m.vsh, d->vsh); cp(m.eta, d->eta);
  }
}

// locatePoint.f90:72-101 (double version; note the n==1 "descending" branch)
static int locate(double xx, int n, const double* x /*1-based*/) {
  int lidx = 0, ridx = n + 1;
  while (ridx - lidx > 1) {
    int midx = (lidx + ridx) / 2;
    if (x[n] > x[1]) {
      if (xx > x[midx]) lidx = midx; else ridx = midx;
    } else {
      if (xx > x[midx]) ridx = midx; else lidx = midx;
    }
  }
  return lidx;
}

// nodeEarthmodel.f90:599-607
static void layerIndex(const Model& m, double r, int& nl, int& top) {
  top = 0;
  nl = locate(r, m.nlay, m.rb.data()) + 1;
  int nlc = std::min(nl, m.nlay);   // guard: r above the model top (not expected)
  if (std::fabs(r / m.rb[nlc] - 1.0) < EPS_D) top = 1;
}
// nodeEarthmodel.f90:616-636
static double abovePhaseChange(const Model& m, int nl) {
  int npc;
  if (m.iflso[nl] == 1) npc = nl;
  else if (nl < m.noc) npc = m.noc - 1;
  else if (nl > m.noc) npc = (m.iflso[m.nlay] == 1) ? m.nlay - 1 : m.nlay;
  else npc = m.nlay;
  return m.rb[npc];
}
// nodeEarthmodel.f90:645-663
static double belowPhaseChange(const Model& m, int nl) {
  int npc;
  if (m.iflso[nl] == 1) npc = nl;
  else if (nl < m.noc) npc = 1;
  else if (nl > m.noc) npc = m.noc + 1;
  else npc = nl;
  return m.rb[npc - 1];
}
static bool hasCore(const Model& m) { return m.noc > 0 && m.iflso[m.noc] == 1; }
static bool hasOcean(const Model& m) { return m.iflso[m.nlay] == 1; }
static double ruc(const Model& m) { return hasOcean(m) ? m.rb[m.nlay - 1] : m.rearth; }

// ===========================================================================
//  Complex elastic constants (complexElasticConstants.f90:48-106)
// ===========================================================================
static void complexVTI(double fratio, double ro, double alfv, double alfh, double betv,
                       double beth, double eta, double qkinv, double qminv, zc* z /*7*/) {
  double phik = std::atan(qkinv), phim = std::atan(qminv);
  zc zqk = Z(std::cos(phik), std::sin(phik)) * std::pow(fratio, 2.0 * phik / PI_F);
  zc zqm = Z(std::cos(phim), std::sin(phim)) * std::pow(fratio, 2.0 * phim / PI_F);
  if (betv > (double)1.e-6f) {
    double epa = ro * alfh * alfh, epc = ro * alfv * alfv;
    double epn = ro * beth * beth, epl = ro * betv * betv;
    double epf = eta * (epa - 2.0 * epl);
    double kappa = (epc + 4.0 * epa - 4.0 * epn + 4.0 * epf) / 9.0;
    double mue = (epc + epa + 6.0 * epl + 5.0 * epn - 2.0 * epf) / 15.0;
    double lamp2mue = kappa + 4.0 * mue / 3.0;
    double lambda = kappa - 2.0 * mue / 3.0;
    double da = epa - lamp2mue, dc = epc - lamp2mue, df = epf - lambda;
    double dn = epn - mue, dl = epl - mue;
    zc zkap = kappa * zqk, zmue = mue * zqm;
    zc zl2m = zkap + (4.0 * zmue) / 3.0;
    zc zlam = zkap - (2.0 * zmue) / 3.0;
    z[0] = zl2m + da; z[1] = zl2m + dc; z[4] = zmue + dn; z[3] = zmue + dl;
    z[2] = zlam + df; z[5] = zkap; z[6] = zmue;
  } else {
    double kappa = ro * alfv * alfv;
    zc zkap = kappa * zqk;
    z[6] = Z(0.0); z[0] = zkap; z[1] = zkap; z[2] = zkap; z[3] = Z(0.0); z[4] = Z(0.0); z[5] = zkap;
  }
}

// LAPACK dgtsv (NRHS = 1): Gaussian elimination with partial pivoting.
// Arrays 1-based: dl[1..n-1], d[1..n], du[1..n-1], b[1..n].
static int dgtsv1(int n, double* dl, double* d, double* du, double* b) {
  if (n == 0) return 0;
  for (int i = 1; i <= n - 2; ++i) {
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        b[i + 1] = b[i + 1] - fact * b[i];
      } else return i;
      dl[i] = 0.0;
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      double temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      dl[i] = du[i + 1];
      du[i + 1] = -fact * dl[i];
      du[i] = temp;
      temp = b[i];
      b[i] = b[i + 1];
      b[i + 1] = temp - fact * b[i + 1];
    }
  }
  if (n > 1) {
    int i = n - 1;
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] != 0.0) {
        double fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        b[i + 1] = b[i + 1] - fact * b[i];
      } else return i;
    } else {
      double fact = d[i] / dl[i];
      d[i] = dl[i];
      double temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      du[i] = temp;
      temp = b[i];
      b[i] = b[i + 1];
      b[i + 1] = temp - fact * b[i + 1];
    }
  }
  if (d[n] == 0.0) return n;
  b[n] = b[n] / d[n];
  if (n > 1) b[n - 1] = (b[n - 1] - du[n - 1] * b[n]) / d[n - 1];
  for (int i = n - 2; i >= 1; --i) b[i] = (b[i] - du[i] * b[i + 1] - dl[i] * b[i + 2]) / d[i];
  return 0;
}

// cubicSpline.f90:74-109 -- y2 of a natural spline through (x,y), 1-based, n points
static int doubleCubicSpline(int n, const double* x, const double* y, double* y2) {
  std::vector<double> dl(n + 2, 0.0), d(n + 2, 0.0), du(n + 2, 0.0);
  for (int j = 2; j <= n - 1; ++j) {
    dl[j - 1] = (x[j] - x[j - 1]) / 6.0;
    d[j] = (x[j + 1] - x[j - 1]) / 3.0;
    du[j] = (x[j + 1] - x[j]) / 6.0;
    y2[j] = (y[j + 1] - y[j]) / (x[j + 1] - x[j]) - (y[j] - y[j - 1]) / (x[j] - x[j - 1]);
  }
  d[1] = x[2] - x[1];
  d[n] = x[n] - x[n - 1];
  du[1] = 0.0;
  dl[n - 1] = 0.0;
  y2[1] = 0.0;
  y2[n] = 0.0;
  return dgtsv1(n, dl.data(), d.data(), du.data(), y2);
}

// ===========================================================================
//  Spline coefficients for one frequency (splineEarthmodelCoefficients.f90)
// ===========================================================================
struct Spline {
  int nk, nlay, equidis;
  std::vector<double> rk, ro, ro2, drk;   // 1-based
  std::vector<int> iktop;
  std::vector<zc> el, el2;                // [(k-1)*7 + c], 1-based k
};

static int computeSpline(const Model& m, double f, int attmode, Spline& s) {
  s.nk = m.nk; s.nlay = m.nlay; s.equidis = m.equidis;
  s.rk = m.rk; s.drk = m.drk; s.iktop = m.iktop;
  s.ro.assign(m.nk + 1, 0.0); s.ro2.assign(m.nk + 1, 0.0);
  s.el.assign((m.nk + 1) * 7, Z(0.0)); s.el2.assign((m.nk + 1) * 7, Z(0.0));
  // nodeEarthmodel.f90:287-330
  for (int j = 1; j <= m.nk; ++j) {
    double fr; double qk, qm;
    switch (attmode) {
      case 0: fr = 1.0; qk = 0.0; qm = 0.0; break;
      case 1: fr = 1.0; qk = m.qkinv[j]; qm = m.qminv[j]; break;
      case 2: fr = f / m.fref; qk = 0.0; qm = 0.0; break;
      default: fr = f / m.fref; qk = m.qkinv[j]; qm = m.qminv[j]; break;
    }
    complexVTI(fr, m.ro[j], m.vpv[j], m.vph[j], m.vsv[j], m.vsh[j], m.eta[j], qk, qm, &s.el[j * 7]);
    s.ro[j] = m.ro[j];
  }
  // do not spline the halfspace (layer 1): splineEarthmodelCoefficients.f90:68-87
  for (int nl = 2; nl <= m.nlay; ++nl) {
    int j1 = m.ikbot[nl], j2 = m.iktop[nl], n = j2 - j1 + 1;
    const double* x = &s.rk[j1 - 1];
    if (doubleCubicSpline(n, x, &s.ro[j1 - 1], &s.ro2[j1 - 1])) return 2;
    std::vector<double> y(n + 1), y2(n + 1);
    for (int k = 0; k < 7; ++k) {
      for (int i = 1; i <= n; ++i) y[i] = s.el[(j1 - 1 + i) * 7 + k].re;
      if (doubleCubicSpline(n, x, y.data(), y2.data())) return 2;
      for (int i = 1; i <= n; ++i) s.el2[(j1 - 1 + i) * 7 + k] = Z(y2[i], 0.0);
      for (int i = 1; i <= n; ++i) y[i] = s.el[(j1 - 1 + i) * 7 + k].im;
      if (doubleCubicSpline(n, x, y.data(), y2.data())) return 2;
      // zy2 = zy2 + zi*y2  (cubicSpline.f90:215-217)
      for (int i = 1; i <= n; ++i) {
        zc& t = s.el2[(j1 - 1 + i) * 7 + k];
        t = t + Z(0.0, 1.0) * y2[i];
      }
    }
  }
  return 0;
}

// splineEarthmodelCoefficients.f90:118-162
static void evalSpline(const Spline& s, double r, int nl, double& ro, zc* z) {
  if (nl == 1) {
    int j = s.iktop[1];
    ro = s.ro[j];
    for (int c = 0; c < 7; ++c) z[c] = s.el[j * 7 + c];
    return;
  }
  int j1 = s.iktop[nl - 1] + 1, j2 = s.iktop[nl], j;
  if (j2 - j1 == 1) j = j1;
  else if (s.equidis == 1) {
    j = (int)((r - s.rk[j1]) / s.drk[nl]) + j1;
    if (j == j2) j = j2 - 1;
  } else {
    j = j1 - 1; int jr = j2 + 1;
    while (jr - j > 1) { int mm = (j + jr) / 2; if (r > s.rk[mm]) j = mm; else jr = mm; }
    if (j == j1 - 1) j = j1;
  }
  j = std::max(1, std::min(j, s.nk - 1));   // memory guard only (in-range inputs unaffected)
  double x1 = s.rk[j], x2 = s.rk[j + 1], h = x2 - x1;
  double a = (x2 - r) / h, b = 1.0 - a;
  if (j2 - j1 == 1) {
    ro = a * s.ro[j] + b * s.ro[j + 1];
    for (int c = 0; c < 7; ++c) z[c] = a * s.el[j * 7 + c] + b * s.el[(j + 1) * 7 + c];
  } else {
    double cc = h * h * a * (a * a - 1.0) / 6.0;
    double dd = h * h * b * (b * b - 1.0) / 6.0;
    ro = a * s.ro[j] + b * s.ro[j + 1] + cc * s.ro2[j] + dd * s.ro2[j + 1];
    for (int c = 0; c < 7; ++c)
      z[c] = a * s.el[j * 7 + c] + b * s.el[(j + 1) * 7 + c] + cc * s.el2[j * 7 + c] +
             dd * s.el2[(j + 1) * 7 + c];
  }
}

// ===========================================================================
//  External radial nodes (externalRadialNodes.f90:82-156,337-418)
// ===========================================================================
struct Nodes {
  int nnod;
  std::vector<double> r;   // 1-based
  std::vector<int> state, layer;
};

static int splitNodes(const Model& m, int nnod, const double* prn /*1-based*/, Nodes& ex) {
  const double* rb = m.rb.data();
  int L = m.nlay;
  double drmin = rb[L] * 1.e-4;
  ex.r.assign(nnod + 2 * L + 1, 0.0); ex.state.assign(nnod + 2 * L + 1, 0);
  ex.layer.assign(nnod + 2 * L + 1, 0);
  int je = 0, ne = 0;
  for (int ib = 1; ib <= L; ++ib) {
    int n = locate(rb[ib], nnod, prn);
    if (n == 0) continue;
    int iflso = m.iflso[ib];
    for (int k = 0; k < n - ne; ++k) {
      ex.r[je + 1 + k] = prn[ne + 1 + k]; ex.layer[je + 1 + k] = ib; ex.state[je + 1 + k] = iflso;
    }
    je = je + n - ne;
    if (n >= nnod) break;
    if (std::fabs(prn[n + 1] - rb[ib]) < drmin && std::fabs(prn[n] - rb[ib]) < drmin) return 2;
    if (std::fabs(prn[n + 1] - rb[ib]) < drmin) {
      ex.r[je + 1] = rb[ib] - drmin * 0.5; ex.layer[je + 1] = ib; ex.state[je + 1] = iflso;
      if (n + 1 < nnod) {
        ex.r[je + 2] = rb[ib] + drmin * 0.5; ex.layer[je + 2] = ib + 1; ex.state[je + 2] = m.iflso[ib + 1];
        je += 2; ne = n + 1;
      } else {
        je += 1; ne = n;
      }
    } else if (std::fabs(prn[n] - rb[ib]) < drmin) {
      ex.r[je] = rb[ib] - drmin * 0.5; ex.layer[je] = ib; ex.state[je] = iflso;
      ex.r[je + 1] = rb[ib] + drmin * 0.5; ex.layer[je + 1] = ib + 1; ex.state[je + 1] = m.iflso[ib + 1];
      je += 1; ne = n;
    } else {
      ne = n;
      ex.r[je + 1] = rb[ib] - drmin * 0.5; ex.layer[je + 1] = ib; ex.state[je + 1] = iflso;
      ex.r[je + 2] = rb[ib] + drmin * 0.5; ex.layer[je + 2] = ib + 1; ex.state[je + 2] = m.iflso[ib + 1];
      je += 2;
    }
  }
  ex.nnod = je;
  ex.r.resize(je + 1); ex.state.resize(je + 1); ex.layer.resize(je + 1);
  return 0;
}

static int createNodes(const Model& m, int nblocks, const int* nnodb, const double* drb,
                       double shift, double rearth, Nodes& ex) {
  int nnod = 1;
  for (int b = 0; b < nblocks; ++b) nnod += nnodb[b];
  std::vector<double> prn(nnod + 1);
  prn[nnod] = rearth - shift;
  int n = nnod;
  for (int ib = 0; ib < nblocks; ++ib) {
    for (int i = 1; i <= nnodb[ib]; ++i) prn[n - i] = prn[n] - i * drb[ib];
    n -= nnodb[ib];
  }
  for (int i = 1; i <= nnod; ++i) if (prn[i] < 0.0) return 2;
  return splitNodes(m, nnod, prn.data(), ex);
}

// ===========================================================================
//  Integration environment (geminiIntegrationEnvironment.f90)
// ===========================================================================
struct Env {
  int nl;
  double omre, omim, dll1;
  const Model* m;
  const Nodes* ex;
  const Spline* s;
};

// getDiscontinuitiesGemini :96-144
static void getDiscos(const Env& e, double x1, double x2, int& jl, int& jr, std::vector<double>& xd) {
  xd.clear();
  double xl = x1, xr = x2;
  if (x1 > x2) { xl = x2; xr = x1; }
  const Model& m = *e.m;
  int n = m.nlay;
  const double* rb = m.rb.data();
  jl = locate(xl, n, rb) + 1;
  if (jl > n) { jr = jl - 1; return; }
  if (std::fabs(1.0 - xl / rb[jl]) < EPS_D) jl = jl + 1;
  if (jl >= n) { jr = jl - 1; return; }
  jr = locate(xr, n, rb);
  if (jr == 0) { jr = 0; jl = 1; return; }
  int nd = jr - jl + 1;
  if (nd > 0) {
    if (x2 >= x1) for (int k = jl; k <= jr; ++k) xd.push_back(rb[k]);
    else for (int k = jr; k >= jl; --k) xd.push_back(rb[k]);
  }
}

// getNodesGemini :160-203
static void getNodes(const Env& e, double x1, double x2, int& jl, int& jr, std::vector<double>& xn) {
  xn.clear();
  double xl = x1, xr = x2;
  if (x1 > x2) { xl = x2; xr = x1; }
  const Nodes& ex = *e.ex;
  int n = ex.nnod;
  const double* rn = ex.r.data();
  jl = locate(xl, n, rn) + 1;
  if (jl > n) { jr = jl - 1; return; }
  jr = locate(xr, n, rn);
  if (jr < n) { if (std::fabs(1.0 - xr / rn[jr + 1]) < EPS_D) jr = jr + 1; }
  if (jr == 0) { jr = 0; jl = 1; return; }
  int nn = jr - jl + 1;
  if (nn > 0) {
    if (x2 >= x1) for (int k = jl; k <= jr; ++k) xn.push_back(rn[k]);
    else for (int k = jr; k >= jl; --k) xn.push_back(rn[k]);
  }
}

// ===========================================================================
//  ODE systems (system matrices, column-major a[i + nvar*j], 0-based)
// ===========================================================================
enum Sys { SYS_MINORS = 0, SYS_FLUID = 1, SYS_RADIAL = 2, SYS_TOROIDAL = 3, SYS_SOLIDT = 4 };
static int nvarOf(int sys) { static const int nv[5] = {5, 2, 2, 2, 4}; return nv[sys]; }

static void sysmat(int sys, const Env& e, double x, zc* a) {
  double ro; zc el[7];
  evalSpline(*e.s, x, e.nl, ro, el);
  zc zom = Z(e.omre, e.omim);
  double dll1 = e.dll1;
  zc zomro = zom * zom * ro;
  int nv = nvarOf(sys);
#define A(i, j) a[((i)-1) + nv * ((j)-1)]
  switch (sys) {
    case SYS_MINORS: {   // minorsOdeSystem.f90:77-126
      double rr = 1.0 / x, rr2 = rr * rr;
      zc zrpc = 1.0 / el[1];
      zc z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
      zc z2 = (2.0 * el[2]) * zrpc;
      zc z3 = (4.0 * z1) * rr2;
      A(1, 1) = Z(-2.0 * rr);
      A(1, 2) = ((-2.0 * dll1) * z1) * rr2;
      A(1, 3) = Z(dll1 * rr);
      A(1, 4) = (((-dll1) * el[2]) * zrpc) * rr;
      A(1, 5) = Z(0.0);
      A(2, 1) = Z(0.0);
      A(2, 2) = (1.0 - z2) * rr;
      A(2, 3) = 1.0 / el[3];
      A(2, 4) = zrpc;
      A(2, 5) = Z(0.0);
      A(3, 1) = (-z2) * rr;
      A(3, 2) = (-zomro) + ((dll1 * (z1 + el[4])) - 2.0 * el[4]) * rr2;
      A(3, 3) = (-(3.0 + z2)) * rr;
      A(3, 4) = Z(0.0);
      A(3, 5) = A(2, 4);
      A(4, 1) = -A(1, 1);
      A(4, 2) = (-zomro) + z3;
      A(4, 3) = Z(0.0);
      A(4, 4) = -A(2, 2);
      A(4, 5) = A(2, 3);
      A(5, 1) = z3;
      A(5, 2) = Z(0.0);
      A(5, 3) = A(4, 2);
      A(5, 4) = A(3, 2);
      A(5, 5) = (z2 - 5.0) * rr;
      break;
    }
    case SYS_FLUID: {    // fluidOdeSystem.f90:78-95
      A(1, 1) = Z(-2.0 / x);
      A(1, 2) = 1.0 / el[1] - dll1 / ((zomro * x) * x);
      A(2, 1) = -zomro;
      A(2, 2) = Z(0.0);
      break;
    }
    case SYS_RADIAL: {   // radialOdeSystem.f90:78-99
      double rr = 1.0 / x, rr2 = rr * rr;
      A(1, 1) = ((-2.0 * el[2]) * rr) / el[1];
      A(1, 2) = 1.0 / el[1];
      A(2, 1) = (-zomro) + (4.0 * rr2) * ((el[0] - (el[2] * el[2]) / el[1]) - el[4]);
      A(2, 2) = (2.0 * rr) * (el[2] / el[1] - 1.0);
      break;
    }
    case SYS_TOROIDAL: { // toroidalOdeSystem.f90:81-102
      double rr = 1.0 / x, rr2 = rr * rr;
      A(1, 1) = Z(rr);
      A(1, 2) = 1.0 / el[3];
      A(2, 1) = (-zomro) - (el[4] * rr2) * (2.0 - dll1);
      A(2, 2) = Z(-3.0 * rr);
      break;
    }
    case SYS_SOLIDT: {   // solidtOdeSystem.f90:77-114
      double rr = 1.0 / x, rr2 = rr * rr;
      zc zrpc = 1.0 / el[1];
      zc z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
      zc z2 = (el[2] * rr) * zrpc;
      zc zdlz1 = dll1 * z1;
      A(1, 1) = 2.0 * z2;
      A(2, 1) = -zrpc;
      A(3, 1) = (-dll1) * z2;
      A(4, 1) = Z(0.0);
      A(1, 2) = zomro - (4.0 * z1) * rr2;
      A(2, 2) = (-A(1, 1)) + 2.0 * rr;
      A(3, 2) = (2.0 * rr2) * zdlz1;
      A(4, 2) = Z((-dll1) * rr);
      A(1, 3) = Z(rr);
      A(2, 3) = Z(0.0);
      A(3, 3) = -A(1, 3);
      A(4, 3) = -(1.0 / el[3]);
      A(1, 4) = (2.0 * z1) * rr2;
      A(2, 4) = z2;
      A(3, 4) = zomro - (zdlz1 + (dll1 - 2.0) * el[4]) * rr2;
      A(4, 4) = Z(3.0 * rr);
      break;
    }
  }
#undef A
}

// flop weights of one system-matrix evaluation (incl. spline interpolation)
// and of one midpoint matrix-vector update; shared with the GPU counters.
static const int FLOP_SYSMAT[5] = {230, 150, 175, 140, 215};
static const int FLOP_MV[5] = {8 * 19 + 4 * 5, 8 * 3 + 4 * 2, 8 * 4 + 4 * 2, 8 * 4 + 4 * 2, 8 * 14 + 4 * 4};

// y = A z  (gfortran matmul order: sum over columns j = 1..n)
static inline void matvec(int nv, const zc* a, const zc* z, zc* y) {
  for (int i = 0; i < nv; ++i) y[i] = Z(0.0);
  for (int j = 0; j < nv; ++j)
    for (int i = 0; i < nv; ++i) y[i] = y[i] + a[i + nv * j] * z[j];
}

// ===========================================================================
//  Bulirsch-Stoer engine (complexBulirschStep.f90)
// ===========================================================================
struct BSEngine {
  int sys, nv;
  const Env* env;
  double eps;
  int donetry;
  bool success;
  zc ysol[7][5];
  zc yext[5];
  zc sm[49][25];
  Stats* st;

  void linearMidpoint(int jtry /*1-based*/, double h, double xstart, const zc* y0) {
    for (int j = 0; j < NXDIV_BS[jtry - 1]; ++j) {
      int ix = IXDIV_BS[jtry - 1][j];
      double x = xstart + ((double)ix * h) / (double)KGV_BS;
      sysmat(sys, *env, x, sm[ix]);
      st->sysmats++; st->flops += FLOP_SYSMAT[sys];
    }
    int nstep = SEQDIV_BS[jtry - 1];
    double hdiv = h / (double)nstep;
    zc z0[5], z1[5], z2[5], t[5];
    for (int i = 0; i < nv; ++i) z0[i] = y0[i];
    matvec(nv, sm[0], z0, t);
    for (int i = 0; i < nv; ++i) z1[i] = z0[i] + hdiv * t[i];   // + hdiv*rhs (rhs = 0)
    for (int m = 1; m <= nstep - 1; ++m) {
      int ix = m * KGV_BS / nstep;
      matvec(nv, sm[ix], z1, t);
      for (int i = 0; i < nv; ++i) z2[i] = z0[i] + (2.0 * hdiv) * t[i];
      for (int i = 0; i < nv; ++i) { z0[i] = z1[i]; z1[i] = z2[i]; }
    }
    matvec(nv, sm[KGV_BS], z1, t);
    for (int i = 0; i < nv; ++i) ysol[jtry - 1][i] = 0.5 * ((z1[i] + z0[i]) + hdiv * t[i]);
    st->matvecs += nstep + 1; st->attempts++;
    st->flops += (int64_t)(nstep + 1) * FLOP_MV[sys];
    donetry = jtry;
  }

  // Neville extrapolation to h = 0 (complexBulirschStep.f90:297-340)
  void extrapolate(double hs, zc* yy, zc* dy) {
    int n = donetry;
    double x[7];
    zc c[7][5], d[7][5], u[5];
    for (int i = 0; i < n; ++i) x[i] = hs / (double)SEQDIV_BS[i];
    int js = n;
    for (int j = 0; j < n; ++j) for (int v = 0; v < nv; ++v) { c[j][v] = ysol[j][v]; d[j][v] = ysol[j][v]; }
    for (int v = 0; v < nv; ++v) yy[v] = ysol[js - 1][v];
    for (int m = 1; m <= n - 1; ++m) {
      for (int i = 1; i <= n - m; ++i) {
        double hh = x[i - 1] - x[i + m - 1];
        for (int v = 0; v < nv; ++v) {
          u[v] = (c[i][v] - d[i - 1][v]) / hh;
          c[i - 1][v] = x[i - 1] * u[v];
          d[i - 1][v] = x[i + m - 1] * u[v];
        }
      }
      for (int v = 0; v < nv; ++v) { yy[v] = yy[v] + d[js - 2][v]; dy[v] = d[js - 2][v]; }
      js = js - 1;
    }
    st->flops += (int64_t)(n * (n - 1) / 2) * 8 * nv + (int64_t)(n - 1) * 2 * nv;
  }

  void fullStep(double h, double xstart, const zc* y0) {
    success = false;
    donetry = 0;
    int ntry = MINTRY_BS, nfirst = 1;
    zc zyy[5], zdy[5];
    for (;;) {
      for (int j = nfirst; j <= ntry; ++j) linearMidpoint(j, h, xstart, y0);
      extrapolate(h, zyy, zdy);
      double s1 = 0.0, s2 = 0.0;
      for (int v = 0; v < nv; ++v) { double a = zabs(zdy[v]); s1 += a * a; }
      for (int v = 0; v < nv; ++v) { double a = zabs(zyy[v]); s2 += a * a; }
      double errmax = std::sqrt(s1 / s2);
      st->flops += 8 * nv + 3;
      if (getenv("ORACLE_DEBUG2")) fprintf(stderr, "  bs sys %d x %.3f h %.6g ntry %d err %.3e yy0 (%.3e,%.3e) y0 (%.3e %.3e) y1 (%.3e %.3e)\n", sys, xstart, h, ntry, errmax, zyy[0].re, zyy[0].im, y0[0].re, y0[0].im, y0[1].re, y0[1].im);
      if (errmax / eps < 1.0) {
        for (int v = 0; v < nv; ++v) yext[v] = zyy[v];
        success = true;
        return;
      }
      if (ntry < MAXTRY_BS) { ntry++; nfirst = ntry; continue; }
      success = false;
      return;
    }
  }

  void adjust(double& h, bool ok) {
    if (ok) {
      if (donetry > OPTTRY_BS) h = h * SHRINK_BS;
      else if (donetry < OPTTRY_BS) h = h * GROW_BS;
    } else {
      h = 0.5 * h / 1.0;   // 2**((maxtry-opttry)/2) = 2**0 = 1
    }
  }
};

// ===========================================================================
//  Integration over one sub-interval (integrationStep.f90:98-190)
// ===========================================================================
// returns 0 ok, 1 step below minimum, 2 maximum number of steps
static int integrationStep(BSEngine& eng, double& hdid, double x1, double x2, zc* y) {
  if (std::fabs(x2 - x1) < MINSIZE_IS) return 0;
  double x = x1;
  double h = std::copysign(hdid, x2 - x1);
  zc ys[5];
  for (int v = 0; v < eng.nv; ++v) ys[v] = y[v];
  int nstep = 0;
  while (nstep < MAXNUM_IS) {
    if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
    eng.fullStep(h, x, ys);
    nstep++;
    if (eng.success) {
      eng.st->steps_ok++;
      x = x + h;
      for (int v = 0; v < eng.nv; ++v) ys[v] = eng.yext[v];
      if (std::fabs(x - x2) < MINSIZE_IS) {
        for (int v = 0; v < eng.nv; ++v) y[v] = ys[v];
        return 0;
      }
      eng.adjust(h, true);
      hdid = h;
    } else {
      eng.st->steps_rej++;
      eng.adjust(h, false);
      if (std::fabs(h) < MINSIZE_IS) {
        if (getenv("ORACLE_DEBUG")) {
          fprintf(stderr, "minsize: sys %d x1 %.6f x2 %.6f x %.6f nl %d dll1 %g om %g y0 (%g,%g)\n", eng.sys, x1, x2, x,
                  eng.env->nl, eng.env->dll1, eng.env->omre, ys[0].re, ys[0].im);
        }
        return 1;
      }
    }
  }
  return 2;
}

// ===========================================================================
//  Propagator (propagateOde.f90:132-331)
// ===========================================================================
struct Prop {
  int sys, nv;
  Env* env;
  double eps;
  bool do_norm;
  double lgnorm;
  zc y[5];
  int jl, jr;
  std::vector<zc> yn;        // [node_k * 5 + v], in integration order
  std::vector<double> lgyn;  // per stored node
  Stats* st;
};

// status: 0 ok, 4 node/disco bookkeeping error, 1/2 integrator errors
static int propagate(Prop& p, double x1, double x2, double htry, const zc* ystart) {
  for (int v = 0; v < p.nv; ++v) p.y[v] = ystart[v];
  p.yn.clear(); p.lgyn.clear();
  std::vector<double> xn, xd;
  int jl, jr;
  getNodes(*p.env, x1, x2, jl, jr, xn);
  p.jl = jl; p.jr = jr;
  int nnod = (int)xn.size();
  getDiscos(*p.env, x1, x2, jl, jr, xd);
  int nd = (int)xd.size();
  p.yn.assign((size_t)nnod * 5, Z(0.0)); p.lgyn.assign(nnod, 0.0);
  int idir = (int)std::copysign(1.0, x2 - x1);
  if (nd > 0) {
    if ((x1 - xd[0]) * idir > 0 || (xd[nd - 1] - x2) * idir > 0) return 4;
  }
  if (nnod > 0) {
    if ((x1 - xn[0]) * idir > 0 || (xn[nnod - 1] - x2) * idir > 0) return 4;
  }
  int jnod, jd;
  if (std::fabs(x2 - x1) < MINSIZE_IS && nnod == 0) return 0;
  else if (std::fabs(x2 - x1) < MINSIZE_IS && nnod > 1) return 4;
  else if (std::fabs(x2 - x1) < MINSIZE_IS && nnod == 1) {
    for (int v = 0; v < p.nv; ++v) p.yn[v] = p.y[v];
    jnod = 2; jd = 1;
  } else {
    BSEngine eng;
    eng.sys = p.sys; eng.nv = p.nv; eng.env = p.env; eng.eps = p.eps; eng.st = p.st;
    double hdid = htry;
    jd = 1; jnod = 1;
    double xa = x1;
    while (std::fabs(x2 - xa) > MINSIZE_IS) {
      double steps[3];
      steps[2] = std::fabs(x2 - xa);
      steps[0] = 2.0 * std::fabs(x2 - x1);
      steps[1] = 3.0 * std::fabs(x2 - x1);
      if (jnod <= nnod) steps[0] = std::fabs(xn[jnod - 1] - xa);
      if (jd <= nd) steps[1] = std::fabs(xd[jd - 1] - xa);
      int kmin = 0;
      for (int k = 1; k < 3; ++k) if (steps[k] < steps[kmin]) kmin = k;
      double xe = xa + idir * steps[kmin];
      int rc = integrationStep(eng, hdid, xa, xe, p.y);
      if (rc) return rc;
      if (p.do_norm) {
        double s = 0.0;
        for (int v = 0; v < p.nv; ++v) s += std::fabs(p.y[v].re) + std::fabs(p.y[v].im);
        double ynorm = s / p.nv;
        if (ynorm > MAXY_PROP) {
          for (int v = 0; v < p.nv; ++v) { p.y[v].re = p.y[v].re / ynorm; p.y[v].im = p.y[v].im / ynorm; }
          p.lgnorm = p.lgnorm + std::log10(ynorm);
        }
      }
      if (kmin == 0) {
        for (int v = 0; v < p.nv; ++v) p.yn[(jnod - 1) * 5 + v] = p.y[v];
        p.lgyn[jnod - 1] = p.lgnorm;
        jnod++;
        if (std::fabs(steps[0] - steps[1]) < MINSIZE_IS) { p.env->nl += idir; jd++; }
      } else if (kmin == 1) {
        jd++;
        p.env->nl += idir;
        if (std::fabs(steps[0] - steps[1]) < MINSIZE_IS) {
          for (int v = 0; v < p.nv; ++v) p.yn[(jnod - 1) * 5 + v] = p.y[v];
          p.lgyn[jnod - 1] = p.lgnorm;
          jnod++;
        }
      }
      xa = xe;
    }
  }
  if (jnod - 1 != nnod) return 4;
  if (jd - 1 != nd) return 4;
  return 0;
}

// ===========================================================================
//  Start radius and initial values (initialValues.f90)
// ===========================================================================
static double vslow(double om, double dll1, double r, double v) {
  return dll1 / (r * r) - (om / v) * (om / v);
}

static double velocityAt(const Env& e, double r, int nl) {
  double ro; zc el[7];
  evalSpline(*e.s, r, nl, ro, el);
  double v = std::sqrt(el[6].re / ro);
  if (e.m->iflso[nl] == 1) v = std::sqrt(el[5].re / ro);
  return v;
}

static double integrateSlowness(const Env& e, double rturn, double dr, double eps, bool tor) {
  const Model& m = *e.m;
  double q = 0.0, r = rturn;
  double rbot = (tor && hasCore(m)) ? m.roc : m.rb[1] - (double)0.1f * dr;
  double qmax = -std::log(eps);
  while (q < qmax) {
    if (r - dr < rbot) { r = rbot; break; }
    r = r - dr;
    int nl, top;
    layerIndex(m, r, nl, top);
    double v = velocityAt(e, r, nl);
    q = q + dr * std::sqrt(vslow(e.omre, e.dll1, r, v));
  }
  return r;
}

// initialValues.f90:71-149
static double startRadius(const Env& e, bool tor) {
  const Model& m = *e.m;
  double dll1 = e.dll1, om = e.omre, rearth = m.rearth, rhs = m.rb[1], roc = m.roc;
  double eps = 1.e-5;
  double r; int nl;
  if (tor && hasCore(m)) { r = roc; nl = m.noc + 1; } else { r = rhs; nl = 1; }
  double dr = (rearth - r) / 400.0;
  double v = velocityAt(e, r, nl);
  double p = vslow(om, dll1, r, v), pold = p;
  if (p <= 0.0) {
    if (tor && hasCore(m)) return roc;
    return rhs - (double)0.1f * dr;
  }
  double rmax = (tor && hasOcean(m)) ? ruc(m) : rearth;
  while (p > 0.0) {
    pold = p;
    if (std::fabs(1.0 - r / rmax) < EPS_D) {
      return integrateSlowness(e, rmax, dr, eps, tor);   // no turning point at all
    }
    r = std::min(r + dr, rmax);
    int top;
    layerIndex(m, r, nl, top);
    v = velocityAt(e, r, nl);
    p = vslow(om, dll1, r, v);
  }
  double rturn = r - dr * p / (p - pold);
  return integrateSlowness(e, rturn, dr, eps, tor);
}

// sphancfInitialValues :487-526 (kindhf 1 or 2); returns 3 on non-convergence
static int sphancf(zc zx, double el, int kindhf, zc& zf) {
  const double tiny = 1.e-30, eps = 1.e-6;
  const zc ci = Z(0.0, 1.0);
  zf = Z(tiny);
  zc zc_ = zf, zd = Z(0.0);
  double elph2 = (el + 0.5) * (el + 0.5);
  int j;
  for (j = 1; j <= 10000; ++j) {
    zc zb = 2.0 * (zx + Z(0.0, (double)j));
    double za = ((double)j - 0.5) * ((double)j - 0.5) - elph2;
    zd = zb + za * zd;
    if (zabs(zd) < tiny) zd = Z(tiny);
    zc_ = zb + za / zc_;
    if (zabs(zc_) < tiny) zc_ = Z(tiny);
    zd = 1.0 / zd;
    zc zdelta = zc_ * zd;
    zf = zf * zdelta;
    if (zabs(zdelta - 1.0) < eps) break;
  }
  if (j > 10000) return 3;
  if (kindhf == 1) zf = ((el + 1.0) - ci * zx) - ci * zf;
  else zf = ((el + 1.0) + ci * zx) + ci * zf;
  return 0;
}

// zetlInitialValues :544-574
static int zetl(zc zx2, double el, zc& z) {
  const double tiny = 1.e-30, eps = 1.e-6;
  z = Z(tiny);
  zc zd = Z(2.0 * el + 3.0);
  zc zc_ = zd + zx2 / z;
  zd = 1.0 / zd;
  zc zdelta = zc_ * zd;
  z = z * zdelta;
  for (int i = 2; i <= 10000; ++i) {
    zd = ((2.0 * (el + (double)i) + 1.0) - zx2 * zd);
    if (zd.re == 0.0 && zd.im == 0.0) zd = Z(tiny);
    zc_ = ((2.0 * (el + (double)i) + 1.0) - zx2 / zc_);
    if (zc_.re == 0.0 && zc_.im == 0.0) zc_ = Z(tiny);
    zd = 1.0 / zd;
    zdelta = zc_ * zd;
    z = z * zdelta;
    if (std::fabs(zabs(zdelta) - 1.0) < eps) return 0;
  }
  return 3;
}

// minorsBottomInitialValues :202-275
static int minorsBottomIV(const Env& e, double rstart, zc* ys, double& htry) {
  const Model& m = *e.m;
  int nl = e.nl;
  double ro; zc el7[7];
  evalSpline(*e.s, rstart, nl, ro, el7);
  bool liquid = m.iflso[nl] == 1;
  double el = -0.5 + std::sqrt(0.25 + e.dll1);
  double elp1 = e.dll1;
  zc zom = Z(e.omre, e.omim);
  double rsq = rstart * rstart;
  double v = std::sqrt(el7[6].re / ro);
  if (liquid) v = std::sqrt(el7[5].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  zc zxa2 = (((ro * zom) * zom) * rsq) / (el7[5] + (4.0 * el7[6]) / 3.0);
  zc zeta = Z(0.0), zetb = Z(0.0), zxb2 = Z(0.0);
  int rc = 0;
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
  if (el < EPS_D) {
    ys[0] = -zeta;
    ys[1] = (((-ro) * rstart) * zom) * zom + ((4.0 * el7[6]) / rstart) * zeta;
  } else {
    if (liquid) {
      ys[0] = (-(1.0 - zeta / el)) / (((zom * zom) * ro) * rstart);
      ys[1] = Z(1.0 / el);
    } else {
      zc za = zeta / el;
      zc zb = zetb / (el + 1.0);
      ys[1] = ((-za) + zb * (za - 1.0)) / el;
      ys[0] = (el7[6] / rstart) * (zxb2 / el + (2.0 * elp1) * ys[1]);
      ys[2] = (el7[6] / rstart) * ((-2.0) * ys[1] + (zxb2 / elp1) * (za - 1.0));
      ys[3] = (-(el7[6] / rstart)) * ((zxb2 / (el * el)) * (1.0 - zb) + 4.0 * ys[1]);
      ys[4] = ((el7[6] * el7[6]) / rsq) *
              ((((-4.0) * (el - 1.0)) * (el + 2.0)) * ys[1] +
               (zxb2 / el) * ((((zxb2 / elp1) - ((2.0 * (el - 1.0)) * (2.0 * el + 1.0)) / elp1) -
                               (4.0 / (el + 1.0)) * za) - (2.0 / el) * zb));
    }
  }
  return 0;
}

// minorsSurfaceInitialValues :287-367
static int minorsSurfaceIV(const Env& e, zc* ys, double& htry) {
  const Model& m = *e.m;
  int nlay = m.nlay;
  double elp1 = e.dll1;
  double el = -0.5 + std::sqrt(0.25 + elp1);
  double rearth = m.rearth;
  zc zom = Z(e.omre, e.omim);
  bool liquid = m.iflso[nlay] == 1;
  double ro; zc el7[7];
  evalSpline(*e.s, rearth, nlay, ro, el7);
  double v = std::sqrt(el7[6].re / ro);
  if (liquid) v = std::sqrt(el7[5].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (m.fsflag == 1) {
    double rsq = rearth * rearth;
    zc zxa2 = (((ro * zom) * zom) * rsq) / (el7[5] + (4.0 * el7[6]) / 3.0);
    zc zeta, zetb = Z(0.0), zxb2 = Z(0.0);
    int rc = sphancf(zsqrt(zxa2), el, 2, zeta); if (rc) return rc;
    if (!liquid) {
      zxb2 = (((ro * zom) * zom) * rsq) / el7[6];
      rc = sphancf(zsqrt(zxb2), el, 2, zetb); if (rc) return rc;
    }
    if (el < EPS_D) {
      ys[0] = -zeta;
      ys[1] = (((-ro) * rearth) * zom) * zom + ((4.0 * el7[6]) / rearth) * zeta;
    } else if (liquid) {
      ys[0] = (-(1.0 - zeta / el)) / (((zom * zom) * ro) * rearth);
      ys[1] = Z(1.0 / el);
    } else {
      zc za = zeta / el;
      zc zb = zetb / (el + 1.0);
      ys[1] = ((-za) + zb * (za - 1.0)) / el;
      ys[0] = (el7[6] / rearth) * (zxb2 / el + (2.0 * elp1) * ys[1]);
      ys[2] = (el7[6] / rearth) * ((-2.0) * ys[1] + (zxb2 / elp1) * (za - 1.0));
      ys[3] = (-(el7[6] / rearth)) * ((zxb2 / (el * el)) * (1.0 - zb) + 4.0 * ys[1]);
      ys[4] = ((el7[6] * el7[6]) / rsq) *
              ((((-4.0) * (el - 1.0)) * (el + 2.0)) * ys[1] +
               (zxb2 / el) * ((((zxb2 / elp1) - ((2.0 * (el - 1.0)) * (2.0 * el + 1.0)) / elp1) -
                               (4.0 / (el + 1.0)) * za) - (2.0 / el) * zb));
    }
  } else {
    if (el < EPS_F) { ys[0] = Z(1.0); ys[1] = Z(0.0); }
    else if (liquid) { ys[0] = Z(1.0); ys[1] = Z(0.0); }
    else { ys[0] = Z(0.0); ys[1] = Z(1.0); ys[2] = Z(0.0); ys[3] = Z(0.0); ys[4] = Z(0.0); }
  }
  return 0;
}

// toroidalBottomInitialValues :376-418
static int toroidalBottomIV(const Env& e, double rstart, zc* ys, double& htry) {
  const Model& m = *e.m;
  double ro; zc el7[7];
  evalSpline(*e.s, rstart, e.nl, ro, el7);
  double el = -0.5 + std::sqrt(0.25 + e.dll1);
  double elp1 = e.dll1;
  zc zom = Z(e.omre, e.omim);
  double rsq = rstart * rstart;
  double v = std::sqrt(el7[6].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (rstart > m.roc) {
    zc zxb2 = (((ro * zom) * zom) * rsq) / el7[6], zetb;
    int rc;
    if (zabs(zxb2 / elp1) < 1.0) rc = zetl(zxb2, el, zetb);
    else rc = sphancf(zsqrt(zxb2), el, 1, zetb);
    if (rc) return rc;
    ys[0] = Z(1.0 / el);
    ys[1] = (el7[6] / (rstart * el)) * ((el - 1.0) - zetb);
  } else {
    ys[0] = Z(1.0 / el);
    ys[1] = Z(0.0);
  }
  return 0;
}

// toroidalSurfaceInitialValues :434-469
static int toroidalSurfaceIV(const Env& e, zc* ys, double& htry, double& rsurf, int& nl) {
  const Model& m = *e.m;
  int nlay = m.nlay;
  if (hasOcean(m)) { nl = nlay - 1; rsurf = ruc(m); } else { nl = nlay; rsurf = m.rearth; }
  double el = -0.5 + std::sqrt(0.25 + e.dll1);
  zc zom = Z(e.omre, e.omim);
  double ro; zc el7[7];
  evalSpline(*e.s, rsurf, nl, ro, el7);
  double v = std::sqrt(el7[6].re / ro);
  htry = ((0.25 * v) * TWO_PI_F) / e.omre;
  if (m.fsflag == 1) {
    double rsq = rsurf * rsurf;
    zc zxb2 = (((ro * zom) * zom) * rsq) / el7[6], zetb;
    int rc = sphancf(zsqrt(zxb2), el, 2, zetb); if (rc) return rc;
    ys[0] = Z(1.0 / el);
    ys[1] = (el7[6] / (rsurf * el)) * ((el - 1.0) - zetb);
  } else {
    ys[0] = Z(1.0); ys[1] = Z(0.0);
  }
  return 0;
}

// ===========================================================================
//  Toroidal minors (toroidalMinors.f90:71-268)
// ===========================================================================
struct TorMin {
  std::vector<zc> u, d;      // [n*2 + c], 1-based n
  std::vector<zc> det;       // 1-based
  bool done = false;
};

static int computeToroidalMinors(TorMin& T, int jsl, int jsr, const Env& gem, double eps, Stats& st) {
  const Nodes& ex = *gem.ex;
  int nnod = ex.nnod;
  if (jsl < 1 || jsl > nnod || jsr < 1 || jsr > nnod) return 4;
  double rstart = startRadius(gem, true);
  Env env = gem;
  T.done = false;
  T.u.assign((nnod + 1) * 2, Z(0.0)); T.d.assign((nnod + 1) * 2, Z(0.0));
  T.det.assign(nnod + 1, Z(0.0));
  if (gem.dll1 < EPS_D) { T.done = true; return 0; }
  double rsl = ex.r[jsl];
  double rmin = std::max(rstart, rsl);
  double rmax = ex.r[jsr];
  if (rstart >= rmax) { T.done = true; return 0; }
  Prop prop; prop.sys = SYS_TOROIDAL; prop.nv = 2; prop.env = &env; prop.eps = eps;
  prop.do_norm = false; prop.lgnorm = 0.0; prop.st = &st;
  zc ys[5]; double htry, rsurf; int nl;
  int rc = toroidalSurfaceIV(env, ys, htry, rsurf, nl); if (rc) return rc;
  if (rsurf < rmin) { T.done = true; return 0; }
  env.nl = nl;
  rc = propagate(prop, rsurf, rmin, htry, ys); if (rc) return rc;
  int jld = prop.jl, jrd = prop.jr;
  if (jrd - jld < 0) return 4;
  for (int k = 0; k <= jrd - jld; ++k)   // descending order in zyn
    for (int c = 0; c < 2; ++c) T.d[(jrd - k) * 2 + c] = prop.yn[k * 5 + c];
  rmax = std::min(rmax, rsurf);
  int top;
  layerIndex(*env.m, rstart, nl, top);
  if (top == 1) nl = nl + 1;
  env.nl = nl;
  rc = toroidalBottomIV(env, rstart, ys, htry); if (rc) return rc;
  rc = propagate(prop, rstart, rmax, htry, ys); if (rc) return rc;
  int jlu = prop.jl, jru = prop.jr;
  if (jru - jlu < 0) return 4;
  for (int k = 0; k <= jru - jlu; ++k)
    for (int c = 0; c < 2; ++c) T.u[(jlu + k) * 2 + c] = prop.yn[k * 5 + c];
  for (int js = jsl; js <= jsr; ++js)
    T.det[js] = T.u[js * 2 + 0] * T.d[js * 2 + 1] - T.d[js * 2 + 0] * T.u[js * 2 + 1];
  T.done = true;
  return 0;
}

// ===========================================================================
//  Spheroidal minors (spheroidalMinors.f90:72-585)
// ===========================================================================
struct SphMin {
  std::vector<zc> u, d;              // minors [n*6 + c]
  std::vector<zc> umtil, dmtil, umeps, dmeps;   // [n*16 + i*4 + j], 0-based i,j
  std::vector<double> ulg, dlg;
  std::vector<zc> det;
  bool done = false;
};

static void fillMtil(SphMin& S, bool up, int n) {
  static const int idx[4][4] = {{0, 1, 2, 3}, {0, 0, 4, 5}, {0, 0, 0, 6}, {0, 0, 0, 0}};
  std::vector<zc>& mi = up ? S.u : S.d;
  std::vector<zc>& mt = up ? S.umtil : S.dmtil;
  std::vector<zc>& me = up ? S.umeps : S.dmeps;
  for (int i = 1; i <= 4; ++i)
    for (int j = i + 1; j <= 4; ++j) {
      double vf = -1.0 + 2.0 * (double)((i + j) % 2);
      int id = idx[i - 1][j - 1];
      mt[n * 16 + (i - 1) * 4 + (j - 1)] = mi[n * 6 + id - 1];
      mt[n * 16 + (j - 1) * 4 + (i - 1)] = -mt[n * 16 + (i - 1) * 4 + (j - 1)];
      me[n * 16 + (i - 1) * 4 + (j - 1)] = vf * mi[n * 6 + (7 - id) - 1];
      me[n * 16 + (j - 1) * 4 + (i - 1)] = -me[n * 16 + (i - 1) * 4 + (j - 1)];
    }
}

static int computeSpheroidalMinors(SphMin& S, int jsl, int jsr, const Env& gem, double eps, Stats& st) {
  const Nodes& ex = *gem.ex;
  const Model& m = *gem.m;
  int nnod = ex.nnod;
  if (jsl < 1 || jsl > nnod || jsr < 1 || jsr > nnod) return 4;
  Env env = gem;
  S.done = false;
  S.u.assign((nnod + 1) * 6, Z(0.0)); S.d.assign((nnod + 1) * 6, Z(0.0));
  S.umtil.assign((nnod + 1) * 16, Z(0.0)); S.dmtil = S.umtil; S.umeps = S.umtil; S.dmeps = S.umtil;
  S.ulg.assign(nnod + 1, 0.0); S.dlg.assign(nnod + 1, 0.0);
  S.det.assign(nnod + 1, Z(0.0));
  double rstart = startRadius(gem, false);
  double rsl = ex.r[jsl];
  double rmin = std::max(rstart, rsl);
  double rmax = ex.r[jsr];
  if (rstart >= rmax) { S.done = true; return 0; }
  double rearth = m.rearth;
  bool l0 = gem.dll1 < EPS_D;
  // ---------------- upward
  double rend = rstart, rbeg = rstart, lgnorm = 0.0, lgnormend = 0.0;
  bool liq_old = false;
  zc yend[5]; int nvold = 0;
  double htry = 0.0;   // keeps its value across phase changes (spheroidalMinors.f90:267-274)
  while (rend < rmax) {
    int nl, top;
    layerIndex(m, rbeg, nl, top);
    if (top == 1) nl = nl + 1;
    bool liq = m.iflso[nl] == 1;
    env.nl = nl;
    rend = abovePhaseChange(m, nl);
    rend = std::min(rend, rmax);
    Prop prop; prop.env = &env; prop.eps = eps; prop.do_norm = true; prop.lgnorm = lgnorm; prop.st = &st;
    if (liq) prop.sys = SYS_FLUID; else prop.sys = l0 ? SYS_RADIAL : SYS_MINORS;
    prop.nv = nvarOf(prop.sys);
    zc ys[5] = {Z(0), Z(0), Z(0), Z(0), Z(0)};
    if (rbeg == rstart) {
      int rc = minorsBottomIV(env, rbeg, ys, htry); if (rc) return rc;
    } else {
      if (liq && !liq_old) {
        if (l0) { ys[0] = yend[0]; ys[1] = yend[1]; } else { ys[0] = yend[2]; ys[1] = yend[4]; }
      } else if (!liq && liq_old) {
        if (l0) { ys[0] = yend[0]; ys[1] = yend[1]; }
        else { ys[3] = yend[1]; ys[1] = yend[0]; ys[0] = Z(0.0); ys[2] = Z(0.0); ys[4] = Z(0.0); }
      } else return 4;
    }
    (void)nvold;
    int rc = propagate(prop, rbeg, rend, htry, ys); if (rc) return rc;
    int jlu = prop.jl, jru = prop.jr;
    if (jru - jlu >= 0) {
      for (int k = 0; k <= jru - jlu; ++k) {
        int n = jlu + k;
        S.ulg[n] = prop.lgyn[k];
        for (int c = 0; c < prop.nv; ++c) S.u[n * 6 + c] = prop.yn[k * 5 + c];
        S.u[n * 6 + 5] = (-S.u[n * 6 + 0]) / env.dll1;
      }
      if (!liq && gem.dll1 > EPS_D)
        for (int n = jlu; n <= jru; ++n) fillMtil(S, true, n);
    }
    liq_old = liq;
    rbeg = rend;
    for (int c = 0; c < prop.nv; ++c) yend[c] = prop.y[c];
    nvold = prop.nv;
    lgnormend = prop.lgnorm;
    lgnorm = lgnormend;
  }
  for (int n = 1; n <= nnod; ++n) {
    double lgn = S.ulg[n] - lgnormend;
    double f = std::pow(10.0, lgn);
    for (int c = 0; c < 6; ++c) S.u[n * 6 + c] = S.u[n * 6 + c] * f;
    for (int c = 0; c < 16; ++c) { S.umtil[n * 16 + c] = S.umtil[n * 16 + c] * f; S.umeps[n * 16 + c] = S.umeps[n * 16 + c] * f; }
  }
  // ---------------- downward
  rbeg = rearth; rend = rearth; liq_old = false; lgnorm = 0.0; lgnormend = 0.0;
  while (rend > rmin) {
    int nl, top;
    layerIndex(m, rbeg, nl, top);
    bool liq = m.iflso[nl] == 1;
    env.nl = nl;
    rend = belowPhaseChange(m, nl);
    rend = std::max(rend, rmin);
    Prop prop; prop.env = &env; prop.eps = eps; prop.do_norm = true; prop.lgnorm = lgnorm; prop.st = &st;
    if (liq) prop.sys = SYS_FLUID; else prop.sys = l0 ? SYS_RADIAL : SYS_MINORS;
    prop.nv = nvarOf(prop.sys);
    zc ys[5] = {Z(0), Z(0), Z(0), Z(0), Z(0)};
    if (rbeg == rearth) {
      int rc = minorsSurfaceIV(env, ys, htry); if (rc) return rc;
    } else {
      if (liq && !liq_old) {
        if (l0) { ys[0] = yend[0]; ys[1] = yend[1]; } else { ys[0] = yend[2]; ys[1] = yend[4]; }
      } else if (!liq && liq_old) {
        if (l0) { ys[0] = yend[0]; ys[1] = yend[1]; }
        else { ys[3] = yend[1]; ys[1] = yend[0]; ys[0] = Z(0.0); ys[2] = Z(0.0); ys[4] = Z(0.0); }
      } else return 4;
    }
    int rc = propagate(prop, rbeg, rend, htry, ys); if (rc) return rc;
    int jld = prop.jl, jrd = prop.jr;
    if (jrd - jld < 0) return 4;
    for (int k = 0; k <= jrd - jld; ++k) {
      int n = jrd - k;
      S.dlg[n] = prop.lgyn[k];
      for (int c = 0; c < prop.nv; ++c) S.d[n * 6 + c] = prop.yn[k * 5 + c];
    }
    for (int n = jld; n <= jrd; ++n) S.d[n * 6 + 5] = (-S.d[n * 6 + 0]) / env.dll1;
    if (!liq && gem.dll1 > EPS_D)
      for (int n = jld; n <= jrd; ++n) fillMtil(S, false, n);
    liq_old = liq;
    rbeg = rend;
    for (int c = 0; c < prop.nv; ++c) yend[c] = prop.y[c];
    lgnormend = prop.lgnorm;
    lgnorm = lgnormend;
  }
  for (int n = 1; n <= nnod; ++n) {
    double lgn = S.dlg[n] - lgnormend;
    double f = std::pow(10.0, lgn);
    for (int c = 0; c < 6; ++c) S.d[n * 6 + c] = S.d[n * 6 + c] * f;
    for (int c = 0; c < 16; ++c) { S.dmtil[n * 16 + c] = S.dmtil[n * 16 + c] * f; S.dmeps[n * 16 + c] = S.dmeps[n * 16 + c] * f; }
  }
  for (int j = jsl; j <= jsr; ++j) {
    const zc* u = &S.u[j * 6];
    const zc* d = &S.d[j * 6];
    if (ex.state[j] == 1 || gem.dll1 < EPS_D) S.det[j] = u[0] * d[1] - d[0] * u[1];
    else S.det[j] = ((((u[0] * d[5] + u[5] * d[0]) - u[1] * d[4]) + u[2] * d[3]) + u[3] * d[2]) - u[4] * d[1];
  }
  S.done = true;
  return 0;
}

// ===========================================================================
//  Spheroidal adjoint (spheroidalAdjoint.f90:53-159)
// ===========================================================================
static int computeAdjoint(std::vector<zc>& adj /*[n*4+c]*/, zc* ystart, double ra, double re,
                          const Env& gem, double eps, Stats& st) {
  const Model& m = *gem.m;
  int nnod = gem.ex->nnod;
  Env env = gem;
  adj.assign((nnod + 1) * 4, Z(0.0));
  int nl, top;
  layerIndex(m, ra, nl, top);
  if (top == 1 && ra < re) nl = std::min(nl + 1, m.nlay);
  env.nl = nl;
  // getSVelocity / getPVelocity (splineEarthmodelCoefficients.f90:179-200)
  double ro; zc el7[7];
  evalSpline(*env.s, ra, nl, ro, el7);
  double v = std::sqrt(el7[6].re / ro);
  if (v < EPS_D) v = std::sqrt((el7[5] + (4.0 / 3.0) * el7[6]).re / ro);
  double htry = ((0.25 * v) * TWO_PI_F) / env.omre;
  Prop prop; prop.sys = SYS_SOLIDT; prop.nv = 4; prop.env = &env; prop.eps = eps;
  prop.do_norm = false; prop.lgnorm = 0.0; prop.st = &st;
  int rc = propagate(prop, ra, re, htry, ystart); if (rc) return rc;
  int jl = prop.jl, jr = prop.jr;
  if (jr - jl < 0) return 4;
  if (re > ra) {
    for (int j = jl; j <= jr; ++j) for (int c = 0; c < 4; ++c) adj[j * 4 + c] = prop.yn[(j - jl) * 5 + c];
  } else {
    for (int j = jl; j <= jr; ++j) for (int c = 0; c < 4; ++c) adj[j * 4 + c] = prop.yn[(jr - j) * 5 + c];
  }
  for (int c = 0; c < 4; ++c) ystart[c] = prop.y[c];
  return 0;
}

// 4x4 complex matrix (stored [i*4+j]) times 4-vector, gfortran matmul order
static void mtilTimes(const zc* mt, const zc* a, zc* out) {
  for (int i = 0; i < 4; ++i) out[i] = Z(0.0);
  for (int j = 0; j < 4; ++j) for (int i = 0; i < 4; ++i) out[i] = out[i] + mt[i * 4 + j] * a[j];
}

// ===========================================================================
//  Unit jump Green functions (unitJumpGreenFunctions.f90:62-380)
// ===========================================================================
struct UJGF {
  std::vector<zc> sph;   // [(n*4 + jump)*4 + comp]  (comp, jump, node)
  std::vector<zc> tor;   // [(n*2 + jump)*2 + comp]
  int njs, njt;
};

static int computeUJGF(UJGF& U, const TorMin& T, const SphMin& S, int jn, const Env& gem,
                       double eps, Stats& st) {
  const Nodes& ex = *gem.ex;
  const Model& m = *gem.m;
  int nnod = ex.nnod;
  if (!T.done || !S.done) return 4;
  if (jn < 1 || jn > nnod) return 4;
  double ruc_ = ruc(m), roc = m.roc, ric = m.ric;
  double ujvs[4][4] = {{0}}, ujvt[2][2] = {{0}};   // [comp][jump]
  if (ex.state[jn] == 1) { U.njs = 2; U.njt = 0; ujvs[0][0] = 1; ujvs[1][1] = 1; }
  else {
    U.njs = 4; U.njt = 2;
    for (int k = 0; k < 4; ++k) ujvs[k][k] = 1.0;
    ujvt[0][0] = 1.0; ujvt[1][1] = 1.0;
  }
  U.sph.assign((size_t)(nnod + 1) * 16, Z(0.0));
  U.tor.assign((size_t)(nnod + 1) * 4, Z(0.0));
  auto SPH = [&](int c, int j, int n) -> zc& { return U.sph[((size_t)n * 4 + j) * 4 + c]; };
  auto TOR = [&](int c, int j, int n) -> zc& { return U.tor[((size_t)n * 2 + j) * 2 + c]; };
  // toroidal
  if (zabs(T.det[jn]) > TINY_D) {
    double rstart = startRadius(gem, true);
    for (int j = 0; j < U.njt; ++j) {
      zc d = (ujvt[1][j] * T.d[jn * 2 + 0] - ujvt[0][j] * T.d[jn * 2 + 1]) / T.det[jn];
      for (int n = 1; n <= jn - 1; ++n)
        if (ex.state[n] == 0 && ex.r[n] > rstart)
          for (int c = 0; c < 2; ++c) TOR(c, j, n) = d * T.u[n * 2 + c];
      zc e = (ujvt[1][j] * T.u[jn * 2 + 0] - ujvt[0][j] * T.u[jn * 2 + 1]) / T.det[jn];
      for (int n = jn; n <= nnod; ++n)
        if (ex.state[n] == 0)
          for (int c = 0; c < 2; ++c) TOR(c, j, n) = e * T.d[n * 2 + c];
    }
  }
  // spheroidal
  if (zabs(S.det[jn]) > TINY_D) {
    if (gem.dll1 < EPS_D) {
      for (int j = 0; j < 2; ++j) {
        zc d = (ujvs[1][j] * S.d[jn * 6 + 0] - ujvs[0][j] * S.d[jn * 6 + 1]) / S.det[jn];
        zc e = (ujvs[1][j] * S.u[jn * 6 + 0] - ujvs[0][j] * S.u[jn * 6 + 1]) / S.det[jn];
        for (int n = jn; n <= nnod; ++n) for (int c = 0; c < 2; ++c) SPH(c, j, n) = e * S.d[n * 6 + c];
        for (int n = jn - 1; n >= 1; --n) for (int c = 0; c < 2; ++c) SPH(c, j, n) = d * S.u[n * 6 + c];
      }
      return 0;
    }
    double rstart = startRadius(gem, false);
    std::vector<zc> adjic, adjma, adjp, adjm;
    adjic.assign((nnod + 1) * 4, Z(0.0));
    double ra = ric, re = std::max(rstart, ex.r[1]);
    if (re < ra) {
      zc ys[4] = {Z(0), Z(0), Z(0), Z(1.0)};
      int rc = computeAdjoint(adjic, ys, ra, re, gem, eps, st); if (rc) return rc;
    }
    if (ex.state[jn] == 1 && ex.layer[jn] == m.nlay) {
      // source in the ocean
      ra = ruc_;
      re = std::max(std::max(rstart, roc), ex.r[1]);
      zc adjma_roc[4] = {Z(0), Z(0), Z(0), Z(0)};
      adjma.assign((nnod + 1) * 4, Z(0.0));
      if (re < ra) {
        zc ys[4] = {Z(0), Z(0), Z(0), Z(1.0)};
        int rc = computeAdjoint(adjma, ys, ra, re, gem, eps, st); if (rc) return rc;
        for (int c = 0; c < 4; ++c) adjma_roc[c] = ys[c];
      }
      for (int j = 0; j < U.njs; ++j) {
        zc d = (ujvs[1][j] * S.d[jn * 6 + 0] - ujvs[0][j] * S.d[jn * 6 + 1]) / S.det[jn];
        zc e = (ujvs[1][j] * S.u[jn * 6 + 0] - ujvs[0][j] * S.u[jn * 6 + 1]) / S.det[jn];
        for (int n = jn; n <= nnod; ++n) for (int c = 0; c < 2; ++c) SPH(c, j, n) = e * S.d[n * 6 + c];
        for (int n = jn - 1; n >= 1; --n) {
          if (ex.state[n] == 1 && ex.r[n] >= rstart) {
            if (ex.r[n] > ruc_) { for (int c = 0; c < 2; ++c) SPH(c, j, n) = d * S.u[n * 6 + c]; }
            else if (ex.r[n] < roc) { for (int c = 0; c < 2; ++c) SPH(c, j, n) = (d * adjma_roc[2]) * S.u[n * 6 + c]; }
          } else if (ex.state[n] == 0 && ex.r[n] >= rstart) {
            zc t[4];
            if (ex.r[n] > roc) {
              mtilTimes(&S.umtil[n * 16], &adjma[n * 4], t);
              for (int c = 0; c < 4; ++c) SPH(c, j, n) = d * t[c];
            } else if (ex.r[n] < ric) {
              mtilTimes(&S.umtil[n * 16], &adjic[n * 4], t);
              for (int c = 0; c < 4; ++c) SPH(c, j, n) = (d * adjma_roc[2]) * t[c];
            }
          }
        }
      }
    } else {
      // source in the mantle
      for (int j = 0; j < U.njs; ++j) {
        zc ys[4] = {Z(0), Z(0), Z(0), Z(0)};
        for (int i = 0; i < U.njs; ++i)
          for (int c = 0; c < 4; ++c) ys[c] = ys[c] - (ujvs[i][j] * S.umeps[jn * 16 + c * 4 + i]) / S.det[jn];
        re = ruc_;
        int rc = computeAdjoint(adjp, ys, ex.r[jn], re, gem, eps, st); if (rc) return rc;
        zc adjma_ruc[4];
        for (int c = 0; c < 4; ++c) adjma_ruc[c] = ys[c];
        zc ys2[4] = {Z(0), Z(0), Z(0), Z(0)};
        for (int i = 0; i < U.njs; ++i)
          for (int c = 0; c < 4; ++c) ys2[c] = ys2[c] + (ujvs[i][j] * S.dmeps[jn * 16 + c * 4 + i]) / S.det[jn];
        re = std::max(std::max(rstart, roc), ex.r[1]);
        rc = computeAdjoint(adjm, ys2, ex.r[jn], re, gem, eps, st); if (rc) return rc;
        zc adjma_roc[4];
        for (int c = 0; c < 4; ++c) adjma_roc[c] = ys2[c];
        for (int n = jn; n <= nnod; ++n) {
          if (ex.state[n] == 0 && ex.r[n] < ruc_) {
            zc t[4]; mtilTimes(&S.dmtil[n * 16], &adjp[n * 4], t);
            for (int c = 0; c < 4; ++c) SPH(c, j, n) = t[c];
          } else if (ex.state[n] == 1 && ex.r[n] > ruc_) {
            for (int c = 0; c < 2; ++c) SPH(c, j, n) = adjma_ruc[2] * S.d[n * 6 + c];
          }
        }
        for (int n = jn - 1; n >= 1; --n) {
          if (ex.state[n] == 0 && ex.r[n] >= rstart) {
            zc t[4];
            if (ex.r[n] > roc) {
              mtilTimes(&S.umtil[n * 16], &adjm[n * 4], t);
              for (int c = 0; c < 4; ++c) SPH(c, j, n) = t[c];
            } else if (ex.r[n] < ric) {
              mtilTimes(&S.umtil[n * 16], &adjic[n * 4], t);
              for (int c = 0; c < 4; ++c) SPH(c, j, n) = adjma_roc[2] * t[c];
            }
          } else if (ex.state[n] == 1 && ex.r[n] >= rstart) {
            for (int c = 0; c < 2; ++c) SPH(c, j, n) = adjma_roc[2] * S.u[n * 6 + c];
          }
        }
      }
    }
  }
  return 0;
}

// ===========================================================================
//  Reciprocity and source terms
// ===========================================================================
// spheroidalReciprocity (reciprocity.f90:82-153); bgin/bgout as [comp][jump]
static void sphRecip(double elp1, double re, double r, int stn, int sts, const zc bgin[4][4],
                     zc bgout[4][4]) {
  double rlp1 = 1.0 / elp1, f = (r / re) * (r / re);
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) bgout[i][j] = Z(0.0);
#define BI(i, j) bgin[(i)-1][(j)-1]
#define BO(i, j) bgout[(i)-1][(j)-1]
  if (stn == 1) {
    if (sts == 1) {
      BO(1, 1) = (-f) * BI(2, 2); BO(2, 1) = f * BI(2, 1); BO(1, 2) = f * BI(1, 2); BO(2, 2) = (-f) * BI(1, 1);
    } else {
      BO(1, 1) = (-f) * BI(2, 2); BO(2, 1) = f * BI(2, 1);
      if (elp1 > EPS_D) { BO(3, 1) = ((-f) * BI(2, 4)) * rlp1; BO(4, 1) = (f * BI(2, 3)) * rlp1; }
      BO(1, 2) = f * BI(1, 2); BO(2, 2) = (-f) * BI(1, 1);
      if (elp1 > EPS_D) { BO(3, 2) = (f * BI(1, 4)) * rlp1; BO(4, 2) = ((-f) * BI(1, 3)) * rlp1; }
    }
  } else {
    if (sts == 1) {
      BO(1, 1) = (-f) * BI(2, 2); BO(1, 2) = f * BI(1, 2);
      BO(1, 3) = ((-f) * BI(4, 2)) * elp1; BO(1, 4) = (f * BI(3, 2)) * elp1;
      BO(2, 1) = f * BI(2, 1); BO(2, 2) = (-f) * BI(1, 1);
      BO(2, 3) = (f * BI(4, 1)) * elp1; BO(2, 4) = ((-f) * BI(3, 1)) * elp1;
    } else {
      BO(1, 1) = (-f) * BI(2, 2); BO(2, 1) = f * BI(2, 1);
      BO(3, 1) = ((-f) * BI(2, 4)) * rlp1; BO(4, 1) = (f * BI(2, 3)) * rlp1;
      BO(1, 2) = f * BI(1, 2); BO(2, 2) = (-f) * BI(1, 1);
      BO(3, 2) = (f * BI(1, 4)) * rlp1; BO(4, 2) = ((-f) * BI(1, 3)) * rlp1;
      BO(1, 3) = ((-f) * BI(4, 2)) * elp1; BO(2, 3) = (f * BI(4, 1)) * elp1;
      BO(3, 3) = (-f) * BI(4, 4); BO(4, 3) = f * BI(4, 3);
      BO(1, 4) = (f * BI(3, 2)) * elp1; BO(2, 4) = ((-f) * BI(3, 1)) * elp1;
      BO(3, 4) = f * BI(3, 4); BO(4, 4) = (-f) * BI(3, 3);
    }
  }
#undef BI
#undef BO
}

// oneNodeSourceTerms (sourceTerms.f90:59-118); zsph [comp][jump], ztor [comp][jump]
static void sourceTerms(int istyp, double elp1, double om, double rs, int state, int nl,
                        const Spline& s, zc zsph[4][4], zc ztor[2][2]) {
  double rr2 = 1.0 / (rs * rs), rr3 = rr2 / rs;
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) zsph[i][j] = Z(0.0);
  for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) ztor[i][j] = Z(0.0);
  double ro; zc el[7];
  evalSpline(s, rs, nl, ro, el);
  if (istyp == 1) {
    if (state == 1) {
      zsph[0][0] = rr2 * (1.0 / el[1] - Z((elp1 * rr2) / ((om * om) * ro)));
      zsph[1][0] = Z(rr3 * 2.0);
      zsph[0][1] = Z((((0.5 * elp1) * rr2) * rr2) / ((om * om) * ro));
      zsph[1][1] = Z(-rr3);
    } else {
      zsph[0][0] = rr2 / el[1];
      zsph[1][0] = ((rr3 * 2.0) * el[2]) / el[1];
      zsph[3][0] = ((-rr3) * el[2]) / el[1];
      zsph[1][1] = Z(-rr3);
      zsph[3][1] = Z(0.5 * rr3);
      zsph[2][2] = (0.5 * rr2) / el[3];
      zsph[3][3] = Z(0.25 * rr3);
      ztor[0][0] = (0.5 * rr2) / el[3];
      ztor[1][1] = Z(0.25 * rr3);
    }
  } else {
    if (state == 1) {
      zsph[0][0] = Z(0.0);
      zsph[1][0] = Z(-rr2);
      zsph[0][1] = Z((elp1 * rr3) / ((om * om) * ro));
      zsph[1][1] = Z(0.0);
    } else {
      zsph[1][0] = Z(-rr2);
      zsph[3][1] = Z(0.5 * rr2);
      ztor[1][0] = Z(0.5 * rr2);
    }
  }
}

// ===========================================================================
//  FK driver for one frequency (computeGreenFKSpectraForSynthetics.f90)
// ===========================================================================
struct Ctx {
  Model m;
  Nodes ex;
};

// ===========================================================================
//  Travel-time table by ray tracing (computeTravelTimeTable.f90:178-226): for
//  each turning radius, Delta(r) and T(r) of the ray integrated upward to the
//  top node with the real Bulirsch-Stoer step (episode/realBulirschStep.f90)
//  and the ray system (rayOdeSystem.f90:151-170).
// ===========================================================================
struct RayEnv {
  const Model* m;
  const Nodes* ex;
  const Spline* s;
  int nl;
  int stype;   // 0 P, 1 S
  double p;    // angular slowness r/v at the turning point
};

// getPVelocitySplineEarthmodel / getSVelocitySplineEarthmodel (splineEarthmodelCoefficients.f90:192-210)
static double rayVelocity(const RayEnv& e, int nl, double r) {
  double ro;
  zc z[7];
  evalSpline(*e.s, r, nl, ro, z);
  if (e.stype == 0) return std::sqrt((z[5].re + (4.0 / 3.0) * z[6].re) / ro);
  return std::sqrt(z[6].re / ro);
}

// derivativeRealRayOdeSystem (rayOdeSystem.f90:151-170)
static void rayDerivative(const RayEnv& e, double x, double* dy) {
  const double v = rayVelocity(e, e.nl, x);
  const double t = x / v;
  const double ur2 = t * t;
  const double q = std::sqrt(ur2 - e.p * e.p);
  dy[0] = e.p / (q * x);
  dy[1] = ur2 / (q * x);
}

struct RayEngine {
  const RayEnv* env;
  double eps;
  int donetry;
  bool success;
  double ysol[7][2];
  double yext[2];

  // doNonLinearModifiedMidpointRealBulirsch (realBulirschStep.f90:222-252)
  void midpoint(int jtry, double h, double xstart, const double* y0) {
    const int nstep = SEQDIV_BS[jtry - 1];
    const double hdiv = h / (double)nstep;
    double z0[2], z1[2], z2[2], d[2];
    for (int i = 0; i < 2; ++i) z0[i] = y0[i];
    rayDerivative(*env, xstart, d);
    for (int i = 0; i < 2; ++i) z1[i] = z0[i] + hdiv * d[i];
    for (int m = 1; m <= nstep - 1; ++m) {
      const double x = xstart + (double)m * hdiv;
      rayDerivative(*env, x, d);
      for (int i = 0; i < 2; ++i) z2[i] = z0[i] + (2.0 * hdiv) * d[i];
      for (int i = 0; i < 2; ++i) { z0[i] = z1[i]; z1[i] = z2[i]; }
    }
    rayDerivative(*env, xstart + h, d);
    for (int i = 0; i < 2; ++i) ysol[jtry - 1][i] = 0.5 * ((z1[i] + z0[i]) + hdiv * d[i]);
    donetry = jtry;
  }
  // extrapolateRealBulirsch (:258-290): the whole tableau from the stored solutions
  void extrapolate(double hs, double* yy, double* dy) {
    const int n = donetry;
    double x[7], c[7][2], dd[7][2], u[2];
    for (int j = 0; j < n; ++j) x[j] = hs / (double)SEQDIV_BS[j];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < 2; ++i) { c[j][i] = ysol[j][i]; dd[j][i] = ysol[j][i]; }
    int js = n;
    for (int i = 0; i < 2; ++i) yy[i] = ysol[js - 1][i];
    for (int m = 1; m <= n - 1; ++m) {
      for (int i = 1; i <= n - m; ++i) {
        const double h = x[i - 1] - x[i + m - 1];
        for (int v = 0; v < 2; ++v) {
          u[v] = (c[i][v] - dd[i - 1][v]) / h;
          c[i - 1][v] = x[i - 1] * u[v];
          dd[i - 1][v] = x[i + m - 1] * u[v];
        }
      }
      for (int v = 0; v < 2; ++v) { yy[v] = yy[v] + dd[js - 2][v]; dy[v] = dd[js - 2][v]; }
      js = js - 1;
    }
  }
  // doFullStepRealBulirsch (:130-176)
  void fullStep(double h, double xstart, const double* y) {
    success = false;
    donetry = 0;
    int ntry = MINTRY_BS, nfirst = 1;
    double yy[2], dy[2];
    for (;;) {
      for (int j = nfirst; j <= ntry; ++j) midpoint(j, h, xstart, y);
      extrapolate(h, yy, dy);
      const double errmax = std::sqrt((dy[0] * dy[0] + dy[1] * dy[1]) / (yy[0] * yy[0] + yy[1] * yy[1]));
      if (errmax / eps < 1.0) {
        yext[0] = yy[0]; yext[1] = yy[1];
        success = true;
        return;
      }
      if (ntry < MAXTRY_BS) { ntry = ntry + 1; nfirst = ntry; }
      else return;
    }
  }
  // adjustStepSizeRealBulirsch (:295-307)
  void adjust(double& h, bool ok) {
    if (ok) {
      if (donetry > OPTTRY_BS) h = h * SHRINK_BS;
      else if (donetry < OPTTRY_BS) h = h * GROW_BS;
    } else {
      h = 0.5 * h / 1.0;
    }
  }
};

// integrationStep.f90:98-190 for the ray system
static int rayIntegrationStep(RayEngine& eng, double& hdid, double x1, double x2, double* y) {
  if (std::fabs(x2 - x1) < MINSIZE_IS) return 0;
  double x = x1;
  double h = std::copysign(hdid, x2 - x1);
  double ys[2] = {y[0], y[1]};
  int nstep = 0;
  while (nstep < MAXNUM_IS) {
    if ((x + h - x2) * (x + h - x1) > 0.0) h = x2 - x;
    eng.fullStep(h, x, ys);
    nstep++;
    if (eng.success) {
      x = x + h;
      ys[0] = eng.yext[0]; ys[1] = eng.yext[1];
      if (std::fabs(x - x2) < MINSIZE_IS) { y[0] = ys[0]; y[1] = ys[1]; return 0; }
      eng.adjust(h, true);
      hdid = h;
    } else {
      eng.adjust(h, false);
      if (std::fabs(h) < MINSIZE_IS) return 1;
    }
  }
  return 2;
}

// propagateOde.f90:132-331 for the ray system (no renormalisation); yn[k*2 + v]
// holds the solution at the k-th node of the interval, jl..jr its indices.
static int rayPropagate(RayEnv& env, double eps, double x1, double x2, double htry, const double* ystart,
                        std::vector<double>& yn, int& jlo, int& jro) {
  double y[2] = {ystart[0], ystart[1]};
  std::vector<double> xn, xd;
  int jl, jr;
  Env ge;   // node and discontinuity lists of the gemini environment (same rules, rayIntegrationEnvironment.f90:43-121)
  ge.m = env.m; ge.ex = env.ex; ge.s = env.s; ge.nl = env.nl; ge.omre = ge.omim = ge.dll1 = 0.0;
  getNodes(ge, x1, x2, jl, jr, xn);
  jlo = jl; jro = jr;
  const int nnod = (int)xn.size();
  getDiscos(ge, x1, x2, jl, jr, xd);
  const int nd = (int)xd.size();
  yn.assign((size_t)nnod * 2, 0.0);
  const int idir = (int)std::copysign(1.0, x2 - x1);
  if (nd > 0 && ((x1 - xd[0]) * idir > 0 || (xd[nd - 1] - x2) * idir > 0)) return 4;
  if (nnod > 0 && ((x1 - xn[0]) * idir > 0 || (xn[nnod - 1] - x2) * idir > 0)) return 4;
  int jnod = 1, jd = 1;
  if (std::fabs(x2 - x1) < MINSIZE_IS && nnod == 0) return 0;
  if (std::fabs(x2 - x1) < MINSIZE_IS && nnod > 1) return 4;
  if (std::fabs(x2 - x1) < MINSIZE_IS && nnod == 1) {
    yn[0] = y[0]; yn[1] = y[1];
    jnod = 2;
  } else {
    RayEngine eng;
    eng.env = &env; eng.eps = eps;
    double hdid = htry, xa = x1;
    while (std::fabs(x2 - xa) > MINSIZE_IS) {
      double steps[3];
      steps[2] = std::fabs(x2 - xa);
      steps[0] = 2.0 * std::fabs(x2 - x1);
      steps[1] = 3.0 * std::fabs(x2 - x1);
      if (jnod <= nnod) steps[0] = std::fabs(xn[jnod - 1] - xa);
      if (jd <= nd) steps[1] = std::fabs(xd[jd - 1] - xa);
      int kmin = 0;
      for (int k = 1; k < 3; ++k) if (steps[k] < steps[kmin]) kmin = k;
      const double xe = xa + idir * steps[kmin];
      int rc = rayIntegrationStep(eng, hdid, xa, xe, y);
      if (rc) return rc;
      if (kmin == 0) {
        yn[(jnod - 1) * 2] = y[0]; yn[(jnod - 1) * 2 + 1] = y[1];
        jnod++;
        if (std::fabs(steps[0] - steps[1]) < MINSIZE_IS) { env.nl += idir; jd++; }
      } else if (kmin == 1) {
        jd++;
        env.nl += idir;
        if (std::fabs(steps[0] - steps[1]) < MINSIZE_IS) {
          yn[(jnod - 1) * 2] = y[0]; yn[(jnod - 1) * 2 + 1] = y[1];
          jnod++;
        }
      }
      xa = xe;
    }
  }
  if (jnod - 1 != nnod || jd - 1 != nd) return 4;
  return 0;
}

extern "C" {

typedef struct {
  int64_t steps_ok, steps_rej, attempts, sysmats, matvecs, flops;
} or_stats;

void* oracle_create(const or_model_desc* md, int nblocks, const int* nnodb, const double* drb,
                    double shift, double rearth_nodes) {
  Ctx* c = new Ctx();
  buildModel(md, c->m);
  if (createNodes(c->m, nblocks, nnodb, drb, shift, rearth_nodes, c->ex)) { delete c; return nullptr; }
  return c;
}

// Nodes given explicitly (radii, state, layer; 1-based semantics, arrays 0-based)
void* oracle_create_nodes(const or_model_desc* md, int nnod, const double* r, const int* state,
                          const int* layer) {
  Ctx* c = new Ctx();
  buildModel(md, c->m);
  c->ex.nnod = nnod;
  c->ex.r.assign(nnod + 1, 0.0); c->ex.state.assign(nnod + 1, 0); c->ex.layer.assign(nnod + 1, 0);
  for (int i = 0; i < nnod; ++i) { c->ex.r[i + 1] = r[i]; c->ex.state[i + 1] = state[i]; c->ex.layer[i + 1] = layer[i]; }
  return c;
}

void oracle_destroy(void* h) { delete (Ctx*)h; }

int oracle_nnod(void* h) { return ((Ctx*)h)->ex.nnod; }

void oracle_nodes(void* h, double* r, int* state, int* layer) {
  Ctx* c = (Ctx*)h;
  for (int i = 1; i <= c->ex.nnod; ++i) { r[i - 1] = c->ex.r[i]; state[i - 1] = c->ex.state[i]; layer[i - 1] = c->ex.layer[i]; }
}

// receiver node index (1-based) closest to radius (externalRadialNodes.f90:547-559)
int oracle_node_index(void* h, double rs) {
  Ctx* c = (Ctx*)h;
  int n = c->ex.nnod;
  int jr = locate(rs, n, c->ex.r.data());
  if (jr == 0) jr = 1;
  if (jr < n) if (std::fabs(rs - c->ex.r[jr]) > std::fabs(rs - c->ex.r[jr + 1])) jr = jr + 1;
  return jr;
}

// spline coefficients at frequency f: ro, ro2 [nk], el, el2 [nk*7] interleaved complex
// Travel-time table (computeTravelTimeTable.f90:160-226): turning radii rtp[i] =
// roc + i*drtp for i < ntp = int(rtmax - roc)/drtp + 1, slowness[i] = rtp/v(rtp), and
// table[(i*nnod + j)*2 + {0,1}] = (Delta, T) of that ray at node j (0 where the ray
// does not reach).  stype 0 P, 1 S.  Returns 0, or 2 if ntp > ntp_cap, or the first
// integrator status.
int oracle_ray_table(void* h, int stype, int attmode, double eps, double drtp, double rtmax, int ntp_cap,
                     int* ntp_out, double* rtp_out, double* slowness, float* table, int* status) {
  Ctx* c = (Ctx*)h;
  const Model& m = c->m;
  const int ntp = (int)((double)(int)(rtmax - m.roc) / drtp + 1.0);
  *ntp_out = ntp;
  if (ntp > ntp_cap || ntp < 1) return 2;
  Spline s;
  if (computeSpline(m, m.fref, attmode, s)) return 2;
  const int nnod = c->ex.nnod;
  const double a0 = std::atan(std::sqrt(2.0 * eps));
  int first = 0;
  for (int n = 0; n < ntp; ++n) {
    const double rtp = m.roc + (double)n * drtp;
    rtp_out[n] = rtp;
    int nl, top;
    layerIndex(m, rtp, nl, top);
    if (top == 1) nl = nl + 1;
    RayEnv e;
    e.m = &m; e.ex = &c->ex; e.s = &s; e.nl = nl; e.stype = stype;
    e.p = rtp / rayVelocity(e, nl, rtp);
    slowness[n] = e.p;
    const double ys[2] = {a0, e.p * a0};
    std::vector<double> yn;
    int jl = 0, jr = -1;
    for (int j = 0; j < nnod; ++j) table[((size_t)n * nnod + j) * 2] = table[((size_t)n * nnod + j) * 2 + 1] = 0.0f;
    int rc = rayPropagate(e, eps, rtp * (1.0 + eps), c->ex.r[nnod], drtp, ys, yn, jl, jr);
    if (!rc && jr - jl < 0) rc = 4;
    status[n] = rc;
    if (rc) { if (!first) first = rc; continue; }
    for (int j = jl; j <= jr; ++j) {
      table[((size_t)n * nnod + (j - 1)) * 2] = (float)yn[(j - jl) * 2];
      table[((size_t)n * nnod + (j - 1)) * 2 + 1] = (float)yn[(j - jl) * 2 + 1];
    }
  }
  return first;
}

int oracle_spline(void* h, double f, int attmode, double* ro, double* ro2, double* el, double* el2) {
  Ctx* c = (Ctx*)h;
  Spline s;
  if (computeSpline(c->m, f, attmode, s)) return 2;
  for (int j = 1; j <= c->m.nk; ++j) {
    ro[j - 1] = s.ro[j]; ro2[j - 1] = s.ro2[j];
    for (int k = 0; k < 7; ++k) {
      el[((j - 1) * 7 + k) * 2] = s.el[j * 7 + k].re; el[((j - 1) * 7 + k) * 2 + 1] = s.el[j * 7 + k].im;
      el2[((j - 1) * 7 + k) * 2] = s.el2[j * 7 + k].re; el2[((j - 1) * 7 + k) * 2 + 1] = s.el2[j * 7 + k].im;
    }
  }
  return 0;
}

// start radius for (f, iwn) -- exposed for unit tests
double oracle_start_radius(void* h, double f, int attmode, double wn, int tor) {
  Ctx* c = (Ctx*)h;
  Spline s;
  computeSpline(c->m, f, attmode, s);
  Env e; e.m = &c->m; e.ex = &c->ex; e.s = &s; e.nl = 1;
  e.omre = 2.0 * PI_F * f; e.omim = 0.0;
  e.dll1 = (wn * c->m.rearth) * (wn * c->m.rearth);
  return startRadius(e, tor != 0);
}

// Analytic checks of the tests (homogeneous sphere).  Environment of one
// (omega, dll1) at frequency f with omim the imaginary part of the complex
// frequency (the FK loop uses -sigma), layer of radius r for an upward start.
static Env analyticEnv(Ctx* c, const Spline& s, double f, double omim, double dll1, double r) {
  Env e; e.m = &c->m; e.ex = &c->ex; e.s = &s;
  e.omre = 2.0 * PI_F * f; e.omim = omim; e.dll1 = dll1;
  int nl, top;
  layerIndex(c->m, r, nl, top);
  if (top == 1) nl = nl + 1;
  e.nl = nl;
  return e;
}

// Start vector of an upward integration at radius r, as the FK loop forms it:
// kind 0 toroidal (toroidalBottomInitialValues, initialValues.f90:376-416; 2
// values), 1 spheroidal minors (minorsBottomInitialValues, :202-275; 5 values).
// y: complex interleaved; returns the status of the continued fractions.
int oracle_bottom_iv(void* h, double f, int attmode, double omim, double dll1, double r, int kind, double* y,
                     double* htry) {
  Ctx* c = (Ctx*)h;
  Spline s;
  if (computeSpline(c->m, f, attmode, s)) return 2;
  Env e = analyticEnv(c, s, f, omim, dll1, r);
  zc ys[5];
  const int rc = kind == 0 ? toroidalBottomIV(e, r, ys, *htry) : minorsBottomIV(e, r, ys, *htry);
  const int nv = kind == 0 ? 2 : 5;
  for (int v = 0; v < nv; ++v) { y[2 * v] = ys[v].re; y[2 * v + 1] = ys[v].im; }
  return rc;
}

// One propagation (propagateOde.f90:132-331, with its renormalisation) of
// system sys (0 minors, 3 toroidal, 4 adjoint solid) from x1 to x2 with start
// vector y0 and initial step htry at accuracy eps: y1 = y(x2) / 10^lgnorm.
int oracle_propagate(void* h, double f, int attmode, double omim, double dll1, int sys, double x1, double x2,
                     double htry, double eps, const double* y0, double* y1, double* lgnorm) {
  Ctx* c = (Ctx*)h;
  if (sys < 0 || sys > 4) return 2;
  Spline s;
  if (computeSpline(c->m, f, attmode, s)) return 2;
  Env e = analyticEnv(c, s, f, omim, dll1, x1);
  if (x2 < x1) {   // downward: the layer containing x1 from above
    int nl, top;
    layerIndex(c->m, x1, nl, top);
    e.nl = nl;
  }
  Stats st{};
  Prop p; p.sys = sys; p.nv = nvarOf(sys); p.env = &e; p.eps = eps;
  p.do_norm = true; p.lgnorm = 0.0; p.st = &st;
  zc ys[5];
  for (int v = 0; v < p.nv; ++v) ys[v] = Z(y0[2 * v], y0[2 * v + 1]);
  const int rc = propagate(p, x1, x2, htry, ys);
  for (int v = 0; v < p.nv; ++v) { y1[2 * v] = p.y[v].re; y1[2 * v + 1] = p.y[v].im; }
  *lgnorm = p.lgnorm;
  return rc;
}

// Number of wavenumbers per frequency (computeGreenFKSpectraForSynthetics.f90:186-236)
// nwn must hold nf2 entries (index jf-1); returns nf1 and nf2 through pointers.
int oracle_nwn(void* h, const or_fk_params* p, int* nf1, int* nf2, int* nwn, int nwn_cap) {
  Ctx* c = (Ctx*)h;
  double df = 1.0 / p->tlen;
  int n2 = (int)std::lround(p->fmax / df) + 1;
  int n1 = std::max((int)std::lround(p->fmin / df), 2);
  double ommax = TWO_PI_F * (double)(n2 - 1) * df;
  double dwn = TWO_PI_F / p->xlen;
  double wnmax = 0.5 * ommax * (p->p1lim + p->p2lim) / (1.0 - p->frac);
  *nf1 = n1; *nf2 = n2;
  if (n2 > nwn_cap) return 2;
  for (int jf = 1; jf <= n2; ++jf) nwn[jf - 1] = 0;
  for (int jf = n1; jf <= n2; ++jf) {
    double f = (double)(jf - 1) * df;
    double omre = 2.0 * PI_F * f;
    double wn2;
    if (f <= (double)0.5f * (double)(n2 - 1) * df) wn2 = omre * p->p1lim + p->frac * wnmax;
    else wn2 = 0.5 * ommax * (p->p1lim + p->p2lim) + (omre - ommax) * p->p2lim + p->frac * wnmax;
    if (p->global == 1) nwn[jf - 1] = (int)std::lround(wn2 * c->m.rearth - (double)0.5f) + 1;
    else nwn[jf - 1] = (int)(wn2 / dwn) + 1;
  }
  return 0;
}

// One frequency jf (1-based): gf[(iwn-1) + nwn*((isp-1) + nsp*(n-1))] complex interleaved,
// status per iwn.  Returns nsp through *nsp_out.
int oracle_fk_frequency(void* h, const or_fk_params* p, int jf, int nwn, double* gf, int* status,
                        or_stats* stats_out, int iwn_lo, int iwn_hi) {
  Ctx* c = (Ctx*)h;
  const Model& m = c->m;
  const Nodes& ex = c->ex;
  int nnod = ex.nnod;
  double df = 1.0 / p->tlen;
  double sigma = 5.0 * df;
  double dwn = TWO_PI_F / p->xlen;
  double f = (double)(jf - 1) * df;
  double omre = 2.0 * PI_F * f;
  Spline s;
  if (computeSpline(m, f, p->attmode, s)) return 2;
  int jre = p->jre;
  int dsvstep = p->stressflag ? 1 : 2;
  int ncsph, nctor, njsph, njtor;
  if (ex.state[jre] == 1) { ncsph = 2; nctor = 0; } else { ncsph = 4; nctor = 2; }
  if (p->istyp == 0) { njsph = 2; njtor = 1; } else { njsph = 4; njtor = 2; }
  // a receiver in the ocean (extra V component, fluidOdeSystem.f90:171-188) is not restated
  if (ex.state[jre] == 1) return -1;
  int dsvs = (dsvstep == 1 ? 4 : 2);   // sum(dsvmask_sph)
  int dsvt = (dsvstep == 1 ? 2 : 1);   // sum(dsvmask_tor)
  int nsp = dsvs * njsph + dsvt * njtor;
  int iwa = (p->global == 1) ? 1 : 2;
  Stats tot;
  int lo = std::max(iwa, iwn_lo), hi = std::min(nwn, iwn_hi);
  for (int iwn = 1; iwn <= nwn; ++iwn) status[iwn - 1] = 0;
  for (int iwn = lo; iwn <= hi; ++iwn) {
    double wn = (double)(iwn - 1) * dwn;
    if (p->global == 1) wn = std::sqrt((double)((int64_t)(iwn - 1) * iwn)) / m.rearth;
    Env gem; gem.m = &m; gem.ex = &ex; gem.s = &s; gem.nl = 1;
    gem.dll1 = (wn * m.rearth) * (wn * m.rearth);
    gem.omre = omre; gem.omim = -sigma;
    Stats st;
    TorMin T; SphMin S; UJGF U;
    int rc = computeToroidalMinors(T, jre, jre, gem, p->eps, st);
    if (!rc) rc = computeSpheroidalMinors(S, jre, jre, gem, p->eps, st);
    if (!rc) rc = computeUJGF(U, T, S, jre, gem, p->eps, st);
    tot.add(st);
    if (rc) { status[iwn - 1] = rc; continue; }
    double re = ex.r[jre];
    for (int n = 1; n <= nnod; ++n) {
      zc bgin[4][4], bgout[4][4], zsph[4][4], ztor[2][2];
      for (int cc = 0; cc < 4; ++cc) for (int j = 0; j < 4; ++j)
        bgin[cc][j] = (j < U.njs) ? U.sph[((size_t)n * 4 + j) * 4 + cc] : Z(0.0);
      sphRecip(gem.dll1, re, ex.r[n], ex.state[n], ex.state[jre], bgin, bgout);
      zc bgtor[2][2] = {{Z(0), Z(0)}, {Z(0), Z(0)}};
      if (nctor > 0) {
        double ft = (ex.r[n] / re) * (ex.r[n] / re);
        zc ti[2][2];
        for (int cc = 0; cc < 2; ++cc) for (int j = 0; j < 2; ++j) ti[cc][j] = U.tor[((size_t)n * 2 + j) * 2 + cc];
        bgtor[0][0] = (-ft) * ti[1][1]; bgtor[1][0] = ft * ti[1][0];
        bgtor[0][1] = ft * ti[0][1]; bgtor[1][1] = (-ft) * ti[0][0];
      }
      sourceTerms(p->istyp, gem.dll1, gem.omre, ex.r[n], ex.state[n], ex.layer[n], s, zsph, ztor);
      zc gfsph[4][4], gftor[2][2];
      for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) gfsph[i][j] = Z(0.0);
      for (int i = 0; i < 2; ++i) for (int j = 0; j < 2; ++j) gftor[i][j] = Z(0.0);
      if (ex.state[n] == 1) {
        for (int j = 0; j < 2; ++j) for (int k = 0; k < 2; ++k) for (int i = 0; i < ncsph; ++i)
          gfsph[i][j] = gfsph[i][j] + bgout[i][k] * zsph[k][j];
      } else {
        for (int j = 0; j < njsph; ++j) for (int k = 0; k < 4; ++k) for (int i = 0; i < ncsph; ++i)
          gfsph[i][j] = gfsph[i][j] + bgout[i][k] * zsph[k][j];
        if (nctor > 0)
          for (int j = 0; j < njtor; ++j) for (int k = 0; k < 2; ++k) for (int i = 0; i < nctor; ++i)
            gftor[i][j] = gftor[i][j] + bgtor[i][k] * ztor[k][j];
      }
      int isp = 0;
      auto put = [&](zc v) {
        size_t o = ((size_t)(iwn - 1) + (size_t)nwn * ((size_t)isp + (size_t)nsp * (n - 1))) * 2;
        gf[o] = v.re; gf[o + 1] = v.im; isp++;
      };
      for (int i = 0; i < ncsph; i += dsvstep) for (int j = 0; j < njsph; ++j) put(gfsph[i][j]);
      for (int i = 0; i < nctor; i += dsvstep) for (int j = 0; j < njtor; ++j) put(gftor[i][j]);
    }
  }
  if (stats_out) {
    stats_out->steps_ok = tot.steps_ok; stats_out->steps_rej = tot.steps_rej;
    stats_out->attempts = tot.attempts; stats_out->sysmats = tot.sysmats;
    stats_out->matvecs = tot.matvecs; stats_out->flops = tot.flops;
  }
  return nsp;
}

}  // extern "C"

// ===========================================================================
//  DSV spectra with radial derivatives for several source nodes
//  (computeGreenFKSpectraForASKI.f90:451-560, dsvDerivatives.f90:39-72)
// ===========================================================================
// solid system matrix (solidOdeSystem.f90:77-114), column-major a[i + 4*j]
static void solidSysmat(const Env& e, double x, zc* a) {
  double ro; zc el[7];
  evalSpline(*e.s, x, e.nl, ro, el);
  zc zom = Z(e.omre, e.omim);
  double dll1 = e.dll1, rr = 1.0 / x, rr2 = rr * rr;
  zc zrpc = 1.0 / el[1];
  zc z1 = el[0] - (el[2] * el[2]) * zrpc - el[4];
  zc z2 = (el[2] * rr) * zrpc;
  zc zdlz1 = dll1 * z1;
  zc zomro = zom * zom * ro;
#define A(i, j) a[((i)-1) + 4 * ((j)-1)]
  A(1, 1) = -(2.0 * z2);
  A(1, 2) = zrpc;
  A(1, 3) = dll1 * z2;
  A(1, 4) = Z(-0.0);
  A(2, 1) = (-zomro) + (4.0 * z1) * rr2;
  A(2, 2) = 2.0 * z2 - 2.0 * rr;
  A(2, 3) = -((2.0 * rr2) * zdlz1);
  A(2, 4) = Z(dll1 * rr);
  A(3, 1) = Z(-rr);
  A(3, 2) = Z(-0.0);
  A(3, 3) = Z(rr);
  A(3, 4) = 1.0 / el[3];
  A(4, 1) = -((2.0 * z1) * rr2);
  A(4, 2) = -z2;
  A(4, 3) = (-zomro) + (zdlz1 + (dll1 - 2.0) * el[4]) * rr2;
  A(4, 4) = Z(-3.0 * rr);
#undef A
}

// gfd = A(r) gf for nj jump vectors of nv components (computeDsvDerivatives:
// layer of r by getLayerIndexNodeEarthmodel, gfortran matmul order)
static void dsvDerivatives(const Env& gem, double r, bool tor, int nj, const zc gf[4][4], zc gfd[4][4]) {
  Env e = gem;
  int nl, top;
  layerIndex(*gem.m, r, nl, top);
  e.nl = nl;
  const int nv = tor ? 2 : 4;
  zc a[16];
  if (tor) sysmat(SYS_TOROIDAL, e, r, a); else solidSysmat(e, r, a);
  for (int j = 0; j < nj; ++j) {
    for (int i = 0; i < nv; ++i) gfd[i][j] = Z(0.0);
    for (int k = 0; k < nv; ++k)
      for (int i = 0; i < nv; ++i) gfd[i][j] = gfd[i][j] + a[i + nv * k] * gf[k][j];
  }
}

extern "C" {
// One frequency jf of the ASKI variant: minors once over the source-node range
// min(jsnod)..max(jsnod), then for each source node jsnod[js] (js < nsnod,
// source type p->istyp) and for a force at p->jre (js = nsnod): U, V, dU/dr,
// dV/dr for every spheroidal jump, then W, dW/dr for every toroidal jump, at
// every node.  gf holds (nsnod+1) blocks of nwn*20*nnod complex values; block
// js is indexed [(iwn-1) + nwn*(isp + nsp_js*(n-1))] and nsp_js goes to
// nsp_out[js].  Sources and nodes in fluid layers are not restated (-1).
int oracle_dsv_frequency(void* h, const or_fk_params* p, const int* jsnod, int nsnod, int jf, int nwn,
                         double* gf, int* nsp_out, int* status, or_stats* stats_out, int iwn_lo, int iwn_hi) {
  Ctx* c = (Ctx*)h;
  const Model& m = c->m;
  const Nodes& ex = c->ex;
  const int nnod = ex.nnod;
  if (nsnod < 1) return -1;
  for (int n = 1; n <= nnod; ++n) if (ex.state[n] != 0) return -1;
  int jsl = jsnod[0], jsr = jsnod[0];
  bool jre_in = false;
  for (int js = 0; js < nsnod; ++js) {
    if (jsnod[js] < 1 || jsnod[js] > nnod) return -1;
    jsl = std::min(jsl, jsnod[js]); jsr = std::max(jsr, jsnod[js]);
    jre_in = jre_in || jsnod[js] == p->jre;
  }
  if (!jre_in) return -1;   // receiver node must also be a source node (:206-209)
  const double df = 1.0 / p->tlen, sigma = 5.0 * df, dwn = TWO_PI_F / p->xlen;
  const double f = (double)(jf - 1) * df, omre = 2.0 * PI_F * f;
  Spline s;
  if (computeSpline(m, f, p->attmode, s)) return 2;
  const size_t block = (size_t)nwn * 20 * nnod * 2;
  for (int js = 0; js <= nsnod; ++js) {
    int ty = js == nsnod ? 0 : p->istyp;
    nsp_out[js] = 4 * (ty == 0 ? 2 : 4) + 2 * (ty == 0 ? 1 : 2);
  }
  const int iwa = (p->global == 1) ? 1 : 2;
  Stats tot;
  for (int iwn = 1; iwn <= nwn; ++iwn) status[iwn - 1] = 0;
  const int lo = std::max(iwa, iwn_lo), hi = std::min(nwn, iwn_hi);
  for (int iwn = lo; iwn <= hi; ++iwn) {
    double wn = (double)(iwn - 1) * dwn;
    if (p->global == 1) wn = std::sqrt((double)((int64_t)(iwn - 1) * iwn)) / m.rearth;
    Env gem; gem.m = &m; gem.ex = &ex; gem.s = &s; gem.nl = 1;
    gem.dll1 = (wn * m.rearth) * (wn * m.rearth);
    gem.omre = omre; gem.omim = -sigma;
    Stats st;
    TorMin T; SphMin S;
    int rc = computeToroidalMinors(T, jsl, jsr, gem, p->eps, st);
    if (!rc) rc = computeSpheroidalMinors(S, jsl, jsr, gem, p->eps, st);
    for (int js = 0; js <= nsnod && !rc; ++js) {
      const int ty = js == nsnod ? 0 : p->istyp;
      const int jsh = js == nsnod ? p->jre : jsnod[js];
      const int njsph = ty == 0 ? 2 : 4, njtor = ty == 0 ? 1 : 2, nsp = nsp_out[js];
      UJGF U;
      rc = computeUJGF(U, T, S, jsh, gem, p->eps, st);
      if (rc) break;
      zc zsph[4][4], ztor[2][2];
      sourceTerms(ty, gem.dll1, gem.omre, ex.r[jsh], ex.state[jsh], ex.layer[jsh], s, zsph, ztor);
      double* g = gf + js * block;
      for (int n = 1; n <= nnod; ++n) {
        zc gfsph[4][4], gftor[4][4], gfds[4][4], gfdt[4][4];
        for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) gfsph[i][j] = gftor[i][j] = Z(0.0);
        for (int j = 0; j < njsph; ++j) for (int k = 0; k < 4; ++k) for (int i = 0; i < 4; ++i)
          gfsph[i][j] = gfsph[i][j] + U.sph[((size_t)n * 4 + k) * 4 + i] * zsph[k][j];
        for (int j = 0; j < njtor; ++j) for (int k = 0; k < 2; ++k) for (int i = 0; i < 2; ++i)
          gftor[i][j] = gftor[i][j] + U.tor[((size_t)n * 2 + k) * 2 + i] * ztor[k][j];
        dsvDerivatives(gem, ex.r[n], false, njsph, gfsph, gfds);
        dsvDerivatives(gem, ex.r[n], true, njtor, gftor, gfdt);
        int isp = 0;
        auto put = [&](zc v) {
          size_t o = ((size_t)(iwn - 1) + (size_t)nwn * ((size_t)isp + (size_t)nsp * (n - 1))) * 2;
          g[o] = v.re; g[o + 1] = v.im; isp++;
        };
        for (int i = 0; i < 4; i += 2) for (int j = 0; j < njsph; ++j) put(gfsph[i][j]);
        for (int i = 0; i < 4; i += 2) for (int j = 0; j < njsph; ++j) put(gfds[i][j]);
        for (int j = 0; j < njtor; ++j) put(gftor[0][j]);
        for (int j = 0; j < njtor; ++j) put(gfdt[0][j]);
      }
    }
    tot.add(st);
    if (rc) {
      status[iwn - 1] = rc;
      for (int js = 0; js <= nsnod; ++js) {   // a failed item leaves zeros, as the GPU path does
        double* g = gf + js * block;
        for (int n = 1; n <= nnod; ++n)
          for (int isp = 0; isp < nsp_out[js]; ++isp) {
            size_t o = ((size_t)(iwn - 1) + (size_t)nwn * ((size_t)isp + (size_t)nsp_out[js] * (n - 1))) * 2;
            g[o] = 0.0; g[o + 1] = 0.0;
          }
      }
    }
  }
  if (stats_out) {
    stats_out->steps_ok = tot.steps_ok; stats_out->steps_rej = tot.steps_rej;
    stats_out->attempts = tot.attempts; stats_out->sysmats = tot.sysmats;
    stats_out->matvecs = tot.matvecs; stats_out->flops = tot.flops;
  }
  return nsnod + 1;
}

}  // extern "C"
