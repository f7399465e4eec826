// =============================================================================
//  GEMINI FK hot path -- CPU FP64 ORACLE, phase 2 (synthetic seismograms).
//  Test infrastructure only; see oracle_core.h for the conventions.
//
//  Restates:
//    legendreFunctions.f90:48-157            (P_l^m, m <= 2, and derivatives)
//    harmonicDegreeSums.f90:231-369,34-45    (moment degree sums, cos^2 taper)
//    displacementSpectra.f90:49-113          (frequency loop, sum -> FK index)
//    singleFrequencyDisplacement.f90:108-125 (ZRT from the 14 sums)
//    eventFilter.f90:40-83, butterworthFilter.f90:49-96 (complex-omega band-pass)
//    computeSyntheticSeismograms.f90:355-388 (time shift, velocity, ZNE rotation)
//    axesRotation.f90:560-568                (RLT -> ZNE)
//    frequencyTime.f90:34-113, fourierTransform.f90:118-192 (iFFT, exp(sigma t))
// =============================================================================
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "oracle_core.h"

using namespace orc;

namespace {

struct Legendre {
  int lmax;
  // [m][l], m = 0..2 ; pdst/dtpdst use m = 1..2 (m = 0 row unused)
  std::vector<double> plm[3], dpdt[3], pdst[3], d2pdt2[3], dtpdst[3];
};

// legendreFunctions.f90:48-157 (mmax = 2)
void computeLegendre(int lmax, double theta, Legendre& a) {
  const int mmax = 2;
  a.lmax = lmax;
  for (int m = 0; m < 3; ++m) {
    a.plm[m].assign(lmax + 2, 0.0); a.dpdt[m].assign(lmax + 2, 0.0); a.pdst[m].assign(lmax + 2, 0.0);
    a.d2pdt2[m].assign(lmax + 2, 0.0); a.dtpdst[m].assign(lmax + 2, 0.0);
  }
  double ct = std::cos(theta), st = std::sin(theta);
  bool atpoles = !(st > 0.0);
  for (int m = 0; m <= mmax; ++m) {
    if (m > lmax) break;
    a.plm[m][m] = 1.0;
    double fact = 1.0;
    for (int j = 1; j <= m; ++j) { a.plm[m][m] = a.plm[m][m] * fact * st; fact = fact + 2.0; }
    if (m + 1 <= lmax) a.plm[m][m + 1] = ct * (double)(2 * m + 1) * a.plm[m][m];
    for (int l = m + 2; l <= lmax; ++l)
      a.plm[m][l] = (ct * (double)(2 * l - 1) * a.plm[m][l - 1] - (double)(l + m - 1) * a.plm[m][l - 2]) /
                    (double)(l - m);
  }
  if (!atpoles) {
    double rst = 1.0 / st;
    for (int m = 0; m <= mmax; ++m) {
      if (m > lmax) break;
      a.dpdt[m][m] = (double)m * ct * a.plm[m][m] * rst;
      for (int l = m + 1; l <= lmax; ++l)
        a.dpdt[m][l] = ((double)l * ct * a.plm[m][l] - (double)(l + m) * a.plm[m][l - 1]) * rst;
    }
    for (int m = 1; m <= mmax; ++m)
      for (int l = m; l <= lmax; ++l) a.pdst[m][l] = a.plm[m][l] * rst;
    for (int m = 0; m <= mmax; ++m)
      for (int l = m; l <= lmax; ++l)
        a.d2pdt2[m][l] = (-ct) * rst * a.dpdt[m][l] + ((double)(m * m) * (rst * rst) - (double)(l * (l + 1))) * a.plm[m][l];
    for (int m = 1; m <= mmax; ++m)
      for (int l = m; l <= lmax; ++l) a.dtpdst[m][l] = rst * (a.dpdt[m][l] - ct * rst * a.plm[m][l]);
  } else {
    int isct = (int)std::copysign(1.0, ct);
    auto ipow = [](int b, int e) { int r = 1; for (int i = 0; i < e; ++i) r *= b; return r; };
    for (int l = 0; l <= lmax; ++l) {
      a.dpdt[0][l] = 0.0;
      a.dpdt[1][l] = 0.5 * (double)(l * (l + 1) * ipow(isct, l));
      a.dpdt[2][l] = 0.0;
    }
    for (int l = 1; l <= lmax; ++l) {
      a.pdst[1][l] = 0.5 * (double)(l * (l + 1) * ipow(isct, l + 1));
      a.pdst[2][l] = 0.0;
    }
    for (int l = 0; l <= lmax; ++l) {
      a.d2pdt2[0][l] = 0.5 * (double)(l * (l + 1) * ipow(isct, l));
      a.d2pdt2[1][l] = 0.0;
      a.d2pdt2[2][l] = 0.25 * (double)((l + 2) * (l + 1) * l * (l - 1) * ipow(isct, l));
    }
    for (int l = 1; l <= lmax; ++l) {
      a.dtpdst[1][l] = 0.0;
      a.dtpdst[2][l] = 0.125 * (double)((l + 2) * (l + 1) * l * (l - 1) * ipow(isct, l + 1));
    }
  }
}

// taperHarmonicDegreeSums (harmonicDegreeSums.f90:356-369)
void taper(int lmax, double tapfrac, std::vector<double>& g) {
  g.assign(lmax + 1, 0.0);
  int jt = std::min((int)std::lround((double)lmax * (1.0 - tapfrac)), lmax);
  jt = std::max(1, jt);
  double c1 = (double)lmax * tapfrac * 2.0 / PI_F;
  double c2 = (1.0 - tapfrac) / tapfrac * 0.5 * PI_F;
  for (int j = 0; j <= jt - 1 && j <= lmax; ++j) g[j] = 1.0;
  for (int j = jt; j <= lmax; ++j) {
    double c = std::cos((double)(float)j / c1 - c2);
    g[j] = c * c;
  }
}

// table kind and factor of the 14 moment sums (harmonicDegreeSums.f90:297-351)
// kind: 0 plm, 1 dpdt, 2 pdst ; m ; l start ; factor numerator (0 => none)
struct SumDef { int kind, m, l0; double fnum; int comp, jump; };
const SumDef MSUM[14] = {
    {0, 0, 0, 0.0, 1, 1},  {0, 0, 0, 0.0, 1, 2},  {0, 1, 1, 2.0, 1, 3},  {0, 2, 2, 2.0, 1, 4},
    {1, 0, 1, 0.0, 3, 1},  {1, 0, 1, 0.0, 3, 2},  {1, 1, 1, 2.0, 3, 3},  {1, 2, 2, 2.0, 3, 4},
    {2, 1, 1, 2.0, 7, 1},  {2, 2, 2, 4.0, 7, 2},  {1, 1, 1, 2.0, 7, 1},  {1, 2, 2, -2.0, 7, 2},
    {2, 1, 1, 2.0, 3, 3},  {2, 2, 2, -4.0, 3, 4}};

// table kind and factor of the 7 force sums (harmonicDegreeSums.f90:110-171):
// kint 1 P_l0 U1, 2 P_l1 (-2/elp1) U2, 3 dpdt_l0 V1, 4 dpdt_l1 (-2/elp1) V2,
// 5 pdst_l1 (-2/elp1) W1, 6 dpdt_l1 (+2/elp1) W1, 7 pdst_l1 (+2/elp1) V2
const SumDef FSUM[7] = {
    {0, 0, 0, 0.0, 1, 1}, {0, 1, 1, -2.0, 1, 2}, {1, 0, 1, 0.0, 3, 1}, {1, 1, 1, -2.0, 3, 2},
    {2, 1, 1, -2.0, 7, 1}, {1, 1, 1, 2.0, 7, 1}, {2, 1, 1, 2.0, 3, 2}};

// forceHarmonicDegreeSums for kint 1..7: T (fnum/elp1) G (2l+1)/4pi taper
zc forceSum(int kint, const float* gr, const float* gi, int nwn, const Legendre& alf, const std::vector<double>& tap) {
  const SumDef& s = FSUM[kint - 1];
  const std::vector<double>& T =
      s.kind == 0 ? alf.plm[s.m] : (s.kind == 1 ? alf.dpdt[s.m] : alf.pdst[s.m]);
  double fourpi = 4.0 * PI_F;
  int lmax = nwn - 1;
  zc z = Z(0.0);
  for (int l = s.l0; l <= lmax; ++l) {
    zc g = Z((double)gr[l], (double)gi[l]);
    zc t;
    if (s.fnum == 0.0) t = T[l] * g;
    else t = (T[l] * (s.fnum / (double)(float)(l * (l + 1)))) * g;
    t = ((t * (2.0 * (double)l + 1.0)) / fourpi) * tap[l];
    z = z + t;
  }
  return z;
}

// momentHarmonicDegreeSums for kint 1..14 over lmax = nwn-1 terms
zc momentSum(int kint, const float* gr, const float* gi, int nwn, const Legendre& alf,
             const std::vector<double>& tap) {
  const SumDef& s = MSUM[kint - 1];
  const std::vector<double>& T =
      s.kind == 0 ? alf.plm[s.m] : (s.kind == 1 ? alf.dpdt[s.m] : alf.pdst[s.m]);
  double fourpi = 4.0 * PI_F;
  int lmax = nwn - 1;
  zc z = Z(0.0);
  for (int l = s.l0; l <= lmax; ++l) {
    zc g = Z((double)gr[l], (double)gi[l]);
    zc t;
    if (s.fnum == 0.0) t = T[l] * g;
    else t = ((T[l] * s.fnum) / (double)(float)(l * (l + 1))) * g;
    t = ((t * (2.0 * (double)l + 1.0)) / fourpi) * tap[l];
    z = z + t;
  }
  return z;
}

// doubleFastFourierTransform (fourierTransform.f90:118-192), 1-based x,y
void fft(std::vector<double>& x, std::vector<double>& y, int n, int is) {
  double piz = 2.0 * PI_F;
  std::vector<int> zh(n + 2);
  zh[1] = 1;
  for (int l = 1; l <= n; ++l) zh[l + 1] = 2 * zh[l];
  int ng = zh[n + 1];
  double gn = 1.0 / (double)ng;
  for (int m = 1; m <= n; ++m) {
    int nar = zh[m], lar = ng / nar, larh = lar / 2;
    double alpha = piz / (double)(is >= 0 ? lar : -lar);
    for (int jr = 1; jr <= larh; ++jr) {
      double beta = alpha * (double)(jr - 1);
      double excos = std::cos(beta), exsin = std::sin(beta);
      int ja = jr - lar;
      for (int nr = 1; nr <= nar; ++nr) {
        ja = ja + lar;
        int jb = ja + larh;
        double zx = x[ja] - x[jb], zy = y[ja] - y[jb];
        x[ja] = x[ja] + x[jb];
        y[ja] = y[ja] + y[jb];
        x[jb] = zx * excos - zy * exsin;
        y[jb] = zx * exsin + zy * excos;
      }
    }
  }
  int ais = is < 0 ? -is : is;
  if (ais == 3) gn = std::sqrt(gn);
  if (ais == 2 || ais == 3) for (int i = 1; i <= ng; ++i) { y[i] *= gn; x[i] *= gn; }
  for (int j = 1; j <= ng; ++j) {
    int js = j - 1, k = 1, nny = n + 1;
    for (int ny = 1; ny <= n; ++ny) {
      nny = nny - 1;
      if (js < zh[nny]) continue;
      js = js - zh[nny];
      k = k + zh[ny];
    }
    if (j - k < 0) {
      std::swap(x[j], x[k]); std::swap(y[j], y[k]);
    }
  }
}

// transformFrequencyTime (frequencyTime.f90:55-113); sp 1-based [1..nf2]
int freqTime(int nf1, int nf2, double df, double sigma, const std::vector<zc>& sp, int nsamp,
             double dt, float* ts, int* warning = nullptr) {
  int nslog = (int)std::ceil((double)std::log((float)nf2) / std::log(2.0)) + 1;
  int ns = 1 << nslog;
  double dts; int ndec;
  if (ns <= nsamp) {
    ns = nsamp;
    nslog = (int)std::ceil(-std::log(df * dt) / std::log(2.0));
    dts = dt; ndec = 1;
  } else {
    dts = 1.0 / (df * ns);
    ndec = (int)std::lround(dt / dts);
    if (std::fabs(dt - ndec * dts) > 1.e-5) return 2;
    if (warning) *warning = 1;   // 'Downsampling to less than 1./(2*fny) requested'
  }
  if ((1 << nslog) != ns) return 2;   // inconsistent nsamp / dt
  if ((long long)ndec * (nsamp - 1) >= ns) return 2;   // beyond the period 1/df
  std::vector<double> x(ns + 1, 0.0), y(ns + 1, 0.0);
  for (int i = nf1; i <= nf2; ++i) { x[i] = sp[i].re; y[i] = sp[i].im; }
  for (int i = ns / 2 + 2; i <= ns; ++i) { x[i] = x[ns - i + 2]; y[i] = -y[ns - i + 2]; }
  fft(x, y, nslog, +1);
  double fac = 1.0, expo = std::exp(sigma * dts);
  for (int i = 1; i <= nsamp; ++i) {
    ts[i - 1] = (float)(x[ndec * (i - 1) + 1] * df * fac);
    fac = fac * expo;
  }
  return 0;
}

// complex-omega Butterworth band-pass (eventFilter.f90:40-83, butterworthFilter.f90:49-96)
void eventFilter(int nordh, double fch, int nordl, double fcl, int nf1, int nf2, double df,
                 double sigma, std::vector<zc>& hfil) {
  hfil.assign(nf2 + 1, Z(0.0));
  int nf = nf2 - nf1 + 1;
  double fmin = (double)(nf1 - 1) * df;
  const zc ci = Z(0.0, 1.0);
  std::vector<zc> hh(nf, Z(1.0)), hl(nf, Z(1.0));
  zc zfna = (fmin - (ci * sigma) / TWO_PI_F) / fch;
  for (int j = 1; j <= nordh; ++j) {
    zc zfn = zfna;
    zc ep = zexp(((ci * PI_F) * ((double)j - 0.5)) / (double)nordh);
    for (int i = 0; i < nf; ++i) { hh[i] = (hh[i] * zfn) / (zfn - ep); zfn = zfn + df / fch; }
  }
  zfna = (fmin - (ci * sigma) / TWO_PI_F) / fcl;
  for (int j = 1; j <= nordl; ++j) {
    zc zfn = zfna;
    zc ep = zexp(((ci * PI_F) * ((double)j - 0.5)) / (double)nordl);
    for (int i = 0; i < nf; ++i) { hl[i] = (hl[i] * (-ci)) / (zfn - ep); zfn = zfn + df / fcl; }
  }
  for (int i = 0; i < nf; ++i) hfil[nf1 + i] = hh[i] * hl[i];
}

}  // namespace


namespace {
// ---------------------------------------------------------------------------
//  Regional (Bessel) mode: wavenumber integrals
// ---------------------------------------------------------------------------
// Bessel functions at the wavenumber points (besselFunctions.f90:33-51): J[3*(j-1) + n]
// for j = 1..nwn, wn accumulated as wn = wn + dwn.  J0 and J1 come from the C
// library (the reference evaluates Cody's rational approximations CALJY0/CALJY1,
// accurate to double precision).
void besselTable(int nwn, double dwn, double x, std::vector<double>& J) {
  J.assign(3 * (size_t)nwn, 0.0);
  J[0] = 1.0;
  double wn = dwn;
  for (int j = 2; j <= nwn; ++j) {
    double j0v = ::j0(wn * x), j1v = ::j1(wn * x);
    J[3 * (j - 1)] = j0v;
    J[3 * (j - 1) + 1] = j1v;
    J[3 * (j - 1) + 2] = -j0v + 2.0 / (wn * x) * j1v;
    wn = wn + dwn;
  }
}

// integrand factor of moment integral kint (1..14) at wavenumber wn from the
// Bessel values b0, b1, b2 at wn*x (wavenumberIntegrals.f90:352-366, 372-386)
double wnKernel(int kint, double wn, double b0, double b1, double b2, double re, double x) {
  switch (kint) {
    case 1: case 2: return wn * b0;
    case 3: return 2.0 / re * b1;
    case 4: return wn * 2.0 * b2;
    case 5: case 6: return wn * (-wn * re) * b1;
    case 7: case 11: return wn * 2.0 * (b0 - b1 / (wn * x));
    case 8: return wn * 2.0 * wn * re * (b1 - 2.0 * b2 / (wn * x));
    case 9: case 13: return wn * 2.0 * b1 / (wn * x);
    case 10: return wn * 4.0 * wn * re * b2 / (wn * x);
    case 12: return -(wn * 2.0 * wn * re * (b1 - 2.0 * b2 / (wn * x)));
    default: return -(wn * 4.0 * wn * re * b2 / (wn * x));   // 14
  }
}

// integrand factor of force integral kint (1..7) (wavenumberIntegrals.f90:160-168, 172-180)
double wnKernelForce(int kint, double wn, double b0, double b1, double b2, double re, double x) {
  (void)b2;
  switch (kint) {
    case 1: return wn * b0;
    case 2: return -2 * b1 / re;
    case 3: return -wn * wn * b1 * re;
    case 4: return -2. * wn * (b0 - b1 / (wn * x));
    case 5: return -2. * wn * b1 / (wn * x);
    case 6: return +2. * wn * (b0 - b1 / (wn * x));
    default: return +2. * wn * b1 / (wn * x);   // 7
  }
}

typedef double (*WnKernelFn)(int, double, double, double, double, double, double);

// cos^2 taper of the wavenumber integrals (wavenumberIntegrals.f90:480-491), 1-based g[j]
void taperWn(int nwn, double dwn, double tapfrac, std::vector<double>& g) {
  int jt = std::min((int)std::lround((double)nwn * (1.0 - tapfrac)), nwn);
  jt = std::max(1, jt);
  double c1 = (double)(nwn - 1) * dwn * tapfrac * 2.0 / PI_F;
  double c2 = (1.0 - tapfrac) / tapfrac * 0.5 * PI_F;
  g.assign(nwn + 1, 1.0);
  for (int j = jt; j <= nwn; ++j) { double c = std::cos((double)(j - 1) * dwn / c1 - c2); g[j] = c * c; }
}

// momentWavenumberIntegrals (wavenumberIntegrals.f90:320-475) for one frequency:
// G 1-based [1..nwn] of the integral's FK column, J the Bessel table of distance xx
zc wavenumberIntegral(WnKernelFn kernfn, int kint, const std::vector<zc>& G, int nwn, double dwn, double re,
                      double xx, const std::vector<double>& J, const std::vector<double>& tap) {
  double x = xx < 3.0 / (dwn * 1.e9) ? 3.0 / (dwn * 1.e9) : xx;
  double wn3 = 3.0 / x;
  int j3 = (int)(wn3 / dwn) + 2;
  wn3 = (double)(j3 - 1) * dwn;
  auto wnb = [&](int j) {
    double wn = (double)(j - 1) * dwn;
    return kernfn(kint, wn, J[3 * (j - 1)], J[3 * (j - 1) + 1], J[3 * (j - 1) + 2], re, x);
  };
  auto ybes = [&](double w) {
    double y0v = ::y0(w * x), y1v = ::y1(w * x);
    double y2v = -y0v + 2.0 / (w * x) * y1v;
    return kernfn(kint, w, y0v, y1v, y2v, re, x);
  };
  double wn3besy = ybes(wn3);
  int j33 = std::min(j3, nwn);
  zc zdis = Z(0.0);
  for (int j = 2; j <= j33 - 1; ++j) zdis = zdis + (G[j] * wnb(j)) * tap[j];
  zdis = zdis + ((0.5 * G[j33]) * wnb(j33)) * tap[j33];
  zdis = zdis * dwn;
  if (j33 != nwn) {
    double wne = (double)(nwn - 1) * dwn;
    double wnbesy = ybes(wne);
    double xdk = x * dwn;
    zc zsum = (G[j3] * wnb(j3)) * tap[j3];
    for (int j = j3 + 1; j <= nwn - 1; ++j) zsum = zsum + ((2.0 * G[j]) * wnb(j)) * tap[j];
    zsum = zsum + (G[nwn] * wnb(nwn)) * tap[nwn];
    zdis = zdis + ((zsum / x) * (1.0 - std::cos(xdk))) / xdk;
    zdis = zdis + (((G[nwn] * wnbesy) * tap[nwn] - (G[j3] * wn3besy) * tap[j3]) / x) * (1.0 - std::sin(xdk) / xdk);
  }
  return zdis * (re * re / (2.0 * PI_F));
}

}  // namespace

extern "C" {

// Wavenumber integrals of the regional mode: hd[(sta*nf2 + jf-1)*nsum + k] complex
// interleaved for the 14 moment (istyp 1) or 7 force (istyp 0) integrals; x: distances in m.
int oracle_wavenumber_integrals_src(int istyp, int nf1, int nf2, const int* nwn, int nwnmax, int nkfmax, int nsp,
                                    const float* gr, const float* gi, double dwn, double rearth, int nsta,
                                    const double* x, double* hd) {
  static const int mcol[14] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 8, 9, 6, 7};   // FK column of each integral
  static const int fcol[7] = {0, 1, 2, 3, 4, 4, 3};
  const int nsum = istyp == 1 ? 14 : 7;
  const int* col = istyp == 1 ? mcol : fcol;
  if (nsp < (istyp == 1 ? 10 : 5)) return 2;
  std::vector<int> koff(nf2 + 1, 0);
  long long k = 0;
  for (int jf = nf1; jf <= nf2; ++jf) { koff[jf] = (int)k; k += nwn[jf - 1]; }
  if (k > nkfmax) return 2;
  std::vector<double> J, tap;
  std::vector<zc> G;
  for (int is = 0; is < nsta; ++is) {
    besselTable(nwnmax, dwn, x[is], J);
    for (int jf = nf1; jf <= nf2; ++jf) {
      const int n = nwn[jf - 1];
      taperWn(n, dwn, 0.2, tap);
      for (int kk = 1; kk <= nsum; ++kk) {
        G.assign(n + 1, Z(0.0));
        const long long o = (long long)col[kk - 1] * nkfmax + koff[jf];
        for (int j = 1; j <= n; ++j) G[j] = Z((double)gr[o + j - 1], (double)gi[o + j - 1]);
        zc z = wavenumberIntegral(istyp == 1 ? wnKernel : wnKernelForce, kk, G, n, dwn, rearth, x[is], J, tap);
        double* h = hd + (((size_t)is * nf2 + (jf - 1)) * nsum + (kk - 1)) * 2;
        h[0] = z.re; h[1] = z.im;
      }
    }
  }
  return 0;
}

int oracle_wavenumber_integrals(int nf1, int nf2, const int* nwn, int nwnmax, int nkfmax, int nsp,
                                const float* gr, const float* gi, double dwn, double rearth, int nsta,
                                const double* x, double* hd) {
  return oracle_wavenumber_integrals_src(1, nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, dwn, rearth, nsta, x, hd);
}

// Legendre tables for the unit tests: out[kind*3*(lmax+1) + m*(lmax+1) + l], kinds
// plm, dpdt, pdst, d2pdt2, dtpdst.
void oracle_legendre(int lmax, double theta, double* out) {
  Legendre a;
  computeLegendre(lmax, theta, a);
  int L = lmax + 1;
  for (int m = 0; m < 3; ++m)
    for (int l = 0; l <= lmax; ++l) {
      out[0 * 3 * L + m * L + l] = a.plm[m][l];
      out[1 * 3 * L + m * L + l] = a.dpdt[m][l];
      out[2 * 3 * L + m * L + l] = a.pdst[m][l];
      out[3 * 3 * L + m * L + l] = a.d2pdt2[m][l];
      out[4 * 3 * L + m * L + l] = a.dtpdst[m][l];
    }
}

// transformFrequencyTime of ntr spectra: spectrum t at sp + 2*t*ldsp (interleaved
// complex, element j is frequency j*df), series t at ts + t*nsamp.  Returns 0, 1
// (decimation warning) or 2 (error), the reference's levels.
int oracle_freq_time(int nf1, int nf2, double df, double sigma, int ntr, const double* sp, long long ldsp,
                     int nsamp, double dt, float* ts) {
  int warning = 0;
  std::vector<zc> z(nf2 + 1);
  for (int t = 0; t < ntr; ++t) {
    const double* s = sp + 2 * (long long)t * ldsp;
    for (int j = 1; j <= nf2; ++j) z[j] = zc{s[2 * (j - 1)], s[2 * (j - 1) + 1]};
    int rc = freqTime(nf1, nf2, df, sigma, z, nsamp, dt, ts + (long long)t * nsamp, &warning);
    if (rc) return rc;
  }
  return warning;
}

void oracle_fft(int n, int is, double* x, double* y) {
  int ng = 1 << n;
  std::vector<double> xx(ng + 1), yy(ng + 1);
  for (int i = 0; i < ng; ++i) { xx[i + 1] = x[i]; yy[i + 1] = y[i]; }
  fft(xx, yy, n, is);
  for (int i = 0; i < ng; ++i) { x[i] = xx[i + 1]; y[i] = yy[i + 1]; }
}

// Harmonic degree sums: hd[(sta*nf2 + jf-1)*14 + k] complex interleaved (jf in nf1..nf2)
// gr/gi: FP32 FK spectra of one node, Fortran (nkfmax, nsp) layout.
int oracle_degree_sums(int nf1, int nf2, const int* nwn, int nwnmax, int nkfmax, int nsp,
                       const float* gr, const float* gi, int nsta, const double* theta,
                       double* hd) {
  // offsets of the 10 moment FK spectra (greenFKSpectra.f90:204-212 with dsvmask U,V,W)
  auto offset = [](int comp, int jump) { return comp == 1 ? jump : (comp == 3 ? 4 + jump : 8 + jump); };
  for (int is = 0; is < nsta; ++is) {
    Legendre alf;
    computeLegendre(nwnmax - 1, theta[is], alf);
    int nwe = 0;
    for (int jf = nf1; jf <= nf2; ++jf) {
      int nwa = nwe + 1;
      nwe = nwe + nwn[jf - 1];
      std::vector<double> tap;
      taper(nwn[jf - 1] - 1, 0.2, tap);
      for (int k = 1; k <= 14; ++k) {
        int col = offset(MSUM[k - 1].comp, MSUM[k - 1].jump) - 1;
        if (col >= nsp) return 2;
        zc z = momentSum(k, gr + (size_t)col * nkfmax + (nwa - 1), gi + (size_t)col * nkfmax + (nwa - 1),
                         nwn[jf - 1], alf, tap);
        size_t o = (((size_t)is * nf2 + (jf - 1)) * 14 + (k - 1)) * 2;
        hd[o] = z.re; hd[o + 1] = z.im;
      }
    }
  }
  return 0;
}

// Force degree sums: hd[(sta*nf2 + jf-1)*7 + k] complex interleaved (5 force FK spectra U, V x 2 jumps, W).
int oracle_degree_sums_force(int nf1, int nf2, const int* nwn, int nwnmax, int nkfmax, int nsp,
                             const float* gr, const float* gi, int nsta, const double* theta, double* hd) {
  auto offset = [](int comp, int jump) { return comp == 1 ? jump : (comp == 3 ? 2 + jump : 4 + jump); };
  for (int is = 0; is < nsta; ++is) {
    Legendre alf;
    computeLegendre(nwnmax - 1, theta[is], alf);
    int nwe = 0;
    for (int jf = nf1; jf <= nf2; ++jf) {
      int nwa = nwe + 1;
      nwe = nwe + nwn[jf - 1];
      std::vector<double> tap;
      taper(nwn[jf - 1] - 1, 0.2, tap);
      for (int k = 1; k <= 7; ++k) {
        int col = offset(FSUM[k - 1].comp, FSUM[k - 1].jump) - 1;
        if (col >= nsp) return 2;
        zc z = forceSum(k, gr + (size_t)col * nkfmax + (nwa - 1), gi + (size_t)col * nkfmax + (nwa - 1),
                        nwn[jf - 1], alf, tap);
        size_t o = (((size_t)is * nf2 + (jf - 1)) * 7 + (k - 1)) * 2;
        hd[o] = z.re; hd[o + 1] = z.im;
      }
    }
  }
  return 0;
}

// Full phase 2 for moment tensor sources: traces[((sta*nmt + imt)*3 + comp)*nsamp + i]
// comp order Z, N, E.  filspecs = {nord_hp, fc_hp, nord_lp, fc_lp}.
}  // extern "C"

namespace {
// Per-station options of the station loop (computeSyntheticSeismograms.f90:344-397); a null
// member keeps the default: the common reduction time, all nsamp samples, the unit station
// filter, no source wavelet.
struct StationOpts {
  const double* tred = nullptr;      // [nsta] reduction time of each station
  const int* nstrue = nullptr;       // [nsta] samples kept (the rest are written as 0)
  const double* stafil = nullptr;    // [nsta][3][nf2] complex interleaved station filter
  int nstf = 0;                      // source wavelet samples
  double tanfstf = 0.0;              // time of the wavelet's first sample
  const float* stf = nullptr;
};

// convolveWithSourceWavelet (computeSyntheticSeismograms.f90:463-484): the sum runs in
// double and is stored to single precision after every term, as the reference's real f(k)
void convolveWavelet(int nd, int nstf, double tanf, double dt, const float* stf, float* urs) {
  const int nhm = (int)std::floor(std::fabs(tanf) / dt + 0.5);
  std::vector<float> f(nd);
  for (int k = 1; k <= nd; ++k) {
    float acc = 0.0f;
    const int n0 = std::max(1, k - nd + nhm + 1), n1 = std::min(k + nhm, nstf);
    for (int n = n0; n <= n1; ++n) {
      const int j = n - nhm;
      acc = (float)((double)acc + (dt * (double)urs[k - j]) * (double)stf[n - 1]);
    }
    f[k - 1] = acc;
  }
  for (int k = 0; k < nd; ++k) urs[k] = f[k];
}

// displacement spectra from the 14 sums or integrals hd, filters, rotation and
// inverse FFT of every station and moment tensor (computeSyntheticSeismograms.f90:336-397)
int synth_from_sums(int istyp, const std::vector<double>& hd, int nf1, int nf2, double df, double sigma, int nsta,
                    const double* phi, const double* propdir, int nmt, const double* mt, const double* filspecs,
                    int velocity, double tred_all, int nsamp, double dt, float* traces,
                    const StationOpts& o = StationOpts()) {
  const int nsum = istyp == 1 ? 14 : 7;
  int rc = 0;
  std::vector<zc> evf;
  eventFilter((int)std::lround(filspecs[0]), filspecs[1], (int)std::lround(filspecs[2]), filspecs[3],
              nf1, nf2, df, sigma, evf);
  const zc ci = Z(0.0, 1.0);
  for (int is = 0; is < nsta; ++is) {
    const double tred = o.tred ? o.tred[is] : tred_all;
    const int nd = o.nstrue ? o.nstrue[is] : nsamp;
    if (nd < 1 || nd > nsamp) return 2;
    double sphi = std::sin(phi[is]), cphi = std::cos(phi[is]);
    double s2phi = std::sin((double)2.0f * phi[is]), c2phi = std::cos((double)2.0f * phi[is]);
    double ca = std::cos(propdir[is]), sa = std::sin(propdir[is]);
    for (int im = 0; im < nmt; ++im) {
      const double* m = mt + im * (istyp == 1 ? 6 : 3);
      std::vector<zc> zsp[3];
      for (int c = 0; c < 3; ++c) zsp[c].assign(nf2 + 1, Z(0.0));
      for (int jf = nf1; jf <= nf2; ++jf) {
        const double* h = &hd[(((size_t)is * nf2 + (jf - 1)) * nsum) * 2];
        zc w[15];
        for (int k = 1; k <= nsum; ++k) w[k] = Z(h[(k - 1) * 2], h[(k - 1) * 2 + 1]);
        if (istyp == 1) {
          // momentSingleFrequencyDisplacement (singleFrequencyDisplacement.f90:108-125)
          double t1 = m[3] * cphi + m[4] * sphi;
          double t2 = (m[2] - m[1]) * c2phi - 2.0 * m[5] * s2phi;
          double t3 = m[4] * cphi - m[3] * sphi;
          double t4 = (m[2] - m[1]) * s2phi + 2.0 * m[5] * c2phi;
          zsp[0][jf] = w[1] * m[0] + w[2] * (m[1] + m[2]) + w[3] * t1 + w[4] * t2;
          zsp[1][jf] = w[5] * m[0] + w[6] * (m[1] + m[2]) + (w[7] + w[9]) * t1 + (w[8] + w[10]) * t2;
          zsp[2][jf] = (w[11] + w[13]) * t3 + (w[12] + w[14]) * t4;
        } else {
          // forceSingleFrequencyDisplacement (singleFrequencyDisplacement.f90:35-46)
          zsp[0][jf] = w[1] * m[0] + w[2] * (m[1] * cphi + m[2] * sphi);
          zsp[1][jf] = w[3] * m[0] + (w[4] + w[5]) * (m[1] * cphi + m[2] * sphi);
          zsp[2][jf] = (w[6] + w[7]) * (m[1] * sphi - m[2] * cphi);
        }
      }
      for (int jf = nf1; jf <= nf2; ++jf) {
        zc tsf = zexp(((ci * TWO_PI_F) * (double)(jf - 1)) * df * tred) * std::exp(sigma * tred);
        for (int c = 0; c < 3; ++c) {
          const zc sf = o.stafil ? Z(o.stafil[(((size_t)is * 3 + c) * nf2 + (jf - 1)) * 2],
                                     o.stafil[(((size_t)is * 3 + c) * nf2 + (jf - 1)) * 2 + 1])
                                 : Z(1.0, 0.0);
          zsp[c][jf] = ((zsp[c][jf] * evf[jf]) * sf) * tsf;
        }
      }
      for (int jf = nf1; jf <= nf2; ++jf) {
        if (velocity) {
          zc zom = Z(TWO_PI_F * (double)(jf - 1) * df, -sigma);
          for (int c = 0; c < 3; ++c) zsp[c][jf] = (zsp[c][jf] * ci) * zom;
        }
        zc ur = zsp[0][jf], ul = zsp[1][jf], ut = zsp[2][jf];
        zc ue = sa * ul + ca * ut;
        zc un = (-ca) * ul + sa * ut;
        zsp[0][jf] = ur; zsp[1][jf] = un; zsp[2][jf] = ue;
      }
      for (int c = 0; c < 3; ++c) {
        float* tr = traces + (((size_t)is * nmt + im) * 3 + c) * nsamp;
        rc = freqTime(nf1, nf2, df, sigma, zsp[c], nsamp, dt, tr);
        if (rc) return rc;
        if (o.nstf > 0) convolveWavelet(nd, o.nstf, o.tanfstf, dt, o.stf, tr);
        for (int k = nd; k < nsamp; ++k) tr[k] = 0.0f;
      }
    }
  }
  return 0;
}
}  // namespace

extern "C" {

// Synthetics of the global mode (harmonic degree sums at colatitudes theta).
int oracle_synthetics(int nf1, int nf2, const int* nwn, int nwnmax, double df, double sigma,
                      int nkfmax, int nsp, const float* gr, const float* gi, int nsta,
                      const double* theta, const double* phi, const double* propdir, int nmt,
                      const double* mt, const double* filspecs, int velocity, double tred,
                      int nsamp, double dt, float* traces) {
  std::vector<double> hd((size_t)nsta * nf2 * 14 * 2, 0.0);
  int rc = oracle_degree_sums(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, nsta, theta, hd.data());
  if (rc) return rc;
  return synth_from_sums(1, hd, nf1, nf2, df, sigma, nsta, phi, propdir, nmt, mt, filspecs, velocity, tred, nsamp, dt,
                         traces);
}

// Synthetics of either source type (istyp 1 moment tensors [nsrc][6], 0 forces
// [nsrc][3] as Fr, Ft, Ff) in either mode (global 1: degree sums at colatitudes
// theta; 0: wavenumber integrals at distances theta * rearth).
int oracle_synthetics_src(int istyp, int global, int nf1, int nf2, const int* nwn, int nwnmax, double df,
                          double sigma, double dwn, double rearth, int nkfmax, int nsp, const float* gr,
                          const float* gi, int nsta, const double* theta, const double* phi, const double* propdir,
                          int nsrc, const double* src, const double* filspecs, int velocity, double tred, int nsamp,
                          double dt, float* traces) {
  const int nsum = istyp == 1 ? 14 : 7;
  std::vector<double> hd((size_t)nsta * nf2 * nsum * 2, 0.0);
  int rc;
  if (global == 1) {
    rc = istyp == 1 ? oracle_degree_sums(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, nsta, theta, hd.data())
                    : oracle_degree_sums_force(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, nsta, theta, hd.data());
  } else {
    std::vector<double> x(nsta);
    for (int i = 0; i < nsta; ++i) x[i] = theta[i] * rearth;
    rc = oracle_wavenumber_integrals_src(istyp, nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, dwn, rearth, nsta,
                                         x.data(), hd.data());
  }
  if (rc) return rc;
  return synth_from_sums(istyp, hd, nf1, nf2, df, sigma, nsta, phi, propdir, nsrc, src, filspecs, velocity, tred,
                         nsamp, dt, traces);
}

// oracle_synthetics_src with the per-station options of the station loop: reduction time
// per station, samples kept per station, station filter, source wavelet (any may be null / 0).
int oracle_synthetics_opts(int istyp, int global, int nf1, int nf2, const int* nwn, int nwnmax, double df,
                           double sigma, double dwn, double rearth, int nkfmax, int nsp, const float* gr,
                           const float* gi, int nsta, const double* theta, const double* phi, const double* propdir,
                           int nsrc, const double* src, const double* filspecs, int velocity, double tred,
                           const double* tred_sta, const int* nstrue, const double* stafil, int nstf,
                           double tanfstf, const float* stf, int nsamp, double dt, float* traces) {
  const int nsum = istyp == 1 ? 14 : 7;
  std::vector<double> hd((size_t)nsta * nf2 * nsum * 2, 0.0);
  int rc;
  if (global == 1) {
    rc = istyp == 1 ? oracle_degree_sums(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, nsta, theta, hd.data())
                    : oracle_degree_sums_force(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, nsta, theta, hd.data());
  } else {
    std::vector<double> x(nsta);
    for (int i = 0; i < nsta; ++i) x[i] = theta[i] * rearth;
    rc = oracle_wavenumber_integrals_src(istyp, nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, dwn, rearth, nsta,
                                         x.data(), hd.data());
  }
  if (rc) return rc;
  StationOpts o;
  o.tred = tred_sta; o.nstrue = nstrue; o.stafil = stafil; o.nstf = nstf; o.tanfstf = tanfstf; o.stf = stf;
  if (nstf > 0 && !stf) return 2;
  return synth_from_sums(istyp, hd, nf1, nf2, df, sigma, nsta, phi, propdir, nsrc, src, filspecs, velocity, tred,
                         nsamp, dt, traces, o);
}

// Synthetics of the regional mode (wavenumber integrals at distances theta * rearth,
// besselDisplacementSpectra, displacementSpectra.f90:125-188).
int oracle_synthetics_bessel(int nf1, int nf2, const int* nwn, int nwnmax, double df, double sigma, double dwn,
                             double rearth, int nkfmax, int nsp, const float* gr, const float* gi, int nsta,
                             const double* theta, const double* phi, const double* propdir, int nmt,
                             const double* mt, const double* filspecs, int velocity, double tred, int nsamp,
                             double dt, float* traces) {
  std::vector<double> x(nsta);
  for (int i = 0; i < nsta; ++i) x[i] = theta[i] * rearth;
  std::vector<double> hd((size_t)nsta * nf2 * 14 * 2, 0.0);
  int rc = oracle_wavenumber_integrals(nf1, nf2, nwn, nwnmax, nkfmax, nsp, gr, gi, dwn, rearth, nsta, x.data(),
                                       hd.data());
  if (rc) return rc;
  return synth_from_sums(1, hd, nf1, nf2, df, sigma, nsta, phi, propdir, nmt, mt, filspecs, velocity, tred, nsamp, dt,
                         traces);
}


}  // extern "C"

// ---------------------------------------------------------------------------
//  SPECFEM coupling: displacement and traction at boundary points
//  (computeSyntheticsForSpecfemCoupling.f90:677-793), moment sources, from the
//  DSV spectra with radial derivatives (nsp = 20: U, V, dU/dr, dV/dr x 4 jumps,
//  W, dW/dr x 2 jumps, computeGreenFKSpectraForASKI.f90:516-541).
// ---------------------------------------------------------------------------
namespace {

// the 42 moment sums with derivatives (harmonicDegreeSums.f90:186-351, index map
// :34-45); kind: 0 plm, 1 dpdt, 2 pdst, 3 d2pdt2, 4 dtpdst
const SumDef DSUM[42] = {
    {0, 0, 0, 0.0, 1, 1},  {0, 0, 0, 0.0, 1, 2},  {0, 1, 1, 2.0, 1, 3},  {0, 2, 2, 2.0, 1, 4},
    {1, 0, 1, 0.0, 3, 1},  {1, 0, 1, 0.0, 3, 2},  {1, 1, 1, 2.0, 3, 3},  {1, 2, 2, 2.0, 3, 4},
    {2, 1, 1, 2.0, 7, 1},  {2, 2, 2, 4.0, 7, 2},  {1, 1, 1, 2.0, 7, 1},  {1, 2, 2, -2.0, 7, 2},
    {2, 1, 1, 2.0, 3, 3},  {2, 2, 2, -4.0, 3, 4},
    {0, 0, 0, 0.0, 5, 1},  {0, 0, 0, 0.0, 5, 2},  {0, 1, 1, 2.0, 5, 3},  {0, 2, 2, 2.0, 5, 4},
    {1, 0, 1, 0.0, 6, 1},  {1, 0, 1, 0.0, 6, 2},  {1, 1, 1, 2.0, 6, 3},  {1, 2, 2, 2.0, 6, 4},
    {2, 1, 1, 2.0, 9, 1},  {2, 2, 2, 4.0, 9, 2},  {1, 1, 1, 2.0, 9, 1},  {1, 2, 2, -2.0, 9, 2},
    {2, 1, 1, 2.0, 6, 3},  {2, 2, 2, -4.0, 6, 4},
    {1, 0, 1, 0.0, 1, 1},  {1, 0, 1, 0.0, 1, 2},  {1, 1, 1, 2.0, 1, 3},  {1, 2, 2, 2.0, 1, 4},
    {3, 0, 1, 0.0, 3, 1},  {3, 0, 1, 0.0, 3, 2},  {3, 1, 1, 2.0, 3, 3},  {3, 2, 2, 2.0, 3, 4},
    {4, 1, 1, 2.0, 7, 1},  {4, 2, 2, 4.0, 7, 2},  {3, 1, 1, 2.0, 7, 1},  {3, 2, 2, -2.0, 7, 2},
    {4, 1, 1, 2.0, 3, 3},  {4, 2, 2, -4.0, 3, 4}};

// the 21 force sums with derivatives (harmonicDegreeSums.f90:95-167, index map :34-37)
const SumDef DSUMF[21] = {
    {0, 0, 0, 0.0, 1, 1},  {0, 1, 1, -2.0, 1, 2}, {1, 0, 1, 0.0, 3, 1},  {1, 1, 1, -2.0, 3, 2},
    {2, 1, 1, -2.0, 7, 1}, {1, 1, 1, 2.0, 7, 1},  {2, 1, 1, 2.0, 3, 2},
    {0, 0, 0, 0.0, 5, 1},  {0, 1, 1, -2.0, 5, 2}, {1, 0, 1, 0.0, 6, 1},  {1, 1, 1, -2.0, 6, 2},
    {2, 1, 1, -2.0, 9, 1}, {1, 1, 1, 2.0, 9, 1},  {2, 1, 1, 2.0, 6, 2},
    {1, 0, 1, 0.0, 1, 1},  {1, 1, 1, -2.0, 1, 2}, {3, 0, 1, 0.0, 3, 1},  {3, 1, 1, -2.0, 3, 2},
    {4, 1, 1, -2.0, 7, 1}, {3, 1, 1, 2.0, 7, 1},  {4, 1, 1, 2.0, 3, 2}};

// column of (component, jump) in the force DSV spectra with derivatives
// (positionDataGreenFKSpectra, greenFKSpectra.f90:204-212: 2 spheroidal jumps, 1 toroidal)
int dsvColumnForce(int comp, int jump) {
  switch (comp) {
    case 1: return jump - 1;
    case 3: return 2 + jump - 1;
    case 5: return 4 + jump - 1;
    case 6: return 6 + jump - 1;
    case 7: return 8;
    default: return 9;
  }
}

zc derivSumForce(int kint, const float* gr, const float* gi, int nwn, const Legendre& alf,
                 const std::vector<double>& tap) {
  const SumDef& s = DSUMF[kint - 1];
  const std::vector<double>& T = s.kind == 0 ? alf.plm[s.m] : s.kind == 1 ? alf.dpdt[s.m] : s.kind == 2 ?
                                 alf.pdst[s.m] : s.kind == 3 ? alf.d2pdt2[s.m] : alf.dtpdst[s.m];
  const double fourpi = 4.0 * PI_F;
  zc z = Z(0.0);
  for (int l = s.l0; l <= nwn - 1; ++l) {
    zc g = Z((double)gr[l], (double)gi[l]);
    zc t;
    if (s.fnum == 0.0) t = T[l] * g;
    else t = (T[l] * (s.fnum / (double)(float)(l * (l + 1)))) * g;
    t = ((t * (2.0 * (double)l + 1.0)) / fourpi) * tap[l];
    z = z + t;
  }
  return z;
}

// column of (component, jump) in the DSV spectra with derivatives
int dsvColumn(int comp, int jump) {
  switch (comp) {
    case 1: return jump - 1;        // U
    case 3: return 4 + jump - 1;    // V
    case 5: return 8 + jump - 1;    // dU/dr
    case 6: return 12 + jump - 1;   // dV/dr
    case 7: return 16 + jump - 1;   // W
    default: return 18 + jump - 1;  // dW/dr
  }
}

zc derivSum(int kint, const float* gr, const float* gi, int nwn, const Legendre& alf,
            const std::vector<double>& tap) {
  const SumDef& s = DSUM[kint - 1];
  const std::vector<double>& T = s.kind == 0 ? alf.plm[s.m] : s.kind == 1 ? alf.dpdt[s.m] : s.kind == 2 ?
                                 alf.pdst[s.m] : s.kind == 3 ? alf.d2pdt2[s.m] : alf.dtpdst[s.m];
  const double fourpi = 4.0 * PI_F;
  zc z = Z(0.0);
  for (int l = s.l0; l <= nwn - 1; ++l) {
    zc g = Z((double)gr[l], (double)gi[l]);
    zc t;
    if (s.fnum == 0.0) t = T[l] * g;
    else t = ((T[l] * s.fnum) / (double)(float)(l * (l + 1))) * g;
    t = ((t * (2.0 * (double)l + 1.0)) / fourpi) * tap[l];
    z = z + t;
  }
  return z;
}

// rotations of complex vectors and tensors (axesRotation.f90:143-152,199-212,321-426,473-477)
void vecLCfromLS(double d, double x, const zc* u, zc* o) {
  double cd = std::cos(d), sd = std::sin(d), cx = std::cos(x), sx = std::sin(x);
  o[0] = ((sd * cx) * u[0] + (cd * cx) * u[1]) - sx * u[2];
  o[1] = ((sd * sx) * u[0] + (cd * sx) * u[1]) + cx * u[2];
  o[2] = cd * u[0] - sd * u[1];
}
void vecGCfromLC(double t, double p, const zc* u, zc* o) {
  double ct = std::cos(t), st = std::sin(t), cp = std::cos(p), sp = std::sin(p);
  o[0] = ((ct * cp) * u[0] - sp * u[1]) + (st * cp) * u[2];
  o[1] = ((ct * sp) * u[0] + cp * u[1]) + (st * sp) * u[2];
  o[2] = (-st) * u[0] + ct * u[2];
}
void vecLCfromGC(double t, double p, const zc* u, zc* o) {
  double ct = std::cos(t), st = std::sin(t), cp = std::cos(p), sp = std::sin(p);
  o[0] = ((ct * cp) * u[0] + (ct * sp) * u[1]) - st * u[2];
  o[1] = (-sp) * u[0] + cp * u[1];
  o[2] = ((st * cp) * u[0] + (st * sp) * u[1]) + ct * u[2];
}
// tensor rotation T' = R T R^T with the row rule v -> R v of a vector rotation
typedef void (*VecRot)(double, double, const zc*, zc*);
void tenRot(VecRot f, double a, double b, const zc t[3][3], zc o[3][3]) {
  zc tp[3][3];
  for (int j = 0; j < 3; ++j) {   // tp(:, j) = R t(:, j): rows combined column by column
    zc col[3] = {t[0][j], t[1][j], t[2][j]}, r[3];
    f(a, b, col, r);
    for (int i = 0; i < 3; ++i) tp[i][j] = r[i];
  }
  for (int i = 0; i < 3; ++i) {   // o(i, :) = R tp(i, :)
    zc row[3] = {tp[i][0], tp[i][1], tp[i][2]}, r[3];
    f(a, b, row, r);
    for (int j = 0; j < 3; ++j) o[i][j] = r[j];
  }
}
void vecLSrot(double d, double x, const zc* u, zc* o) { vecLCfromLS(d, x, u, o); }

}  // namespace

extern "C" {
// istyp 1: moment tensor mt[6] and DSV spectra of a moment (nsp >= 20, 42 sums);
// istyp 0: force mt[3] = (Fr, Ft, Ff) and those of a force (nsp >= 10, 21 sums).
// Per boundary point p (epicentral distance delta[p], azimuth xi[p] from south over
// east, outward normal nrm[3p..3p+2] in box coordinates) at radius re of the DSV node:
// the 42 degree sums, displacement and its derivatives, strain and stress
// (singleFrequencyDisplacement.f90:108-278 with zelcon of the node per frequency,
// zelcon[(jf-1)*14 + 2c + {0,1}]), rotation to the box (computeTension :677-705),
// traction = stress * n.  spectra != 0 (COMPUTE_SPECTRA): spec[((p*6 + c)*nf2 + jf-1)*2]
// holds displacement x,y,z then traction x,y,z, unfiltered.  Otherwise velocity and
// traction through the event filter and the time shift of tred, then the inverse FFT:
// traces[(p*6 + c)*nsamp + i].  dbg (nullable): the LS displacement, d/dr, (1/r)d/dtheta
// and (1/(r sin)) d/dphi at dbg[((p*nf2 + jf-1)*12 + 3q + c)*2].
int oracle_coupling(int istyp, int nf1, int nf2, const int* nwn, int nwnmax, int nkfmax, int nsp, const float* gr,
                    const float* gi, double df, double sigma, double re, const double* zelcon, const double* mt,
                    const double* filspecs, double tred, int nsamp, double dt, double thetas, double phis,
                    double thetac, double phic, int npts, const double* delta, const double* xi,
                    const double* nrm, int spectra, double* spec, float* traces, double* dbg) {
  if (nsp < (istyp == 1 ? 20 : 10)) return 2;
  const int nsum = istyp == 1 ? 42 : 21;
  std::vector<zc> evf;
  eventFilter((int)std::lround(filspecs[0]), filspecs[1], (int)std::lround(filspecs[2]), filspecs[3], nf1, nf2, df,
              sigma, evf);
  const zc ci = Z(0.0, 1.0);
  const double gam = 0.5 * PI_F;
  for (int ip = 0; ip < npts; ++ip) {
    Legendre alf;
    computeLegendre(nwnmax - 1, delta[ip], alf);
    const double phi = xi[ip], dl = delta[ip];
    const double sphi = std::sin(phi), cphi = std::cos(phi);
    const double s2phi = std::sin(2.0 * phi), c2phi = std::cos(2.0 * phi);
    std::vector<zc> out[6];
    for (int c = 0; c < 6; ++c) out[c].assign(nf2 + 1, Z(0.0));
    int nwe = 0;
    for (int jf = nf1; jf <= nf2; ++jf) {
      const int nwa = nwe + 1;
      nwe += nwn[jf - 1];
      std::vector<double> tap;
      taper(nwn[jf - 1] - 1, 0.2, tap);
      zc w[43];
      for (int k = 1; k <= nsum; ++k) {
        const SumDef& sd = istyp == 1 ? DSUM[k - 1] : DSUMF[k - 1];
        const int col = istyp == 1 ? dsvColumn(sd.comp, sd.jump) : dsvColumnForce(sd.comp, sd.jump);
        const float* a = gr + (size_t)col * nkfmax + (nwa - 1);
        const float* b = gi + (size_t)col * nkfmax + (nwa - 1);
        w[k] = istyp == 1 ? derivSum(k, a, b, nwn[jf - 1], alf, tap) : derivSumForce(k, a, b, nwn[jf - 1], alf, tap);
      }
      const double* m = mt;
      zc u[3], ur[3], ut[3], uf[3];
      const double rst = re * std::sin(dl);
      if (istyp == 0) {
        // force{,RadDeriv,ThetaDeriv,PhiDeriv}SingleFrequencyDisplacement (:35-103)
        const double fh = m[1] * cphi + m[2] * sphi, ft = m[1] * sphi - m[2] * cphi;
        const double fp = (-m[1]) * sphi + m[2] * cphi, fq = m[1] * cphi + m[2] * sphi;
        for (int q = 0; q < 3; ++q) {
          zc* v = q == 0 ? u : (q == 1 ? ur : ut);
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
      // momentSingleFrequencyDisplacement (:108-125)
      u[0] = w[1] * m[0] + w[2] * (m[1] + m[2]) + w[3] * t1 + w[4] * t2;
      u[1] = w[5] * m[0] + w[6] * (m[1] + m[2]) + (w[7] + w[9]) * t1 + (w[8] + w[10]) * t2;
      u[2] = (w[11] + w[13]) * t3 + (w[12] + w[14]) * t4;
      // momentRadDerivSingleFrequencyDisplacement (:130-148)
      ur[0] = w[15] * m[0] + w[16] * (m[1] + m[2]) + w[17] * t1 + w[18] * t2;
      ur[1] = w[19] * m[0] + w[20] * (m[1] + m[2]) + (w[21] + w[23]) * t1 + (w[22] + w[24]) * t2;
      ur[2] = (w[25] + w[27]) * t3 + (w[26] + w[28]) * t4;
      // momentThetaDerivSingleFrequencyDisplacement (:155-173)
      ut[0] = w[29] * m[0] + w[30] * (m[1] + m[2]) + w[31] * t1 + w[32] * t2;
      ut[1] = w[33] * m[0] + w[34] * (m[1] + m[2]) + (w[35] + w[37]) * t1 + (w[36] + w[38]) * t2;
      ut[2] = (w[39] + w[41]) * t3 + (w[40] + w[42]) * t4;
      for (int c = 0; c < 3; ++c) ut[c] = ut[c] / re;
      // momentPhiDerivSingleFrequencyDisplacement (:181-199)
      const double p1 = (-m[3]) * sphi + m[4] * cphi;
      const double p2 = (-2.0) * (m[2] - m[1]) * s2phi - 4.0 * m[5] * c2phi;
      const double p3 = (-m[4]) * sphi - m[3] * cphi;
      const double p4 = 2.0 * (m[2] - m[1]) * c2phi - 4.0 * m[5] * s2phi;
      uf[0] = w[3] * p1 + w[4] * p2;
      uf[1] = (w[7] + w[9]) * p1 + (w[8] + w[10]) * p2;
      uf[2] = (w[11] + w[13]) * p3 + (w[12] + w[14]) * p4;
      for (int c = 0; c < 3; ++c) uf[c] = uf[c] / rst;
      }
      if (dbg) {
        const zc* q[4] = {u, ur, ut, uf};
        for (int a = 0; a < 4; ++a)
          for (int c = 0; c < 3; ++c) {
            size_t o = ((((size_t)ip * nf2 + (jf - 1)) * 12) + 3 * a + c) * 2;
            dbg[o] = q[a][c].re; dbg[o + 1] = q[a][c].im;
          }
      }
      // sphericalStrainSingleFrequencyDisplacement (:229-244)
      const double rtd = re * std::tan(dl);
      zc e[3][3];
      e[0][0] = ur[0];
      e[1][1] = ut[1] + u[0] / re;
      e[2][2] = (uf[2] + u[0] / re) + u[1] / rtd;
      e[0][1] = 0.5 * ((ut[0] + ur[1]) - u[1] / re);
      e[0][2] = 0.5 * ((uf[0] + ur[2]) - u[2] / re);
      e[1][2] = 0.5 * ((uf[1] + ut[2]) - u[2] / rtd);
      e[2][1] = e[1][2]; e[2][0] = e[0][2]; e[1][0] = e[0][1];
      // sphericalStressSingleFrequencyDisplacement (:250-262)
      zc el[5];
      for (int c = 0; c < 5; ++c) el[c] = Z(zelcon[((size_t)(jf - 1) * 7 + c) * 2], zelcon[((size_t)(jf - 1) * 7 + c) * 2 + 1]);
      zc sg[3][3];
      sg[0][0] = el[1] * e[0][0] + el[2] * (e[1][1] + e[2][2]);
      sg[1][1] = (el[2] * e[0][0] + el[0] * (e[1][1] + e[2][2])) - (2.0 * el[4]) * e[2][2];
      sg[2][2] = (el[2] * e[0][0] + el[0] * (e[1][1] + e[2][2])) - (2.0 * el[4]) * e[1][1];
      sg[0][1] = (2.0 * el[3]) * e[0][1];
      sg[0][2] = (2.0 * el[3]) * e[0][2];
      sg[1][2] = (2.0 * el[4]) * e[1][2];
      sg[1][0] = sg[0][1]; sg[2][0] = sg[0][2]; sg[2][1] = sg[1][2];
      // computeTension (:677-705): epicentral LS -> LC -> global -> box LC -> box RC
      zc a[3], b[3];
      vecLCfromLS(dl, phi, u, a);
      vecGCfromLC(thetas, phis, a, b);
      vecLCfromGC(thetac, phic, b, a);
      vecLCfromGC(0.0, gam, a, b);
      zc ta[3][3], tb[3][3];
      tenRot(vecLSrot, dl, phi, sg, ta);
      tenRot(vecGCfromLC, thetas, phis, ta, tb);
      tenRot(vecLCfromGC, thetac, phic, tb, ta);
      tenRot(vecLCfromGC, 0.0, gam, ta, tb);
      const double* n = nrm + 3 * ip;
      zc tr[3];
      for (int i = 0; i < 3; ++i) tr[i] = ((Z(0.0) + tb[i][0] * n[0]) + tb[i][1] * n[1]) + tb[i][2] * n[2];
      if (!spectra) {
        const zc zom = Z(TWO_PI_F * (double)(jf - 1) * df, -sigma);
        const zc tsf = zexp(((ci * TWO_PI_F) * (double)(jf - 1)) * df * tred) * std::exp(sigma * tred);
        for (int c = 0; c < 3; ++c) {
          b[c] = (((b[c] * evf[jf]) * ci) * zom) * tsf;
          tr[c] = (tr[c] * evf[jf]) * tsf;
        }
      }
      for (int c = 0; c < 3; ++c) { out[c][jf] = b[c]; out[3 + c][jf] = tr[c]; }
    }
    for (int c = 0; c < 6; ++c) {
      if (spectra) {
        if (spec)
          for (int jf = 1; jf <= nf2; ++jf) {
            size_t o = (((size_t)ip * 6 + c) * nf2 + (jf - 1)) * 2;
            spec[o] = out[c][jf].re; spec[o + 1] = out[c][jf].im;
          }
      } else if (traces) {
        int rc = freqTime(nf1, nf2, df, sigma, out[c], nsamp, dt, traces + ((size_t)ip * 6 + c) * nsamp);
        if (rc) return rc;
      }
    }
  }
  return 0;
}

}  // extern "C"
