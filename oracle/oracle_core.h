// =============================================================================
//  GEMINI FK hot path -- CPU FP64 ORACLE (test infrastructure only).
//
//  This is a plain C++ restatement of the reference Fortran algorithm
//  (seismology-RUB/GEMINI_UNIFIED), written to check the CUDA product path.
//  Only the test suite, the smoke check and the CPU-baseline leg of the bench
//  may load it.  Nothing in the product library links or calls it.
//
//  Parity status: the reference cannot be compiled in this environment (no
//  Fortran compiler, MPI or HDF5), so FK spectra and seismograms are
//  "parity unpinned" against the reference binary.  The model reader is
//  pinned by the reference's own known-answer test
//  (f90/testReadNodeEarthmodel.f90:55-80) through the Python JSON loader.
//
//  Numeric conventions follow gfortran -O3 on x86-64 (no FMA contraction):
//    * complex*complex = (ar*br - ai*bi, ar*bi + ai*br)
//    * complex/complex by Smith's method (GCC's -fcx-fortran-rules lowering)
//    * real (op) complex acts component-wise on the complex operand
//    * default-REAL literals (e.g. 0.8, 0.1, pi) are rounded to float first
//  Compile with -ffp-contract=off.
// =============================================================================
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- complex ---
struct zc {
  double re, im;
};
static inline zc Z(double r, double i = 0.0) { return zc{r, i}; }
static inline zc operator+(zc a, zc b) { return {a.re + b.re, a.im + b.im}; }
static inline zc operator-(zc a, zc b) { return {a.re - b.re, a.im - b.im}; }
static inline zc operator-(zc a) { return {-a.re, -a.im}; }
static inline zc operator*(zc a, zc b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
static inline zc operator*(double a, zc b) { return {a * b.re, a * b.im}; }
static inline zc operator*(zc a, double b) { return {a.re * b, a.im * b}; }
static inline zc operator/(zc a, double b) { return {a.re / b, a.im / b}; }
static inline zc operator+(double a, zc b) { return {a + b.re, b.im}; }
static inline zc operator+(zc a, double b) { return {a.re + b, a.im}; }
static inline zc operator-(double a, zc b) { return {a - b.re, -b.im}; }
static inline zc operator-(zc a, double b) { return {a.re - b, a.im}; }
// Smith's algorithm as lowered by GCC for Fortran complex division.
static inline zc operator/(zc a, zc b) {
  double ar = a.re, ai = a.im, br = b.re, bi = b.im;
  if (std::fabs(br) < std::fabs(bi)) {
    double ratio = br / bi;
    double div = (br * ratio) + bi;
    double tr = (ar * ratio) + ai;
    double ti = (ai * ratio) - ar;
    return {tr / div, ti / div};
  } else {
    double ratio = bi / br;
    double div = (bi * ratio) + br;
    double tr = (ai * ratio) + ar;
    double ti = ai - (ar * ratio);
    return {tr / div, ti / div};
  }
}
static inline zc operator/(double a, zc b) { return zc{a, 0.0} / b; }
static inline double zabs(zc a) { return std::hypot(a.re, a.im); }
static inline zc zsqrt(zc a) {
  std::complex<double> s = std::sqrt(std::complex<double>(a.re, a.im));
  return {s.real(), s.imag()};
}
static inline zc zexp(zc a) {
  std::complex<double> s = std::exp(std::complex<double>(a.re, a.im));
  return {s.real(), s.imag()};
}

// ------------------------------------------------------------- constants ---
// mathConstants.f90:28,34 -- pi literals are default REAL: pi rounded to float.
static const double PI_F = (double)(float)3.141592653589793;
static const double TWO_PI_F = 2.0 * PI_F;
static const double EPS_D = 2.220446049250313e-16;  // epsilon(1.d0)
static const double EPS_F = (double)1.1920928955078125e-07;  // epsilon(1.0)
static const double TINY_D = 2.2250738585072014e-308;  // tiny(1.d0)

// parametersBulirschStep.f90:28-48
static const double GROW_BS = 1.25;
static const double SHRINK_BS = (double)(float)0.8;
static const int MAXTRY_BS = 7, MINTRY_BS = 3, OPTTRY_BS = 6, KGV_BS = 48;
static const int SEQDIV_BS[7] = {2, 4, 6, 8, 12, 16, 24};
static const int NXDIV_BS[7] = {3, 2, 4, 4, 4, 8, 8};
static const int IXDIV_BS[7][8] = {
    {0, 24, 48, 0, 0, 0, 0, 0},     {12, 36, 0, 0, 0, 0, 0, 0},
    {8, 16, 32, 40, 0, 0, 0, 0},    {6, 18, 30, 42, 0, 0, 0, 0},
    {4, 20, 28, 44, 0, 0, 0, 0},    {3, 9, 15, 21, 27, 33, 39, 45},
    {2, 10, 14, 22, 26, 34, 38, 46}};
// integrationStep.f90:35-36
static const double MINSIZE_IS = 1.0e-12;
static const int MAXNUM_IS = 200000;
// propagateOde.f90:54
static const double MAXY_PROP = 1.0e10;

// ------------------------------------------------------------ statistics ---
struct Stats {
  int64_t steps_ok = 0;      // accepted BS steps
  int64_t steps_rej = 0;     // rejected BS steps
  int64_t attempts = 0;      // modified-midpoint attempts
  int64_t sysmats = 0;       // system-matrix evaluations
  int64_t matvecs = 0;       // nvar x nvar matrix-vector products
  int64_t flops = 0;         // algorithmic flop count (see flop weights)
  void add(const Stats& o) {
    steps_ok += o.steps_ok; steps_rej += o.steps_rej; attempts += o.attempts;
    sysmats += o.sysmats; matvecs += o.matvecs; flops += o.flops;
  }
};

}  // namespace orc
