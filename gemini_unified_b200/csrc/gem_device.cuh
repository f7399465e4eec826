// Device-side complex arithmetic and shared constants of the FK solver.
//
// Complex operations follow the Fortran semantics the reference is built with
// (gfortran, x86-64): complex*complex = (ar*br - ai*bi, ar*bi + ai*br); complex
// division by Smith's method; a real operand acts component-wise.  Built with
// --fmad=false the kernel repeats the reference's rounding step by step.
#pragma once
#include <cstdint>

namespace gem {

struct dz {
  double re, im;
};

__host__ __device__ __forceinline__ dz mk(double r, double i = 0.0) { return dz{r, i}; }
__host__ __device__ __forceinline__ dz operator+(dz a, dz b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ dz operator-(dz a, dz b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ dz operator-(dz a) { return {-a.re, -a.im}; }
__host__ __device__ __forceinline__ dz operator*(dz a, dz b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ dz operator*(double a, dz b) { return {a * b.re, a * b.im}; }
__host__ __device__ __forceinline__ dz operator*(dz a, double b) { return {a.re * b, a.im * b}; }
__host__ __device__ __forceinline__ dz operator/(dz a, double b) { return {a.re / b, a.im / b}; }
__host__ __device__ __forceinline__ dz operator+(double a, dz b) { return {a + b.re, b.im}; }
__host__ __device__ __forceinline__ dz operator+(dz a, double b) { return {a.re + b, a.im}; }
__host__ __device__ __forceinline__ dz operator-(double a, dz b) { return {a - b.re, -b.im}; }
__host__ __device__ __forceinline__ dz operator-(dz a, double b) { return {a.re - b, a.im}; }
__host__ __device__ __forceinline__ dz operator/(dz a, dz b) {
  double ar = a.re, ai = a.im, br = b.re, bi = b.im;
  if (fabs(br) < fabs(bi)) {
    double ratio = br / bi;
    double div = (br * ratio) + bi;
    return {((ar * ratio) + ai) / div, ((ai * ratio) - ar) / div};
  } else {
    double ratio = bi / br;
    double div = (bi * ratio) + br;
    return {((ai * ratio) + ar) / div, (ai - (ar * ratio)) / div};
  }
}
__host__ __device__ __forceinline__ dz operator/(double a, dz b) { return dz{a, 0.0} / b; }
__device__ __forceinline__ double zabs(dz a) { return hypot(a.re, a.im); }
// 1/z = conj(z) / |z|^2 (one reciprocal; used by the fast variant only)
__device__ __forceinline__ dz zinv_fast(dz z) {
  double r = __drcp_rn(z.re * z.re + z.im * z.im);
  return {z.re * r, -z.im * r};
}

// principal square root (Kahan's formulation, branch cut on the negative axis)
__device__ __forceinline__ dz zsqrt(dz z) {
  double x = z.re, y = z.im;
  if (x == 0.0 && y == 0.0) return {0.0, y};
  double t = sqrt((fabs(x) + hypot(x, y)) * 0.5);
  if (x >= 0.0) return {t, y / (2.0 * t)};
  return {fabs(y) / (2.0 * t), copysign(t, y)};
}

// pi as the reference spells it: a default-REAL literal (mathConstants.f90:34)
constexpr double PI_F = 3.1415927410125732;
constexpr double TWO_PI_F = 2.0 * PI_F;
constexpr double EPS_D = 2.220446049250313e-16;
constexpr double EPS_F = 1.1920928955078125e-07;
constexpr double TINY_D = 2.2250738585072014e-308;
constexpr double SHRINK_BS = 0.800000011920928955078125;   // REAL literal 0.8
constexpr double GROW_BS = 1.25;
constexpr double TENTH_F = 0.100000001490116119384765625;  // REAL literal 0.1
constexpr double ONE_EM6_F = 9.999999974752427e-07;        // REAL literal 1.e-6
constexpr double MINSIZE_IS = 1.0e-12;
constexpr int MAXNUM_IS = 200000;
constexpr double MAXY_PROP = 1.0e10;


// Limits of the fixed-size parameter block
constexpr int MAXLAY = 32;
constexpr int MAXKNOT = 256;
constexpr int MAXNOD = 96;
constexpr int SPL_STRIDE = 32;   // doubles per knot in the spline table

// Item status codes (C-ABI contract)
enum : int {
  ST_OK = 0,
  ST_MINSTEP = 1,      // step size below minimum (integrationStep.f90:176-180)
  ST_MAXSTEPS = 2,     // maximum number of steps (integrationStep.f90:186)
  ST_CF = 3,           // continued fraction did not converge (initialValues.f90:490-574)
  ST_BOOKKEEPING = 4,  // node / discontinuity bookkeeping (propagateOde.f90:177-186,319-324)
  ST_NONFINITE = 5,
  ST_UNSUPPORTED = 7,  // receiver or source in an ocean layer
};


}  // namespace gem
