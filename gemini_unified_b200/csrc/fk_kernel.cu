// FK spectra on the GPU: model preparation (complex elastic constants and
// natural cubic splines per frequency) and the persistent (omega, l) solver.
//
// Reference: computeGreenFKSpectraForSynthetics.f90:380-501 (frequency and
// wavenumber loops), toroidalMinors.f90, spheroidalMinors.f90,
// unitJumpGreenFunctions.f90, reciprocity.f90, sourceTerms.f90.
#include <cuda_runtime.h>

#include "fk_kernel.h"
#include "fk_types.cuh"

namespace gem {

// =========================================================================
//  K3: model preparation (nodeEarthmodel.f90:287-330,
//  complexElasticConstants.f90:48-106, cubicSpline.f90:74-109,176-221)
// =========================================================================
__global__ void knots_kernel(PrepArgs A) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int nk = A.nk;
  if (idx >= A.nslot * nk) return;
  int slot = idx / nk, k = idx % nk + 1;   // 1-based knot
  double f = (double)(A.jf[slot] - 1) * A.df;
  double fratio, qk, qm;
  switch (A.attmode) {
    case 0: fratio = 1.0; qk = 0.0; qm = 0.0; break;
    case 1: fratio = 1.0; qk = A.qkinv[k]; qm = A.qminv[k]; break;
    case 2: fratio = f / A.fref; qk = 0.0; qm = 0.0; break;
    default: fratio = f / A.fref; qk = A.qkinv[k]; qm = A.qminv[k]; break;
  }
  double ro = A.ro[k], alfv = A.vpv[k], alfh = A.vph[k], betv = A.vsv[k], beth = A.vsh[k], eta = A.eta[k];
  double phik = atan(qk), phim = atan(qm);
  dz zqk = dz{cos(phik), sin(phik)} * pow(fratio, 2.0 * phik / PI_F);
  dz zqm = dz{cos(phim), sin(phim)} * pow(fratio, 2.0 * phim / PI_F);
  dz z[7];
  if (betv > ONE_EM6_F) {
    double epa = ro * alfh * alfh, epc = ro * alfv * alfv;
    double epn = ro * beth * beth, epl = ro * betv * betv;
    double epf = eta * (epa - 2.0 * epl);
    double kappa = (epc + 4.0 * epa - 4.0 * epn + 4.0 * epf) / 9.0;
    double mue = (epc + epa + 6.0 * epl + 5.0 * epn - 2.0 * epf) / 15.0;
    double lamp2mue = kappa + 4.0 * mue / 3.0;
    double lambda = kappa - 2.0 * mue / 3.0;
    dz zkap = kappa * zqk, zmue = mue * zqm;
    dz zl2m = zkap + (4.0 * zmue) / 3.0;
    dz zlam = zkap - (2.0 * zmue) / 3.0;
    z[0] = zl2m + (epa - lamp2mue); z[1] = zl2m + (epc - lamp2mue); z[2] = zlam + (epf - lambda);
    z[3] = zmue + (epl - mue); z[4] = zmue + (epn - mue); z[5] = zkap; z[6] = zmue;
  } else {
    double kappa = ro * alfv * alfv;
    dz zkap = kappa * zqk;
    z[0] = zkap; z[1] = zkap; z[2] = zkap; z[3] = dz{0, 0}; z[4] = dz{0, 0}; z[5] = zkap; z[6] = dz{0, 0};
  }
  double* t = A.spl + ((long long)slot * (nk + 1) + k) * SPL_STRIDE;
  t[0] = ro;
  for (int c = 0; c < 7; ++c) { t[2 + 2 * c] = z[c].re; t[3 + 2 * c] = z[c].im; }
}

// LAPACK dgtsv (NRHS = 1) on 1-based local arrays
__device__ int dgtsv1(int n, double* dl, double* d, double* du, double* b) {
  for (int i = 1; i <= n - 2; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] == 0.0) return i;
      double fact = dl[i] / d[i];
      d[i + 1] = d[i + 1] - fact * du[i];
      b[i + 1] = b[i + 1] - fact * b[i];
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
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] == 0.0) return i;
      double fact = dl[i] / d[i];
      d[i + 1] = d[i + 1] - fact * du[i];
      b[i + 1] = b[i + 1] - fact * b[i];
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

// one thread per (frequency slot, layer >= 2, series); series 0 = density,
// 1..14 = real/imaginary part of the 7 constants.  Layer 1 is not splined.
__global__ void spline_kernel(PrepArgs A, int* err) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int nl_count = A.nlay - 1;
  if (idx >= A.nslot * nl_count * 15) return;
  int series = idx % 15;
  int nl = (idx / 15) % nl_count + 2;
  int slot = idx / (15 * nl_count);
  int j1 = A.ikbot[nl], j2 = A.iktop[nl], n = j2 - j1 + 1;
  if (n > MAX_LAYER_KNOTS) { atomicExch(err, 1); return; }
  double* base = A.spl + (long long)slot * (A.nk + 1) * SPL_STRIDE;
  int cin = series == 0 ? 0 : 2 + (series - 1);
  int cout = series == 0 ? 1 : 16 + (series - 1);
  double x[MAX_LAYER_KNOTS + 2], y[MAX_LAYER_KNOTS + 2];
  double dl[MAX_LAYER_KNOTS + 2], d[MAX_LAYER_KNOTS + 2], du[MAX_LAYER_KNOTS + 2], y2[MAX_LAYER_KNOTS + 2];
  for (int i = 1; i <= n; ++i) {
    x[i] = A.rk[j1 - 1 + i];
    y[i] = base[(j1 - 1 + i) * SPL_STRIDE + cin];
    dl[i] = 0.0; d[i] = 0.0; du[i] = 0.0; y2[i] = 0.0;
  }
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
  if (dgtsv1(n, dl, d, du, y2)) { atomicExch(err, 2); return; }
  // imaginary part of zy2 is formed as 0 + 1*y2 (cubicSpline.f90:215-217), the real part as y2
  for (int i = 1; i <= n; ++i) base[(j1 - 1 + i) * SPL_STRIDE + cout] = y2[i];
}


// cubic coefficients per knot interval in t = r - rk(j) (fast variant): from
// y = a y1 + b y2 + cc s1 + dd s2 with b = t/h, a = 1 - b,
// cc = h^2 a (a^2 - 1)/6, dd = h^2 b (b^2 - 1)/6 (splineEarthmodelCoefficients.f90:143-160).
// Layer 1 (homogeneous) keeps the constant of knot iktop(1) in c0.
__global__ void poly_kernel(PrepArgs A, double* poly) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  int nk = A.nk;
  if (idx >= A.nslot * nk) return;
  int slot = idx / nk, j = idx % nk + 1;   // interval [rk(j), rk(j+1)]
  const double* base = A.spl + (long long)slot * (nk + 1) * SPL_STRIDE;
  double* q = poly + ((long long)slot * (nk + 1) + j) * POLY_STRIDE;
  // interval inside a layer: ikbot(nl) <= j < iktop(nl) for some layer nl >= 2;
  // otherwise (homogeneous layer 1, the top knot of a layer) the value is constant
  bool inside = false;
  for (int nl = 2; nl <= A.nlay; ++nl) inside |= (j >= A.ikbot[nl] && j < A.iktop[nl]);
  const bool last = !inside;
  double h = last ? 1.0 : A.rk[j + 1] - A.rk[j];
  for (int v = 0; v < 15; ++v) {
    int ci = v == 0 ? 0 : 2 + (v - 1);
    int c2i = v == 0 ? 1 : 16 + (v - 1);
    double y1 = base[j * SPL_STRIDE + ci];
    double s1 = base[j * SPL_STRIDE + c2i];
    double c0 = y1, c1 = 0, c2 = 0, c3 = 0;
    if (!last) {
      double y2 = base[(j + 1) * SPL_STRIDE + ci];
      double s2 = base[(j + 1) * SPL_STRIDE + c2i];
      c1 = ((y2 - y1) - h * h * (2.0 * s1 + s2) / 6.0) / h;
      c2 = 0.5 * s1;
      c3 = (s2 - s1) / (6.0 * h);
    }
    q[4 * v + 0] = c3; q[4 * v + 1] = c2; q[4 * v + 2] = c1; q[4 * v + 3] = c0;
  }
}

cudaError_t launch_prep(const PrepArgs& A, int* d_err, cudaStream_t st) {
  int n1 = A.nslot * A.nk;
  knots_kernel<<<(n1 + 127) / 128, 128, 0, st>>>(A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  int n2 = A.nslot * (A.nlay - 1) * 15;
  if (n2 > 0) spline_kernel<<<(n2 + 63) / 64, 64, 0, st>>>(A, d_err);
  return cudaGetLastError();
}

cudaError_t launch_poly(const PrepArgs& A, double* poly, cudaStream_t st) {
  int n = A.nslot * A.nk;
  poly_kernel<<<(n + 127) / 128, 128, 0, st>>>(A, poly);
  return cudaGetLastError();
}

}  // namespace gem
