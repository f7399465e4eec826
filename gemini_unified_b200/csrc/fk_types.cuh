// Data structures shared by the FK solver kernel and its host launcher.
#pragma once
#include "gem_device.cuh"

namespace gem {

// ------------------------------------------------------------------------
//  Parameter block (passed by value to the kernel)
// ------------------------------------------------------------------------
struct FKStatic {
  int nlay, nk, noc, nic, equidis, fsflag, nnod, jre;
  int hascore, hasocean, istyp, stressflag, global_, nsp;
  int ncsph, nctor, njsph, njtor, dsvstep;
  double rearth, ric, roc, rhs, ruc, eps, sigma, df, dwn;
  int kopt;   // attempt the step-size control aims at (opttry, parametersBulirschStep.f90:28-48: 6)
  int dsv;    // 1: DSV spectra with radial derivatives of a source at node jre (no reciprocity)
  int jsl, jsr;   // node range of the minors (spheroidalMinors.f90:72-585): jre..jre, or a set of source nodes
  double rb[MAXLAY + 1];
  double drk[MAXLAY + 1];
  int iflso[MAXLAY + 1];
  int iktop[MAXLAY + 1];
  double rk[MAXKNOT + 1];
  double rnod[MAXNOD + 1];
  int state[MAXNOD + 1];
  int layer[MAXNOD + 1];
};

struct Counters {
  long long steps_ok, steps_rej, attempts, sysmats, matvecs, flops;
  long long warp_attempts, lane_attempts;   // lockstep utilisation (instrumentation)
};

// knot and layer tables used at every spline evaluation, copied to shared
// memory (lanes index them divergently)
struct Tab {
  double rk[MAXKNOT + 1];
  double drk[MAXLAY + 1];
  double rdrk[MAXLAY + 1];   // 1/drk (fast variant)
  int iktop[MAXLAY + 1];
};

constexpr int POLY_STRIDE = 64;   // doubles per knot interval in the polynomial table

struct Env {
  const Tab* tab;                   // shared-memory copy of the knot tables
  const double* __restrict__ spl;   // spline table of this frequency, [knot][SPL_STRIDE]
  const double* __restrict__ poly;  // cubic coefficients per knot interval (fast variant), [knot][POLY_STRIDE]
  int nl;
  double omre, omim, dll1;
};

// per-thread scratch slot: element e of this thread at base[e * stride]
struct Slot {
  double2* base;
  long long stride;
  __device__ __forceinline__ dz get(int e) const {
    double2 v = base[(long long)e * stride];
    return dz{v.x, v.y};
  }
  __device__ __forceinline__ void put(int e, dz v) const { base[(long long)e * stride] = make_double2(v.re, v.im); }
};

// scratch element offsets for NN = nnod + 1 (1-based node index n)
struct Layout {
  int NN;
  __device__ __forceinline__ int ut(int n, int c) const { return n * 2 + c; }
  __device__ __forceinline__ int dt(int n, int c) const { return 2 * NN + n * 2 + c; }
  __device__ __forceinline__ int um(int n, int c) const { return 4 * NN + n * 6 + c; }
  __device__ __forceinline__ int dm(int n, int c) const { return 10 * NN + n * 6 + c; }
  __device__ __forceinline__ int sph(int n, int j, int c) const { return 16 * NN + n * 16 + j * 4 + c; }
  __device__ __forceinline__ int tor(int n, int j, int c) const { return 32 * NN + n * 4 + j * 2 + c; }
  __device__ __forceinline__ int ulg(int n) const { return 36 * NN + n; }
  __device__ __forceinline__ int dlg(int n) const { return 37 * NN + n; }
  __device__ __forceinline__ int adjic(int n, int c) const { return 38 * NN + n * 4 + c; }
  static constexpr int PER_NODE = 42;
};

}  // namespace gem
