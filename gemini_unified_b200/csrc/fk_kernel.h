// Launch-level structures of the FK kernels (device pointers only).
#pragma once
#include <cstdint>

#include "gem_device.cuh"

namespace gem {

constexpr int FK_BLOCK = 256;          // threads per block of the solver
constexpr int MAX_LAYER_KNOTS = 64;    // knots per layer handled by the spline kernel

struct PrepArgs {
  int nslot, nk, nlay, attmode;
  double df, fref;
  const int* jf;        // [nslot] frequency index of each slot
  const double* ro;     // 1-based knot arrays [nk+1]
  const double* vpv;
  const double* vph;
  const double* vsv;
  const double* vsh;
  const double* eta;
  const double* qkinv;
  const double* qminv;
  const double* rk;
  const int* iktop;     // 1-based [nlay+1]
  const int* ikbot;
  double* spl;          // [nslot][nk+1][SPL_STRIDE]
};

struct FKLaunch {
  const double* spl;    // spline tables [nslot][nk+1][SPL_STRIDE]
  const int* jf;        // [nslot]
  const int* koff;      // [nslot] output index of (slot, iwn = 1)
  const int2* items;    // (slot, iwn), most expensive first
  int nitems;
  long long nkf;        // extent of the wavenumber-frequency index in the outputs
  double2* gf64;        // optional FP64 output (nkf, nsp, nnod)
  float* gfre;          // optional FP32 real part
  float* gfim;          // optional FP32 imaginary part
  int* status;          // optional per-k status
  double2* scratch;     // per-thread node storage, element-major
  long long nthreads;   // scratch stride
  unsigned int* queue;  // work-queue counter (zeroed before launch)
  unsigned long long* stats;   // 6 counters
};

struct FKStatic;
}  // namespace gem

#include <cuda_runtime.h>
namespace gem {
cudaError_t launch_prep(const PrepArgs& A, int* d_err, cudaStream_t st);
cudaError_t launch_fk(const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st);
int fk_blocks_per_sm();
}  // namespace gem
