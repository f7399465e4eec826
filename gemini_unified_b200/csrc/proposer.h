// Learned step/order proposer: shapes, launch arguments and launchers.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "gem_device.cuh"

namespace gem {

constexpr int PROP_NF = 11;   // features
constexpr int PROP_H = 64;    // width of the hidden layers
constexpr int PROP_NO = 3;    // outputs: log work ratio at attempt 5, at attempt 7, log initial-step factor
constexpr int PROP_NPARAM = PROP_H * PROP_NF + PROP_H + PROP_H * PROP_H + PROP_H + PROP_NO * PROP_H + PROP_NO;
constexpr int PROP_NNORM = 2 * PROP_NF;   // feature mean and deviation
constexpr float PROP_HS_CLIP = 1.4f;      // |log initial-step factor| <= 1.4 (factor 0.25 .. 4)
constexpr int PROP_USE_ORDER = 1;         // apply the proposed order target
constexpr int PROP_USE_STEP = 2;          // apply the proposed initial-step factor

struct PropArgs {
  const int2* items;      // (slot, iwn) of each item k
  const int* jf;          // frequency index of each slot
  const double* rstart;   // [2][nkf] start radii (toroidal, spheroidal)
  long long nkf;
  int nitems, nk, nlay, use;
  float margin;           // least predicted saving (log work ratio) that moves the order target off 6
  double df, rearth;
  double rk[MAXKNOT + 1];   // knot radii, 1-based
  double rb[MAXLAY + 1];    // layer tops, 1-based
  float knot_feat[3 * (MAXKNOT + 1)];   // vp, vs, rho / 1e4 at each knot
};

cudaError_t prop_features_launch(const PropArgs& A, float* out, cudaStream_t st);
cudaError_t prop_infer_launch(const PropArgs& A, const __half* w, const float* norm, signed char* kopt, float* hs,
                              cudaStream_t st);

}  // namespace gem
