// Launch-level structure of the synthetics kernels (device pointers only).
#pragma once
#include "../../include/gemini_fk.h"
#include "gem_device.cuh"

namespace gem {

struct SynthDev {
  int nf1, nf2, nsta, nmt, lmax, lcap, ns, nslog, nsamp, ndec, velocity;
  long long nkf;
  double df, sigma, tred;
  int nsk[8];               // sums per Legendre table kind
  long long aoff[8], coff[8];   // offsets of each kind's coefficient and result matrices
  int col_off[10];          // FK column of each (component, jump) spectrum
  const int* nwn;           // [nf2]
  const int* koff;          // [nf] first index of each frequency in the FK slab
};

__device__ __forceinline__ dz zexp_dev(dz z) {
  double e = exp(z.re);
  return dz{e * cos(z.im), e * sin(z.im)};
}

}  // namespace gem

// error / timing hooks of the context (defined with gem_ctx)
int gem_set_error(gem_ctx* ctx, const char* msg);
void gem_note_synth_ms(gem_ctx* ctx, float ms);
