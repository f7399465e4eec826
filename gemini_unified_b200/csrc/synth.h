// Launch-level structure of the synthetics kernels (device pointers only).
#pragma once
#include <vector>
#include "../../include/gemini_fk.h"
#include "gem_device.cuh"

namespace gem {

struct SynthDev {
  int nf1, nf2, nsta, nmt, lmax, lcap, ns, nslog, nsamp, ndec, velocity;
  long long nkf;
  long long ldx;            // complex elements between consecutive spectra of the FFT input
  double df, sigma, tred;
  double dwn, rearth;       // regional mode: wavenumber spacing, earth radius
  int istyp, nsum;          // source type (0 force, 1 moment tensor) and its number of sums
  const double* tred_sta;   // [nsta] reduction time per station, or null: tred
  const double2* stafil;    // [nsta][3][nf2] station filter per component, or null: unit filter
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

namespace gem {

// Length and decimation of the inverse FFT (frequencyTime.f90:65-84).
struct FftGeometry {
  int ns, nslog, ndec;
  double dts;
  bool decimated;   // the reference's warning 'Downsampling to less than 1./(2*fny) requested'
};
// Fills g; returns nullptr or the reason the sizes are rejected.
const char* fft_geometry(int nf1, int nf2, double df, int nsamp, double dt, FftGeometry& g);
constexpr int IFFT_MAX_NS = 8192;   // one series in shared memory: 8192 * 16 B
constexpr int IFFT_THREADS = 512;

// twiddles of the radix-2 stages (fourierTransform.f90:139-147) and
// fac[i] = expo^i by the reference's sequential product (frequencyTime.f90:105-110)
__global__ void ifft_tables_kernel(int ns, int nslog, int nsamp, double expo, double2* tw, double* fac);
__global__ void __launch_bounds__(512) ifft_kernel(SynthDev S, const double2* __restrict__ X, const double2* __restrict__ tw,
                            const double* __restrict__ fac, float* traces);
inline size_t ifft_table_bytes(int ns, int nsamp) { return (size_t)ns * sizeof(double2) + (size_t)nsamp * sizeof(double); }

// fast-form inverse FFT (ifft_fast.cu): real output from a half-length radix-16
// transform; ns in 512..8192; tw: ns + IFFT_TW_EXTRA entries, e^{2 pi i m/ns} for
// m < ns followed by the tables of the radix-16 passes (IFFT_TWA, IFFT_TWB)
constexpr int IFFT_TWA = 0, IFFT_TWB = 256, IFFT_TW_EXTRA = 4096;
inline size_t ifft_fast_twiddle_bytes(int ns) { return ((size_t)ns + IFFT_TW_EXTRA) * sizeof(double2); }
cudaError_t ifft_fast_launch(const SynthDev& S, long long ntr, const double2* X, const double2* tw, const double* fac,
                             float* traces, cudaStream_t st);
cudaError_t ifft_fast_twiddles_launch(int N, double2* tw, cudaStream_t st);
inline bool ifft_fast_supported(int ns) { return ns >= 512 && ns <= IFFT_MAX_NS; }

// fast-form Legendre tables (legendre_fast.cu): the tables of legendre_kernel with
// the recurrence's division replaced by a reciprocal table; lmax up to 25,599
bool legendre_fast_supported(int lmax);
cudaError_t legendre_fast_launch(int nsta, int lmax, int lcap, const double* theta, double* tab, cudaStream_t st);

// event filter of the synthetics (Butterworth band-pass at f - i sigma/2pi), h[jf] for jf = nf1..nf2
void event_filter_host(const gem_synth_params* p, std::vector<double2>& h);

// sliced-integer tensor-core degree sums (sums_tc.cu).  One product per table
// kind: C[coff[kind] + row * ncol + col] = sum_l A[row][l] T[kind][l][col] for the
// 2 * nf * nsk[kind] rows of the kind (frequency slot slowest, then sum rank, then
// re/im; the rows of all kinds contiguous in A with leading dimension lcap), and
// T[kind][l][col] = tab[(kind * lcap + l) * ncol + col].
constexpr int TC_MAX_KIND = 16;
struct TcProblem {
  int nkind, ncol, lcap, lmax, nf1, nf2;
  int nslice;   // 7-bit slices per operand: 6 (0 selects it; 42 bits) or 7 (49 bits)
  int nsk[TC_MAX_KIND];
  long long coff[TC_MAX_KIND];
};
TcProblem tc_problem_of(const SynthDev& S);   // the synthetics' 8 Legendre / Bessel kinds
// workspace size and run; nwn: host copy of the wavenumber counts per frequency
// (1-based frequency index); wait_ns: limit of each pipeline wait (0: 1 s)
size_t sums_tc_workspace(const TcProblem& P, long long mtot, int* Kp_out);
const char* sums_tc_run(const TcProblem& P, const int* nwn, long long mtot, const double* tab, const double* A,
                        double* C, void* ws, size_t ws_bytes, unsigned long long wait_ns, cudaStream_t st);

}  // namespace gem

// error / timing / buffer hooks of the context (defined with gem_ctx)
int gem_set_error(gem_ctx* ctx, const char* msg);
void gem_note_synth_ms(gem_ctx* ctx, float ms);
int gem_ctx_device(const gem_ctx* ctx);
int gem_ctx_backend(const gem_ctx* ctx);
unsigned long long gem_ctx_tc_wait_ns(const gem_ctx* ctx);
void* gem_ctx_aux(gem_ctx* ctx, int slot, size_t bytes);
