// gem_ifft_run_noalloc: the batched inverse FFT of gem_ifft_run_device for
// callers that cannot allocate device memory when they call it -- a code whose
// device memory is already handed out by its own pool allocator (a PyTorch
// caching allocator, a solver that reserves HBM at start-up), or one that must
// not let cudaMalloc/cudaFree synchronise the device while its other streams
// run.  It needs no context either.
//
// The transform's tables (the twiddles of every radix-2 stage and the
// exp(sigma t) factors: at most 8192*16 + 8192*8 = 196,608 bytes, since the
// FFT length is limited to 8192) live in one file-scope device array of
// NOALLOC_SCRATCH_BYTES = 256 KiB, which every GPU that loads this library
// holds until the process exits.  Nothing is allocated per call: no cudaMalloc,
// no cudaFree, no allocating library routine, no host heap.
//
// Sharing rules: all calls on one device share the array, and it keeps the
// last call's tables.  Nothing in it has to start at zero: each call rewrites
// the whole table region it reads, on its stream, before its transform kernel
// runs.  Calls that overlap on the GPU (different streams, or host threads
// whose work runs concurrently on the same device) race on the array and give
// wrong series; order them on one stream.
//
// Set-up: every call, with the caller's device current, looks up the array's
// device address in the current context with cudaGetSymbolAddress (a lookup,
// not an allocation), so the address stays right after cudaDeviceReset or in
// a recreated context.  The first call on a device may load the library's
// device code into the context (CUDA's lazy module loading); make that first
// call on each device before any stream capture.
#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "synth.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 256 * 1024;
// the FFT length limit of fft_geometry is what keeps the tables inside the array
static_assert((size_t)gem::IFFT_MAX_NS * (sizeof(double2) + sizeof(double)) <= NOALLOC_SCRATCH_BYTES,
              "inverse-FFT tables of the longest transform exceed the no-allocation scratch array");

}  // namespace

// In host code this name stands for the device array; its device address comes
// from cudaGetSymbolAddress at set-up.
static __device__ __align__(256) unsigned char g_ifft_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

int report(char* errbuf, int errlen, int level, const char* fmt, ...) {
  if (errbuf && errlen > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(errbuf, (size_t)errlen, fmt, ap);
    va_end(ap);
  }
  return level;
}

// Device address of the scratch array in the current context, looked up on every call.
int scratch_address(void** out, char* errbuf, int errlen) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_ifft_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
  *out = p;
  return GEM_OK;
}

}  // namespace

extern "C" int gem_ifft_run_noalloc(int nf1, int nf2, double df, double sigma, int ntr, const double* d_sp,
                                    long long ldsp, int nsamp, double dt, float* d_ts, void* stream, char* errbuf,
                                    int errlen) {
  using namespace gem;
  if (errbuf && errlen > 0) errbuf[0] = '\0';
  if (!d_sp || !d_ts) return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: null spectrum or time-series buffer");
  if (ntr < 1 || ldsp < nf2) return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: need ntr >= 1 and ldsp >= nf2");
  FftGeometry g;
  if (const char* why = fft_geometry(nf1, nf2, df, nsamp, dt, g)) return report(errbuf, errlen, GEM_ERROR, "%s", why);
  void* scratch = nullptr;
  if (int rc = scratch_address(&scratch, errbuf, errlen)) return rc;
  double2* tw = (double2*)scratch;
  double* fac = (double*)((char*)scratch + (size_t)g.ns * sizeof(double2));
  SynthDev S{};
  S.nf1 = nf1; S.nf2 = nf2; S.ns = g.ns; S.nslog = g.nslog; S.nsamp = nsamp; S.ndec = g.ndec; S.df = df;
  S.sigma = sigma; S.ldx = ldsp;
  // one series in shared memory: the limit is set per call, as the other transform paths set their own
  const size_t smem = (size_t)g.ns * sizeof(double2);
  cudaError_t e = cudaFuncSetAttribute(ifft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  cudaStream_t st = (cudaStream_t)stream;
  // launched through cudaLaunchKernel, whose return value is this launch's own
  // status: an error the caller left pending is neither reported nor cleared
  int ns = g.ns, nslog = g.nslog, ns_out = nsamp;
  double efac = std::exp(sigma * g.dts);
  double2* tw_arg = tw;
  double* fac_arg = fac;
  void* targs[] = {&ns, &nslog, &ns_out, &efac, &tw_arg, &fac_arg};
  e = cudaLaunchKernel((const void*)ifft_tables_kernel, dim3(8), dim3(256), targs, 0, st);
  if (e != cudaSuccess)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: table kernel launch: %s", cudaGetErrorString(e));
  const double2* sp_arg = (const double2*)d_sp;
  const double2* twc = tw;
  const double* facc = fac;
  float* ts_arg = d_ts;
  void* fargs[] = {&S, &sp_arg, &twc, &facc, &ts_arg};
  e = cudaLaunchKernel((const void*)ifft_kernel, dim3((unsigned)ntr), dim3(IFFT_THREADS), fargs, smem, st);
  if (e != cudaSuccess)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: transform kernel launch: %s", cudaGetErrorString(e));
  if (g.decimated) return report(errbuf, errlen, GEM_WARNING, "Downsampling to less than 1./(2*fny) requested");
  return GEM_OK;
}
