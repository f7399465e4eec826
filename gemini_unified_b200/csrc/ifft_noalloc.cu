// gem_ifft_run_noalloc: the batched inverse FFT of gem_ifft_run_device for
// callers that cannot allocate device memory when they call it -- a code whose
// device memory is already handed out by its own pool allocator (a PyTorch
// caching allocator, a solver that reserves HBM at start-up), or one that must
// not let cudaMalloc/cudaFree synchronise the device while its other streams
// run.  It needs no context either.
//
// The transform's tables (the twiddles of every radix-2 stage and the
// exp(sigma t) factors: at most 8192*16 + 8192*8 = 196,608 bytes) live in one
// file-scope device array of NOALLOC_SCRATCH_BYTES = 256 KiB, which every GPU
// that loads this library holds until the process exits.  Nothing is allocated
// per call: no cudaMalloc, no cudaFree, no allocating library routine, no host
// heap.
//
// Sharing rules: all calls on one device share the array, and it keeps the
// last call's tables.  Nothing in it has to start at zero: each call rewrites
// the whole table region it reads, on its stream, before its transform kernel
// runs.  Calls that overlap on the GPU (different streams, or host threads
// whose work runs concurrently on the same device) race on the array and give
// wrong series; order them on one stream.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address with cudaGetSymbolAddress; later calls reuse the
// address.  Make that first call on each device before any stream capture.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "synth.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 256 * 1024;
constexpr int NOALLOC_MAX_DEVICES = 64;

}  // namespace

// In host code this name stands for the device array; its device address comes
// from cudaGetSymbolAddress at set-up.
static __device__ __align__(256) unsigned char g_ifft_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

void* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_setup_lock;

int report(char* errbuf, int errlen, int level, const char* fmt, ...) {
  if (errbuf && errlen > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(errbuf, (size_t)errlen, fmt, ap);
    va_end(ap);
  }
  return level;
}

// Device address of the scratch array on the current device (set-up on first use).
int scratch_address(void** out, char* errbuf, int errlen) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: device %d above the %d devices supported", dev,
                  NOALLOC_MAX_DEVICES);
  std::lock_guard<std::mutex> guard(g_setup_lock);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ifft_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
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
  const size_t need = ifft_table_bytes(g.ns, nsamp);
  if (need > NOALLOC_SCRATCH_BYTES)
    return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: tables need %zu bytes, above the %zu-byte scratch", need,
                  NOALLOC_SCRATCH_BYTES);
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
  ifft_tables_kernel<<<8, 256, 0, st>>>(g.ns, g.nslog, nsamp, std::exp(sigma * g.dts), tw, fac);
  ifft_kernel<<<(unsigned)ntr, IFFT_THREADS, smem, st>>>(S, (const double2*)d_sp, tw, fac, d_ts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return report(errbuf, errlen, GEM_ERROR, "ifft_noalloc: launch: %s", cudaGetErrorString(e));
  if (g.decimated) return report(errbuf, errlen, GEM_WARNING, "Downsampling to less than 1./(2*fny) requested");
  return GEM_OK;
}
