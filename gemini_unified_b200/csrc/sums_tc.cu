// Degree sums on the 5th-generation tensor cores with sliced integer operands.
//
// The degree sums of harmonicDegreeSums.f90:95-351 are, for every Legendre
// table kind, the product C[row, station] = sum_l A[row, l] * T[l, station]
// (rows: frequency x sum x re/im; see synth.cu).  The FP64 form runs it on
// CUDA cores.  Here the Legendre recurrences and the coefficient weights stay
// FP64 and the product runs on tcgen05 as an exact integer computation:
//
//   T[l, n] = s_l c_n t,    s_l, c_n powers of two, |t| < 1
//   A[m, l] s_l = r_m a,    r_m a power of two,      |a| < 1
//   a = sum_i a_i 128^-(i+1), t = sum_j t_j 128^-(j+1), a_i, t_j in [-127, 127]
//   C[m, n] = r_m c_n sum_{w=0}^{S-1} 128^-(w+2) sum_{i+j=w} (sum_l a_i t_j)
//
// with S = 6 slices of 7 bits (42 bits of each operand relative to its row or
// column scale; terms with i + j >= S are dropped).  The slice products are
// accumulated exactly in INT32 by tcgen05.mma kind::i8 and combined in FP64,
// so the result keeps FP64-level accuracy even where the degree sum cancels by
// five orders of magnitude (near-antipodal stations), which FP16 operands with
// FP32 accumulation cannot.
//
// GEMM kernel: one CTA per 128 x BN output tile (BN 80 with 6 slices, 64 with 7).  Per k-block of 64 degrees,
// warp 0 issues TMA loads (64-byte swizzle) of the S slices of A and of T into
// a 2-stage shared-memory ring; warp 1 issues the S(S+1)/2 slice products (2 MMAs
// of K 32 each) into S TMEM accumulators of BN columns, one per weight w = i + j;
// warps 2-5 combine the accumulators in FP64 and write C.  All mbarrier waits
// of the pipeline are bounded by a timer (1 s unless the context sets another
// limit): a wait that runs out records an error flag, the CTA stops issuing
// work, waits (bounded by 1 s, whatever the limit) for its own copies and
// products, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "synth.h"

namespace gem {

// Slices per operand.  Measured on the tensor-core-sums configuration (synthetics step,
// worst trace error against the FP64 form): 7: 12.6 ms; 6: 11.3 ms, both at the FFT's
// own 1.75e-7; 5: 10.1 ms, but near-zero traces of the global configuration then miss
// the 1e-5 per-trace bar (1.4e-4); 4: 9.1 ms, 2.5e-6 (all with 128 x 64 tiles).  With six
// slices, 128 x 80 tiles (480 of the 512 TMEM columns) take the step from 11.3 to 10.4 ms
// at the same error: each A tile is loaded for 80 stations instead of 64.
constexpr int TC_S = 6;
constexpr int TC_BM = 128, TC_BN = 80, TC_BK = 64;      // tile; BK int8 = one swizzle row (64 or 32 bytes)
// The coupling synthetics combine 42 sums into strain, stress and traction, whose cancellations amplify
// the products' error: with 6 slices their spectra reach 5e-8 of a spectrum's peak against the oracle,
// with 7 (49 bits; 7 accumulators of 64 columns) the FP64 level.
constexpr int TC_S_FINE = 7, TC_BN_FINE = 64;
static_assert(TC_BK == 64 || TC_BK == 32, "swizzle spans of 64 or 32 bytes");
// Two stages: measured on the same step, 3 stages at N = 64 (8.51 ms) and 5 stages of BK = 32
// at N = 80 (8.74 ms) both lose to 2 stages of BK = 64 at N = 80 (7.63 ms): the operand bytes
// per product from L2 bound the main loop, not the depth of the pipeline.
constexpr int TC_STAGES = 2;
constexpr int TC_A_BYTES = TC_BM * TC_BK;               // 8 KiB per slice
constexpr int TC_THREADS = 192;
constexpr int TC_TMEM_COLS = 512;                       // NS accumulators of BN columns (power-of-two allocation)
// shape of one product: NS slices per operand, BN stations (columns) per tile
template <int NS, int BN> struct TcShape {
  static constexpr int B_BYTES = BN * TC_BK;                        // 5 KiB per slice at BN = 80
  static constexpr int STAGE_BYTES = NS * (TC_A_BYTES + B_BYTES);   // 78 KiB at (6, 80), 84 KiB at (7, 64)
  static constexpr int SMEM = TC_STAGES * STAGE_BYTES + 1024 /* alignment */ + 256 /* barriers */;
  static_assert(NS * BN <= TC_TMEM_COLS, "the accumulators must fit the tensor memory");
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "MMA N of kind::i8 with M = 128");
  static_assert(SMEM <= 227 * 1024, "stages must fit the shared memory of a CTA");
};
constexpr unsigned long long TC_WAIT_NS = 1000000000ull;   // default pipeline wait limit and the drain limit

// ---------------------------------------------------------------------------
//  Operand preparation (FP64 in, INT8 slices out)
// ---------------------------------------------------------------------------

// smallest power of two strictly above |x| (1 for 0 or non-finite)
__device__ __forceinline__ double pow2_above(double x) {
  if (!(x > 0.0) || !isfinite(x)) return 1.0;
  int e;
  frexp(x, &e);   // x = f 2^e, f in [0.5, 1)
  return ldexp(1.0, e);
}

// the 7-bit slices of x, |x| < 1: x = sum_i q_i 128^-(i+1) + O(128^-S).  The
// slices are the base-128 digits of u = trunc(|x| 128^S) with the sign of x
// (x 128^S is exact and the conversion truncates), the same digits as S
// rounds of x *= 128, q = trunc(x), x -= q, all of which are exact.
template <int NS>
__device__ __forceinline__ void slices_of(double x, signed char q[NS]) {
  static_assert(NS <= 8, "the digits must fit a 64-bit integer");
  const long long y = (long long)(x * (double)(1ull << (7 * NS)));
  const unsigned long long u = y < 0 ? (unsigned long long)(-y) : (unsigned long long)y;
#pragma unroll
  for (int i = 0; i < NS; ++i) {
    const int d = (int)((u >> (7 * (NS - 1 - i))) & 127u);
    q[i] = (signed char)(y < 0 ? -d : d);
  }
}

// 1/s for a power of two s whose reciprocal is a normal double (then x * (1/s)
// equals x / s exactly), else 0: the callers then divide
__device__ __forceinline__ double inv_pow2(double s) { return s >= 0x1p-1021 && s <= 0x1p1021 ? 1.0 / s : 0.0; }
__device__ __forceinline__ double div_pow2(double x, double s, double inv) { return inv != 0.0 ? x * inv : x / s; }

__device__ __forceinline__ double block_max(double m) {
  __shared__ double red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

// s[kind][l] = power of two above max over stations of |T[kind][l][sta]| (one block per (l, kind))
__global__ void tab_scale_kernel(int nsta, int lcap, int K, const double* __restrict__ tab, double* lscale, int Kp) {
  const int l = blockIdx.x, kind = blockIdx.y;
  double m = 0.0;
  if (l < K) {
    const double* row = tab + ((long long)kind * lcap + l) * nsta;
    for (int i = threadIdx.x; i < nsta; i += blockDim.x) m = fmax(m, fabs(row[i]));
  }
  m = block_max(m);
  if (threadIdx.x == 0) lscale[(long long)kind * Kp + l] = pow2_above(m);
}

// per (kind, station) max over l of |T[kind][l][sta] / s_l|, as the bits of a
// non-negative double (whose order is the unsigned integer order): blocks of
// 128 stations x 64 degrees
__global__ void tab_colmax_kernel(int nsta, int lcap, int K, int Kp, const double* __restrict__ tab,
                                  const double* __restrict__ lscale, unsigned long long* colmax) {
  __shared__ double sl[64], il[64];
  const int sta = blockIdx.x * blockDim.x + threadIdx.x, kind = blockIdx.z;
  const int l0 = blockIdx.y * 64, l1 = min(l0 + 64, K);
  if (threadIdx.x < 64 && l0 + (int)threadIdx.x < l1) {
    sl[threadIdx.x] = lscale[(long long)kind * Kp + l0 + threadIdx.x];
    il[threadIdx.x] = inv_pow2(sl[threadIdx.x]);
  }
  __syncthreads();
  if (sta >= nsta) return;
  double m = 0.0;
  for (int l = l0; l < l1; ++l)
    m = fmax(m, fabs(div_pow2(tab[((long long)kind * lcap + l) * nsta + sta], sl[l - l0], il[l - l0])));
  atomicMax(colmax + (long long)kind * nsta + sta, (unsigned long long)__double_as_longlong(m));
}

// c[kind][sta] = power of two above that maximum
__global__ void tab_colscale_kernel(int n, const unsigned long long* __restrict__ colmax, double* cscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cscale[i] = pow2_above(__longlong_as_double((long long)colmax[i]));
}

// T8[j][kind*nsta + sta][l] = slice j of T / (s_l c_sta) for a tile of 64 degrees x 64
// stations: slices formed on the coalesced read (consecutive stations) into a
// shared byte tile [slice][station][degree], written back as 4-degree words
template <int NS>
__global__ void tab_slice_kernel(int nkind, int nsta, int lcap, int K, int Kp, const double* __restrict__ tab,
                                 const double* __restrict__ lscale, const double* __restrict__ cscale,
                                 signed char* T8) {
  constexpr int ROW = 68;   // bytes per station row: 17 words, so the byte writes of a warp hit distinct banks
  __shared__ __align__(16) signed char dig[NS][64][ROW];
  __shared__ double sl[64], il[64];
  const int kind = blockIdx.z;
  const int l0 = blockIdx.x * 64, s0 = blockIdx.y * 64;
  const int tx = threadIdx.x & 63, ty = threadIdx.x >> 6;   // 256 threads: 64 x 4
  if (threadIdx.x < 64) {
    const int l = l0 + threadIdx.x;
    sl[threadIdx.x] = l < K ? lscale[(long long)kind * Kp + l] : 1.0;
    il[threadIdx.x] = inv_pow2(sl[threadIdx.x]);
  }
  __syncthreads();
  const int sta = s0 + tx;
  const double cs = sta < nsta ? cscale[(long long)kind * nsta + sta] : 1.0, ic = inv_pow2(cs);
  for (int r = ty; r < 64; r += 4) {
    const int l = l0 + r;
    double v = 0.0;
    if (l < K && sta < nsta) v = div_pow2(div_pow2(tab[((long long)kind * lcap + l) * nsta + sta], sl[r], il[r]), cs, ic);
    signed char q[NS];
    slices_of<NS>(v, q);
#pragma unroll
    for (int j = 0; j < NS; ++j) dig[j][tx][r] = q[j];
  }
  __syncthreads();
  const long long plane = (long long)nkind * nsta * Kp;
  for (int e = threadIdx.x; e < 64 * 16; e += 256) {
    const int r = e >> 4, w = e & 15;   // station row of the tile, word of 4 degrees
    if (s0 + r >= nsta) continue;
    const long long o = ((long long)kind * nsta + s0 + r) * Kp + l0 + 4 * w;   // Kp, l0: multiples of 64
#pragma unroll
    for (int j = 0; j < NS; ++j)
      *reinterpret_cast<uint32_t*>(T8 + j * plane + o) = *reinterpret_cast<const uint32_t*>(&dig[j][r][4 * w]);
  }
}

// A8[i][row][l] = slice i of A[row][l] s_l / r_row; one block per row of every kind
template <int NS>
__global__ void coef_slice_kernel(int lcap, long long mtot, int K, int Kp, const double* __restrict__ A,
                                  const double* __restrict__ lscale, const int* __restrict__ row_kind,
                                  signed char* A8, double* rscale) {
  const long long row = blockIdx.x;
  const int kind = row_kind[row];
  const double* a = A + row * lcap;
  const double* sl = lscale + (long long)kind * Kp;
  double m = 0.0;
  for (int l = threadIdx.x; l < K; l += blockDim.x) m = fmax(m, fabs(a[l] * sl[l]));
  const double r = pow2_above(block_max(m)), ir = inv_pow2(r);
  if (threadIdx.x == 0) rscale[row] = r;
  const long long plane = mtot * Kp;
  for (int l = threadIdx.x; l < Kp; l += blockDim.x) {
    signed char q[NS];
    slices_of<NS>(l < K ? div_pow2(a[l] * sl[l], r, ir) : 0.0, q);
#pragma unroll
    for (int i = 0; i < NS; ++i) A8[i * plane + row * Kp + l] = q[i];
  }
}

// ---------------------------------------------------------------------------
//  tcgen05 integer GEMM
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: true when the phase completed, false after limit_ns or when
// another role of this CTA has already given up (abort flag).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          unsigned long long limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > limit_ns) {
      *abort_flag = 1;
      return false;
    }
  }
}

// wait that ignores the abort flag (used to drain this CTA's own copies before exit)
__device__ __forceinline__ void mbar_drain(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = global_ns();
  while (!mbar_try(bar, parity) && global_ns() - t0 < TC_WAIT_NS) {
  }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// K-major operand swizzled over rows of TC_BK bytes (64 or 32): 8-row groups 8 TC_BK bytes apart
__device__ __forceinline__ uint64_t smem_desc_kmajor(const void* p) {
  const uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;                   // start address
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((8 * TC_BK) >> 4) << 32;        // stride byte offset: 8 rows x TC_BK bytes
  d |= (uint64_t)1 << 46;                         // descriptor version (tcgen05)
  d |= (uint64_t)(TC_BK == 64 ? 4 : 6) << 61;     // SWIZZLE_64B / SWIZZLE_32B
  return d;
}

// kind::i8 instruction descriptor: D s32, A/B signed 8-bit, both K-major, N = BN, M = 128
template <int BN>
__host__ __device__ constexpr uint32_t tc_idesc() {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_BM >> 4) << 24);
}

// The 16 columns [taddr + w stride, + 16) of the NS accumulators w = 0..NS-1,
// loaded by one asm statement that ends with the wait for all of them: the NS
// loads are in flight together, and the compiler sees the registers defined
// only after the wait.
#define GEM_TM16(a, k)                                                                                        \
  "=r"(a[k][0]), "=r"(a[k][1]), "=r"(a[k][2]), "=r"(a[k][3]), "=r"(a[k][4]), "=r"(a[k][5]), "=r"(a[k][6]),    \
      "=r"(a[k][7]), "=r"(a[k][8]), "=r"(a[k][9]), "=r"(a[k][10]), "=r"(a[k][11]), "=r"(a[k][12]),             \
      "=r"(a[k][13]), "=r"(a[k][14]), "=r"(a[k][15])
template <int NS>
__device__ __forceinline__ void tmem_ld_acc16(uint32_t taddr, uint32_t stride, uint32_t (&v)[NS][16]) {
  static_assert(NS == 6 || NS == 7, "six or seven accumulators");
  if constexpr (NS == 6) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%96];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%97];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%98];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%99];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%64,%65,%66,%67,%68,%69,%70,%71,%72,%73,%74,%75,%76,%77,%78,%79}, [%100];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%80,%81,%82,%83,%84,%85,%86,%87,%88,%89,%90,%91,%92,%93,%94,%95}, [%101];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : GEM_TM16(v, 0), GEM_TM16(v, 1), GEM_TM16(v, 2), GEM_TM16(v, 3),
          GEM_TM16(v, 4), GEM_TM16(v, 5)
        : "r"(taddr + 0u * stride), "r"(taddr + 1u * stride), "r"(taddr + 2u * stride), "r"(taddr + 3u * stride),
          "r"(taddr + 4u * stride), "r"(taddr + 5u * stride));
  } else {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%112];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%113];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%114];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%115];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%64,%65,%66,%67,%68,%69,%70,%71,%72,%73,%74,%75,%76,%77,%78,%79}, [%116];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%80,%81,%82,%83,%84,%85,%86,%87,%88,%89,%90,%91,%92,%93,%94,%95}, [%117];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%96,%97,%98,%99,%100,%101,%102,%103,%104,%105,%106,%107,%108,%109,%110,%111}, [%118];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : GEM_TM16(v, 0), GEM_TM16(v, 1), GEM_TM16(v, 2), GEM_TM16(v, 3),
          GEM_TM16(v, 4), GEM_TM16(v, 5), GEM_TM16(v, 6)
        : "r"(taddr + 0u * stride), "r"(taddr + 1u * stride), "r"(taddr + 2u * stride), "r"(taddr + 3u * stride),
          "r"(taddr + 4u * stride), "r"(taddr + 5u * stride), "r"(taddr + 6u * stride));
  }
}
#undef GEM_TM16

template <int NS, int BN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    sums_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                   const int4* __restrict__ tiles, const int* __restrict__ kind_rows,
                   const long long* __restrict__ kind_rowoff, const long long* __restrict__ coff, int nkind, int nsta,
                   long long mtot, const double* __restrict__ rscale, const double* __restrict__ cscale,
                   double* C, int* err, unsigned long long wait_ns) {
  using Sh = TcShape<NS, BN>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t* full = (uint64_t*)(smem + TC_STAGES * Sh::STAGE_BYTES);
  uint64_t* empty = full + TC_STAGES;
  uint64_t* acc_full = empty + TC_STAGES;
  uint32_t* tmem_slot = (uint32_t*)(acc_full + 1);
  volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // (kind, first row of the tile within the kind, k-blocks): the tile's rows are zero
  // beyond its largest wavenumber count, so its k-loop stops there
  const int4 t = tiles[blockIdx.y];
  const int kind = t.x, m0 = t.y, nkb = t.z;
  const int n0 = blockIdx.x * BN;
  const int Mk = kind_rows[kind];
  const long long rowA = kind_rowoff[kind] + m0;
  const long long rowB = (long long)kind * nsta + n0;

  if (threadIdx.x == 0) {
    for (int s = 0; s < TC_STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
    mbar_init(acc_full, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TC_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: the S slices of A and of T per k-block
    int issued = 0;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % TC_STAGES;
      if (kb >= TC_STAGES && !mbar_wait(&empty[s], ((kb / TC_STAGES) - 1) & 1, abort_flag, wait_ns)) break;
      unsigned char* st = smem + s * Sh::STAGE_BYTES;
      mbar_expect_tx(&full[s], Sh::STAGE_BYTES);
#pragma unroll 1
      for (int i = 0; i < NS; ++i)
        tma_load_2d(st + i * TC_A_BYTES, &mapA, &full[s], kb * TC_BK, (int)(i * mtot + rowA));
#pragma unroll 1
      for (int j = 0; j < NS; ++j)
        tma_load_2d(st + NS * TC_A_BYTES + j * Sh::B_BYTES, &mapB, &full[s], kb * TC_BK,
                    (int)(j * (long long)nkind * nsta + rowB));
      ++issued;
    }
    for (int kb = (issued > TC_STAGES ? issued - TC_STAGES : 0); kb < issued; ++kb)
      mbar_drain(&full[kb % TC_STAGES], (kb / TC_STAGES) & 1);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: accumulator w = i + j at TMEM columns BN w
    bool ok = true;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % TC_STAGES;
      if (!mbar_wait(&full[s], (kb / TC_STAGES) & 1, abort_flag, wait_ns)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const unsigned char* st = smem + s * Sh::STAGE_BYTES;
#pragma unroll 1
      for (int i = 0; i < NS; ++i) {
        const uint64_t da = smem_desc_kmajor(st + i * TC_A_BYTES);
#pragma unroll 1
        for (int j = 0; j + i < NS; ++j) {
          const uint64_t db = smem_desc_kmajor(st + NS * TC_A_BYTES + j * Sh::B_BYTES);
          const uint32_t dtm = tmem + (uint32_t)((i + j) * BN);
#pragma unroll
          for (int kk = 0; kk < TC_BK / 32; ++kk) {
            const uint64_t adv = (uint64_t)((kk * 32) >> 4);   // 32 int8 = 32 bytes along K
            const uint32_t acc = (kb > 0 || kk > 0 || i > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtm),
                "l"(da + adv), "l"(db + adv), "r"(tc_idesc<BN>()), "r"(acc));
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&empty[s]))
                   : "memory");
    }
    // signals the epilogue once every product issued above has completed
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(acc_full))
                 : "memory");
    if (!ok) *abort_flag = 1;
    // the products issued above write TMEM and read the stages.  After an abort
    // (set here or by the epilogue at any time) nobody else waits for them, so
    // they are always drained here, before the CTA's closing barrier frees the
    // tensor memory; without an abort the epilogue has waited for the same phase
    mbar_drain(acc_full, 0);
  } else if (warp >= 2) {
    // ---- epilogue: TMEM lanes 32*(warp % 4) .. +31 hold rows of the tile
    const int q = warp & 3;
    const bool done = mbar_wait(acc_full, 0, abort_flag, wait_ns);
    asm volatile("tcgen05.fence::after_thread_sync;");
    const int r = m0 + q * 32 + lane;   // row within the kind
    // the ring is idle once every product has completed: each warp stages its
    // 32 rows x 16 columns there and writes them row by row (a row's 16
    // doubles are one 128-byte segment), not as 32 strided rows per store
    const bool store = __all_sync(0xffffffffu, done && !*abort_flag);
    const double rs = (store && r < Mk) ? rscale[kind_rowoff[kind] + r] : 0.0;
    double* ck = C + coff[kind];
    const double* cs = cscale + (long long)kind * nsta;
    double* stg = reinterpret_cast<double*>(smem) + q * (32 * 17);   // 17: one pad double per row
    // columns in chunks of 16 (BN is a multiple of 16); the NS accumulators of a
    // chunk are loaded together, then combined smallest weights first
#pragma unroll 1
    for (int c = 0; c < BN / 16; ++c) {
      uint32_t v[NS][16];
      tmem_ld_acc16<NS>(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(c * 16), (uint32_t)BN, v);
      double sum[16];
#pragma unroll
      for (int jj = 0; jj < 16; ++jj) sum[jj] = 0.0;
#pragma unroll
      for (int w = NS - 1; w >= 0; --w) {
        const double wgt = ldexp(1.0, -7 * (w + 2));
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) sum[jj] += (double)(int)v[w][jj] * wgt;
      }
      if (store) {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj) stg[lane * 17 + jj] = sum[jj] * rs;
        __syncwarp();
        const int col = lane & 15, n = n0 + c * 16 + col;
        const double csn = n < nsta ? cs[n] : 0.0;
#pragma unroll 4
        for (int k = 0; k < 16; ++k) {
          const int row = 2 * k + (lane >> 4), rg = m0 + q * 32 + row;
          if (rg < Mk && n < nsta) ck[(long long)rg * nsta + n] = stg[row * 17 + col] * csn;
        }
        __syncwarp();
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(err, 1);
}

}  // namespace gem

// ===========================================================================
//  Host side
// ===========================================================================
using namespace gem;

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2D map over int8 rows of Kp bytes, box TC_BK bytes x box_rows, swizzled over TC_BK bytes
bool make_map(CUtensorMap* map, const signed char* base, long long rows, long long kp, int box_rows) {
  EncodeTiledFn f = encode_fn();
  if (!f) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kp};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return f(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, TC_BK == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct TcLayout {
  int Kp;
  size_t off[10], total;
};

int tc_slices(const TcProblem& P) { return P.nslice == TC_S_FINE ? TC_S_FINE : TC_S; }

TcLayout tc_layout(const TcProblem& P, long long mtot) {
  TcLayout L{};
  const int K = P.lmax + 1, nk = P.nkind, ns = tc_slices(P);
  L.Kp = (K + 63) / 64 * 64;   // the slicing kernels work on 64-degree tiles
  const size_t sz[10] = {(size_t)ns * nk * P.ncol * L.Kp,             // T8
                        (size_t)ns * mtot * L.Kp,                     // A8
                        (size_t)nk * L.Kp * sizeof(double),           // lscale
                        (size_t)nk * P.ncol * sizeof(double),         // cscale
                        (size_t)mtot * sizeof(double),                // rscale
                        (size_t)mtot * sizeof(int),                   // row kind
                        (size_t)(mtot / TC_BM + nk + 1) * sizeof(int4),   // tiles
                        (size_t)3 * TC_MAX_KIND * sizeof(long long),  // per-kind tables
                        (size_t)(TC_MAX_KIND + 8) * sizeof(int),      // kind rows + error flag
                        (size_t)nk * P.ncol * sizeof(unsigned long long)};   // column maxima
  size_t b = 0;
  for (int i = 0; i < 10; ++i) {
    L.off[i] = b;
    b += (sz[i] + 1023) / 1024 * 1024;
  }
  L.total = b + 1024;
  return L;
}

}  // namespace

namespace gem {

TcProblem tc_problem_of(const SynthDev& S) {
  TcProblem P{};
  P.nkind = 8; P.ncol = S.nsta; P.lcap = S.lcap; P.lmax = S.lmax; P.nf1 = S.nf1; P.nf2 = S.nf2;
  for (int k = 0; k < 8; ++k) { P.nsk[k] = S.nsk[k]; P.coff[k] = S.coff[k]; }
  return P;
}

size_t sums_tc_workspace(const TcProblem& P, long long mtot, int* Kp_out) {
  TcLayout L = tc_layout(P, mtot);
  if (Kp_out) *Kp_out = L.Kp;
  return L.total;
}

// operand slices of NS digits and the products on BN-column tiles (blocking)
template <int NS, int BN>
const char* tc_slice_and_multiply(const TcProblem& P, long long mtot, int K, int Kp, const double* tab, const double* A,
                                  const double* lscale, const double* cscale, const int* row_kind, signed char* T8,
                                  signed char* A8, double* rscale, const int4* tiles, size_t ntiles, int* ints,
                                  const long long* tabs, double* C, unsigned long long wait_ns, cudaStream_t st) {
  using Sh = TcShape<NS, BN>;
  const int nk = P.nkind, ncol = P.ncol;
  tab_slice_kernel<NS><<<dim3(Kp / 64, (ncol + 63) / 64, nk), 256, 0, st>>>(nk, ncol, P.lcap, K, Kp, tab, lscale,
                                                                            cscale, T8);
  coef_slice_kernel<NS><<<(unsigned)mtot, 256, 0, st>>>(P.lcap, mtot, K, Kp, A, lscale, row_kind, A8, rscale);
  // tensor maps over A8 [NS mtot][Kp] and T8 [NS * nkind * ncol][Kp]
  CUtensorMap mA, mB;
  if (!make_map(&mA, A8, NS * mtot, Kp, TC_BM) || !make_map(&mB, T8, NS * (long long)nk * ncol, Kp, BN))
    return "sums_tc: cuTensorMapEncodeTiled failed";
  if (cudaFuncSetAttribute(sums_tc_kernel<NS, BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, Sh::SMEM) !=
      cudaSuccess)
    return "sums_tc: shared-memory attribute";
  if (cudaMemsetAsync(ints + TC_MAX_KIND, 0, sizeof(int), st) != cudaSuccess) return "sums_tc: upload failed";
  dim3 grid((ncol + BN - 1) / BN, (unsigned)ntiles);
  sums_tc_kernel<NS, BN><<<grid, TC_THREADS, Sh::SMEM, st>>>(mA, mB, tiles, ints, tabs + TC_MAX_KIND,
                                                             tabs + 2 * TC_MAX_KIND, nk, ncol, mtot, rscale, cscale,
                                                             C, ints + TC_MAX_KIND, wait_ns ? wait_ns : TC_WAIT_NS);
  if (cudaGetLastError() != cudaSuccess) return "sums_tc: launch failed";
  int herr = 0;
  if (cudaMemcpyAsync(&herr, ints + TC_MAX_KIND, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return "sums_tc: execution failed";
  if (herr) return "sums_tc: a pipeline wait timed out";
  return nullptr;
}

// Sliced-integer sums: from the FP64 tables tab[kind][l][col] and coefficients
// A[kind rows][lcap], write C[kind][row][col] in FP64.  ws: device workspace of
// sums_tc_workspace bytes; wait_ns: limit of each pipeline wait (0: 1 s).
// Blocking (synchronises the stream).
const char* sums_tc_run(const TcProblem& P, const int* nwn, long long mtot, const double* tab, const double* A,
                        double* C, void* ws, size_t ws_bytes, unsigned long long wait_ns, cudaStream_t st) {
  if (P.nkind < 1 || P.nkind > TC_MAX_KIND) return "sums_tc: table kinds outside 1..16";
  TcLayout L = tc_layout(P, mtot);
  if (ws_bytes < L.total) return "sums_tc: workspace too small";
  const int nk = P.nkind, ncol = P.ncol;
  if (7LL * mtot >= (1LL << 31) || 7LL * nk * ncol >= (1LL << 31)) return "sums_tc: operand rows exceed 2^31";
  if ((long long)L.Kp * tc_slices(P) * 127 * 127 >= (1LL << 31))
    return "sums_tc: degree range too large for INT32 accumulation";
  if (P.nslice != 0 && P.nslice != TC_S && P.nslice != TC_S_FINE) return "sums_tc: 6 or 7 slices per operand";
  const int K = P.lmax + 1, Kp = L.Kp;
  const int nf = P.nf2 - P.nf1 + 1;
  char* base = (char*)(((uintptr_t)ws + 1023) & ~(uintptr_t)1023);
  signed char* T8 = (signed char*)(base + L.off[0]);
  signed char* A8 = (signed char*)(base + L.off[1]);
  double* lscale = (double*)(base + L.off[2]);
  double* cscale = (double*)(base + L.off[3]);
  double* rscale = (double*)(base + L.off[4]);
  int* row_kind = (int*)(base + L.off[5]);
  int4* tiles = (int4*)(base + L.off[6]);
  long long* tabs = (long long*)(base + L.off[7]);
  int* ints = (int*)(base + L.off[8]);   // [0..15] rows per kind, [16] error flag
  unsigned long long* colmax = (unsigned long long*)(base + L.off[9]);
  int krows[TC_MAX_KIND + 8] = {0};
  long long htabs[3 * TC_MAX_KIND] = {0};
  std::vector<int4> htiles;
  std::vector<int> hrk((size_t)mtot);
  long long ro = 0;
  for (int k = 0; k < nk; ++k) {
    krows[k] = 2 * nf * P.nsk[k];
    htabs[TC_MAX_KIND + k] = ro;
    htabs[2 * TC_MAX_KIND + k] = P.coff[k];
    for (int m = 0; m < krows[k]; m += TC_BM) {
      // rows 2 (slot nsk + rank) + re/im; the coefficients of frequency slot are zero
      // from degree nwn[nf1 - 1 + slot] on
      const int s0 = m / (2 * P.nsk[k]), s1 = std::min(nf - 1, (m + TC_BM - 1) / (2 * P.nsk[k]));
      int ext = 0;
      for (int s = s0; s <= s1; ++s) ext = std::max(ext, nwn[P.nf1 - 1 + s]);
      ext = std::min(ext, K);
      htiles.push_back(make_int4(k, m, std::max(1, (ext + TC_BK - 1) / TC_BK), 0));
    }
    for (int m = 0; m < krows[k]; ++m) hrk[(size_t)(ro + m)] = k;
    ro += krows[k];
  }
  if (ro != mtot) return "sums_tc: row count mismatch";
  if (htiles.empty()) return nullptr;
  // longest k-loops first: the short tiles fill the last wave
  std::stable_sort(htiles.begin(), htiles.end(), [](const int4& a, const int4& b) { return a.z > b.z; });
  if (cudaMemcpyAsync(tiles, htiles.data(), htiles.size() * sizeof(int4), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(row_kind, hrk.data(), hrk.size() * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(tabs, htabs, sizeof htabs, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(ints, krows, sizeof krows, cudaMemcpyHostToDevice, st) != cudaSuccess)
    return "sums_tc: upload failed";
  // operands
  tab_scale_kernel<<<dim3(Kp, nk), 256, 0, st>>>(ncol, P.lcap, K, tab, lscale, Kp);
  if (cudaMemsetAsync(colmax, 0, (size_t)nk * ncol * sizeof(unsigned long long), st) != cudaSuccess)
    return "sums_tc: upload failed";
  tab_colmax_kernel<<<dim3((ncol + 127) / 128, (K + 63) / 64, nk), 128, 0, st>>>(ncol, P.lcap, K, Kp, tab, lscale,
                                                                                colmax);
  tab_colscale_kernel<<<(nk * ncol + 255) / 256, 256, 0, st>>>(nk * ncol, colmax, cscale);
  if (tc_slices(P) == TC_S_FINE)
    return tc_slice_and_multiply<TC_S_FINE, TC_BN_FINE>(P, mtot, K, Kp, tab, A, lscale, cscale, row_kind, T8, A8,
                                                      rscale, tiles, htiles.size(), ints, tabs, C, wait_ns, st);
  return tc_slice_and_multiply<TC_S, TC_BN>(P, mtot, K, Kp, tab, A, lscale, cscale, row_kind, T8, A8, rscale, tiles,
                                            htiles.size(), ints, tabs, C, wait_ns, st);
}

}  // namespace gem
