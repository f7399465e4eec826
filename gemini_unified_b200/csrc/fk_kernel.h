// Launch-level structures of the FK kernels (device pointers only).
#pragma once
#include <cstdint>

#include "gem_device.cuh"

namespace gem {

// Schedules of a solver phase kernel (one block per SM): threads per block,
// and whether the 4- and 5-variable systems keep their half- and end-step
// matrices across the attempts of a Bulirsch-Stoer step (fast build; the
// 2-variable systems always do, the plain build never).  The autotuner picks
// one per phase; defaults measured at the batched configuration.
constexpr int FK_NSCHED = 6;
constexpr int FK_SCHED_BLOCK[FK_NSCHED] = {384, 512, 256, 384, 512, 256};
constexpr int FK_SCHED_BIGCACHE[FK_NSCHED] = {0, 0, 0, 1, 1, 1};
constexpr int FK_SCHED_DEFAULT[3] = {1, 0, 1};   // toroidal 512, spheroidal 384, adjoint 512 threads
// candidate deferrals of the bookkeeping passes (lanes waiting, trips waited);
// the last waits for the whole warp: its lanes, on adjacent degrees of one
// frequency, reach their sub-interval ends within a few steps of each other
constexpr int FK_NDEFER = 6;
constexpr int FK_DEFER_MIN[FK_NDEFER] = {1, 8, 16, 32, 32, 32};
constexpr int FK_DEFER_WAIT[FK_NDEFER] = {0, 6, 10, 24, 48, 1000000};
constexpr int FK_DEFER_DEFAULT = 4;
// queue granularity: consecutive queue positions a lane reserves per fetch (it
// takes the next of its run without the queue until the run is used up), or,
// with FK_QCHUNK > 0, runs of that many positions the warps of a block share
constexpr int FK_NGRAN = 4;
constexpr int FK_GRAN[FK_NGRAN] = {1, 2, 4, 1};
constexpr int FK_QCHUNK[FK_NGRAN] = {0, 0, 0, 1024};
constexpr int FK_GRAN_DEFAULT = 0;
constexpr int MAX_LAYER_KNOTS = 64;    // knots per layer handled by the spline kernel
// per-lane scratch elements (double2) of one Bulirsch-Stoer step, after the
// lane's node storage: A(x0) y0 and the last level of the Neville diagonal
constexpr int FK_LANE_STEP_SLOTS = 10;

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
  const double* poly;   // cubic coefficients per knot interval [nslot][nk+1][POLY_STRIDE] (fast variant)
  const int* jf;        // [nslot]
  const int* koff;      // [nslot] output index of (slot, iwn = 1)
  const int2* items;    // (slot, iwn) of each output index k
  const int* order;     // queue position -> k, most expensive first
  int nitems;
  long long nkf;        // extent of the wavenumber-frequency index in the outputs
  double2* gf64;        // optional FP64 output (nkf, nsp, nnod)
  float* gfre;          // optional FP32 real part
  float* gfim;          // optional FP32 imaginary part
  int* status;          // optional per-k status
  double2* scratch;     // per-thread node storage, element-major
  long long nthreads;   // scratch stride
  unsigned int* queue;  // work-queue counters, one per phase (zeroed before launch)
  double* rstart;       // [2][nkf] start radius, toroidal then spheroidal
  double2* um;          // [jre*6][nkf] upward minors at nodes 1..jre
  double2* dm;          // [(nnod-jre+1)*6][nkf] downward minors at nodes jre..nnod
  double2* dets;        // [nkf] spheroidal determinant at the receiver
  unsigned long long* stats;   // 6 counters
  unsigned long long* prof;    // optional lockstep counters [8]
  unsigned long long* warp_ns; // optional per-warp (start, end) globaltimer stamps
  const signed char* prop_kopt;   // optional proposed order target per (phase, k): [3][nkf]
  const float* prop_hs;           // optional proposed multiplier of the initial step per (phase, k): [3][nkf]
  struct StepRec* steplog;     // optional record of every step attempt
  unsigned long long steplog_cap;
  unsigned long long* steplog_n;
  // deferral of the bookkeeping between integrations: a pass runs when
  // adv_min lanes wait, one has waited adv_wait trips, or none integrates
  int adv_min, adv_wait;
  int qgran;            // queue positions reserved per fetch (FK_GRAN)
  int qchunk;           // > 0: runs of queue positions shared by the warps of a block (FK_QCHUNK)
  // toroidal phase of a set of source nodes (nsrc > 0): per source b its node and
  // type (0 force, 1 moment), passed by value; its output block starts at
  // element b * src_blk
  int nsrc;
  long long src_blk;
  unsigned char src_node[MAXNOD + 2];
  unsigned char src_type[MAXNOD + 2];
};
static_assert(MAXNOD + 1 <= 255, "source-node table entries are bytes");

// One Bulirsch-Stoer step attempt as the step log records it (32 bytes).
struct StepRec {
  double x;             // radius at the start of the step
  double h;             // step tried (signed)
  int k;                // item (wavenumber-frequency index of the run)
  float lgy;            // log10 of the mean |y| of the solution, including the renormalisation
  short nl;             // layer
  signed char sys;      // system (toroidal, minors, fluid, radial, adjoint)
  signed char result;   // attempt at which the step converged (3..7); 0: rejected
  short phase;          // phase kernel (0 toroidal, 1 spheroidal, 2 adjoint)
  short nstep;          // step number within the sub-interval
};

struct FKStatic;
}  // namespace gem

#include <cuda_runtime.h>
namespace gem {
cudaError_t launch_prep(const PrepArgs& A, int* d_err, cudaStream_t st);
cudaError_t launch_poly(const PrepArgs& A, double* poly, cudaStream_t st);
}  // namespace gem

// Two builds of the solver: gem_plain (parity path, no FMA contraction) and
// gem_fast (FMA, division-free spline, reciprocal complex inverses).
#define GEM_DECLARE_SOLVER(NS)                                                                          \
  namespace NS {                                                                                     \
  /* phase < 0: start radii; 0 toroidal, 1 spheroidal minors, 2 adjoint + spheroidal spectra;     */ \
  /* sched: index into FK_SCHED_BLOCK / FK_SCHED_BIGCACHE                                           */ \
  cudaError_t launch_fk_phase(int phase, int sched, const gem::FKStatic& P, const gem::FKLaunch& L, int grid,  \
                              cudaStream_t st);                                                      \
  int fk_phase_blocks_per_sm(int phase, int sched);                                                  \
  int fk_lane_slot_per_node();                                                                       \
  }
GEM_DECLARE_SOLVER(gem_plain)
GEM_DECLARE_SOLVER(gem_fast)
namespace gem_ray {
// travel-time table by ray tracing (raytable.cu): one thread per turning radius
cudaError_t launch_ray_table(const gem::FKStatic& P, const double* spl, int ntp, int stype, double eps, double drtp,
                             double a0, double* rtp, double* slowness, float* table, int* status, cudaStream_t st);
}
namespace gem {
}  // namespace gem
