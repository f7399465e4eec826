// One build of the FK solver kernels: the including file defines GEM_NS and
// GEM_FAST (gem_plain / 0 and gem_fast / 1).
#include <cuda_runtime.h>

#include "fk_kernel.h"
#include "fk_solver.cuh"
#include "fk_phases.cuh"

namespace GEM_NS {
template <int PH, int BLK>
static size_t phase_smem() {
  return (size_t)(BLK / 32) * PhaseDiag<PH, BLK>::L * PhaseNV<PH>::NV * 32 * sizeof(double2);
}

template <int PH, int BLK, bool BIG>
static cudaError_t phase_attr() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fk_phase_kernel<PH, BLK, BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)phase_smem<PH, BLK>());
  if (e == cudaSuccess) done = true;
  return e;
}

template <int PH, int BLK, bool BIG>
static cudaError_t launch_ph(const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st) {
  cudaError_t e = phase_attr<PH, BLK, BIG>();
  if (e != cudaSuccess) return e;
  fk_phase_kernel<PH, BLK, BIG><<<grid, BLK, phase_smem<PH, BLK>(), st>>>(P, L);
  return cudaGetLastError();
}

template <int PH, int BLK, bool BIG>
static int bps() {
  if (phase_attr<PH, BLK, BIG>() != cudaSuccess) return 1;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fk_phase_kernel<PH, BLK, BIG>, BLK, phase_smem<PH, BLK>()) !=
      cudaSuccess)
    return 1;
  return nb < 1 ? 1 : nb;
}

// The matrix-caching flag only changes the 4- and 5-variable systems of the
// fast build: the toroidal phase and the plain build use the schedule's block
// size alone.
template <int PH>
static constexpr bool big_applies() { return GEM_FAST && PH != PH_TOR; }

template <int PH>
static cudaError_t launch_sched(int sched, const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st) {
  const bool big = big_applies<PH>() && FK_SCHED_BIGCACHE[sched];
  switch (FK_SCHED_BLOCK[sched]) {
    case 256: return big ? launch_ph<PH, 256, big_applies<PH>()>(P, L, grid, st) : launch_ph<PH, 256, false>(P, L, grid, st);
    case 512: return big ? launch_ph<PH, 512, big_applies<PH>()>(P, L, grid, st) : launch_ph<PH, 512, false>(P, L, grid, st);
    default: return big ? launch_ph<PH, 384, big_applies<PH>()>(P, L, grid, st) : launch_ph<PH, 384, false>(P, L, grid, st);
  }
}

template <int PH>
static int bps_sched(int sched) {
  const bool big = big_applies<PH>() && FK_SCHED_BIGCACHE[sched];
  switch (FK_SCHED_BLOCK[sched]) {
    case 256: return big ? bps<PH, 256, big_applies<PH>()>() : bps<PH, 256, false>();
    case 512: return big ? bps<PH, 512, big_applies<PH>()>() : bps<PH, 512, false>();
    default: return big ? bps<PH, 384, big_applies<PH>()>() : bps<PH, 384, false>();
  }
}

cudaError_t launch_fk_phase(int phase, int sched, const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st) {
  if (sched < 0 || sched >= FK_NSCHED) sched = 0;
  switch (phase) {
    case PH_TOR: return launch_sched<PH_TOR>(sched, P, L, grid, st);
    case PH_SPH: return launch_sched<PH_SPH>(sched, P, L, grid, st);
    case PH_ADJ: return launch_sched<PH_ADJ>(sched, P, L, grid, st);
    default:
      fk_setup_kernel<<<grid, 128, 0, st>>>(P, L);
      return cudaGetLastError();
  }
}

int fk_phase_blocks_per_sm(int phase, int sched) {
  if (sched < 0 || sched >= FK_NSCHED) sched = 0;
  switch (phase) {
    case PH_TOR: return bps_sched<PH_TOR>(sched);
    case PH_SPH: return bps_sched<PH_SPH>(sched);
    case PH_ADJ: return bps_sched<PH_ADJ>(sched);
    default: return 8;
  }
}

int fk_lane_slot_per_node() { return LaneLayout::PER_NODE; }

}  // namespace GEM_NS
