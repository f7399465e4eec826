// One build of the FK solver kernels: the including file defines GEM_NS and
// GEM_FAST (gem_plain / 0 and gem_fast / 1).
#include <cuda_runtime.h>

#include "fk_kernel.h"
#include "fk_solver.cuh"
#include "fk_phases.cuh"

namespace GEM_NS {
template <int PH>
static size_t phase_smem() {
  return (size_t)(FK_BLOCK_PH[PH] / 32) * PhaseDiag<PH>::L * PhaseNV<PH>::NV * 32 * sizeof(double2);
}

template <int PH>
static cudaError_t phase_attr() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(fk_phase_kernel<PH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)phase_smem<PH>());
  if (e == cudaSuccess) done = true;
  return e;
}

template <int PH>
static cudaError_t launch_ph(const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st) {
  cudaError_t e = phase_attr<PH>();
  if (e != cudaSuccess) return e;
  fk_phase_kernel<PH><<<grid, FK_BLOCK_PH[PH], phase_smem<PH>(), st>>>(P, L);
  return cudaGetLastError();
}

cudaError_t launch_fk_phase(int phase, const FKStatic& P, const FKLaunch& L, int grid, cudaStream_t st) {
  switch (phase) {
    case PH_TOR: return launch_ph<PH_TOR>(P, L, grid, st);
    case PH_SPH: return launch_ph<PH_SPH>(P, L, grid, st);
    case PH_ADJ: return launch_ph<PH_ADJ>(P, L, grid, st);
    default:
      fk_setup_kernel<<<grid, 128, 0, st>>>(P, L);
      return cudaGetLastError();
  }
}

template <int PH>
static int bps() {
  if (phase_attr<PH>() != cudaSuccess) return 1;
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fk_phase_kernel<PH>, FK_BLOCK_PH[PH], phase_smem<PH>()) != cudaSuccess) return 1;
  return nb < 1 ? 1 : nb;
}

int fk_phase_blocks_per_sm(int phase) {
  switch (phase) {
    case PH_TOR: return bps<PH_TOR>();
    case PH_SPH: return bps<PH_SPH>();
    case PH_ADJ: return bps<PH_ADJ>();
    default: return 8;
  }
}

int fk_lane_slot_per_node() { return LaneLayout::PER_NODE; }

}  // namespace GEM_NS
