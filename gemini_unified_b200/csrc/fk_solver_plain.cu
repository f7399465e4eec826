// FK solver, parity build: arithmetic in the reference's operation order, no
// FMA contraction (compiled with --fmad=false).
#define GEM_NS gem_plain
#define GEM_FAST 0
#include "fk_solver_tu.cuh"
