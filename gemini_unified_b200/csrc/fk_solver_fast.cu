// FK solver, fast build: FMA contraction, division-free spline evaluation,
// reciprocal-based complex inverses and squared-modulus error test
// (compiled with --fmad=true).
#define GEM_NS gem_fast
#define GEM_FAST 1
#include "fk_solver_tu.cuh"
