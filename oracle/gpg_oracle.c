/*
 * gpg_oracle.c -- CPU oracle for the per-patch Poisson-gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * CPU solvers (CPU_Solver/CPU_PoissonSolver_SOR.cpp, CPU_PoissonSolver_MG.cpp,
 * CPU_GravitySolver.cpp, CPU_PoissonGravitySolver.cpp) with runtime sizes.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
 * as the checker; the library never links or calls it.
 *
 * Parity pin: tests/golden/ holds outputs of the reference's own CPU code
 * (compiled from its sources by oracle/build_ref.py) and tests check this
 * restatement against them bit for bit.
 *
 * Build: gcc -O3 -fopenmp -fPIC -shared (baseline x86-64, no -march and no
 * -ffast-math: FMA contraction or reassociation would break bit parity).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/gpg.h"

#define T float
#define SFX f32
#define TABS fabsf
#include "gpg_oracle_body.h"
#undef T
#undef SFX
#undef TABS

#define T double
#define SFX f64
#define TABS fabs
#include "gpg_oracle_body.h"
#undef T
#undef SFX
#undef TABS

/* Interpolation alone, for unit tests: coarse [POT_NXT]^3 -> cube [N]^3. */
void oracle_interp_cube_f32(const float *cp, float *cube, int g, int s) { oracle_interp_f32(cp, cube, g, s); }
void oracle_interp_cube_f64(const double *cp, double *cube, int g, int s) { oracle_interp_f64(cp, cube, g, s); }

int oracle_max_threads(void)
{
#ifdef _OPENMP
   return omp_get_max_threads();
#else
   return 1;
#endif
}
