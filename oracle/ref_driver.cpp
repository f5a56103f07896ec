// ref_driver.cpp -- C entry point around the reference's own CPU solver.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.py compiles this file together
// with the unmodified reference sources CPU_Solver/*.cpp and Auxiliary/*.cpp
// (read in place from the reference tree, never copied) into one shared
// object per compile-time configuration under oracle/_ref/.  The object
// exports three C symbols so that tests can call CPU_PoissonGravitySolver
// (CPU_Solver/CPU_PoissonGravitySolver.cpp:133-168) on arrays from numpy.
//
// The reference prints one "Patch %4d : number of iterations = %3d" line per
// patch to stdout from inside the SOR loop (CPU_PoissonSolver_SOR.cpp:288).
// ref_run() sends fd 1 to a temporary file for the duration of the call and,
// when asked, parses those lines back into a per-patch iteration array.
#include "GAMER.h"

#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>

#define EXPORT extern "C" __attribute__((visibility("default")))

EXPORT int ref_config(int *ghost, int *gra_ghost, int *real_size, int *scheme, int *patch_size)
{
   *ghost = POT_GHOST_SIZE;
   *gra_ghost = GRA_GHOST_SIZE;
   *real_size = (int)sizeof(real);
   *scheme = POT_SCHEME;
   *patch_size = PATCH_SIZE;
   return 0;
}

EXPORT int ref_max_threads(void)
{
#ifdef _OPENMP
   return omp_get_max_threads();
#else
   return 1;
#endif
}

// Runs CPU_PoissonGravitySolver on npatch_group*8 patches.  `iters` (may be
// NULL) receives the per-patch SOR iteration counts parsed from the
// reference's own report; entries stay -1 for patches it did not report.
EXPORT int ref_run(const void *rho, void *pot_in, void *pot_out, void *flu, int npatch_group,
                   double dt, double dh, int sor_min_iter, int sor_max_iter, double sor_omega,
                   int mg_max_iter, int mg_npre, int mg_npost, double mg_tol, double poi_coeff,
                   int int_scheme, int p5_gradient, int poisson, int gra_acc, int nthreads,
                   int *iters)
{
#ifdef _OPENMP
   if (nthreads > 0) omp_set_num_threads(nthreads);
#else
   (void)nthreads;
#endif
   const int npatch = 8 * npatch_group;
   if (iters)
      for (int p = 0; p < npatch; p++) iters[p] = -1;

   fflush(stdout);
   FILE *tmp = tmpfile();
   const int saved = dup(1);
   if (tmp == NULL || saved < 0) return 1;
   dup2(fileno(tmp), 1);

   CPU_PoissonGravitySolver((const real(*)[RHO_NXT][RHO_NXT][RHO_NXT])rho,
                            (real(*)[POT_NXT][POT_NXT][POT_NXT])pot_in,
                            (real(*)[GRA_NXT][GRA_NXT][GRA_NXT])pot_out,
                            (real(*)[5][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE])flu, npatch_group,
                            (real)dt, (real)dh, sor_min_iter, sor_max_iter, (real)sor_omega,
                            mg_max_iter, mg_npre, mg_npost, (real)mg_tol, (real)poi_coeff,
                            (IntScheme_t)int_scheme, p5_gradient != 0, poisson != 0, gra_acc != 0);

   fflush(stdout);
   dup2(saved, 1);
   close(saved);

   if (iters) {
      rewind(tmp);
      char line[256];
      while (fgets(line, sizeof line, tmp)) {
         int p, it;
         if (sscanf(line, "Patch %d : number of iterations = %d", &p, &it) == 2 && p >= 0 &&
             p < npatch)
            iters[p] = it;
      }
   }
   fclose(tmp);
   return 0;
}
