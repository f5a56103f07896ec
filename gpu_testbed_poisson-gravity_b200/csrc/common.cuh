// common.cuh -- shared device helpers for the per-patch Poisson-gravity kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gpg {

// ---------------------------------------------------------------------------
// IEEE-exact arithmetic.  The reference CPU solvers evaluate every expression
// as separate float/double operations in source order (gcc, baseline x86-64,
// no FMA).  These wrappers are never contracted into FMA by nvcc, so a kernel
// that keeps the reference's operand order produces bit-identical values.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float absval(float a) { return fabsf(a); }
__device__ __forceinline__ double absval(double a) { return fabs(a); }
// a / b with IEEE round-to-nearest (the reference's `(real)0.5/rho`).
__device__ __forceinline__ float divide(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double divide(double a, double b) { return __ddiv_rn(a, b); }

// ---------------------------------------------------------------------------
// Patch geometry (Header/Macro.h:53-61), compile-time in the ghost size G.
//   N     fine cube edge the solver works in: 8 + 2G (interior + 1 ghost layer)
//   M     interior edge = RHO_NXT = N - 2
//   PN    POT_NXT = 4 + 2*((G+3)/2)
//   U     POT_USELESS = G % 2 (layers of the interpolated array outside the cube)
// ---------------------------------------------------------------------------
template <int G>
struct Geo {
  static constexpr int N = 8 + 2 * G;
  static constexpr int M = N - 2;
  static constexpr int HALF = M / 2;
  static constexpr int POT_INT = (G + 3) / 2;
  static constexpr int PN = 4 + 2 * POT_INT;
  static constexpr int U = G % 2;
  static constexpr int RHO3 = M * M * M;
  static constexpr int PN3 = PN * PN * PN;
  // number of interior x-pairs per patch (one SOR lane each)
  static constexpr int NPAIR = HALF * M;
};

// Colour of fine-cube cell (x, y, z): the SOR pass that updates it.  Pass 0 of
// the reference (CPU_PoissonSolver_SOR.cpp:220-270) updates interior cells
// whose rho index (x-1, y-1, z-1) has an even sum.
__host__ __device__ constexpr int colour(int x, int y, int z) { return (x + y + z + 1) & 1; }

// Team barrier: a warp barrier for one-warp teams, a named barrier (id = team
// index + 1, count = team threads) otherwise, so teams of one CTA that stop
// at different iterations never wait for each other.
template <int TEAM>
__device__ __forceinline__ void team_sync(int team) {
  if constexpr (TEAM == 32) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(TEAM) : "memory");
  }
}

__device__ __forceinline__ double warp_sum(double v) {
  // xor butterfly: every lane ends with the same bits (a+b == b+a exactly)
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

// Kernel arguments shared by the Poisson kernels (values already rounded to
// `real` exactly where the reference rounds them).
template <typename T>
struct SolveArgs {
  const T *rho;
  const T *pot_in;
  T *pot_out;
  T *flu;
  const T *guess;
  int32_t *iters;
  double *resid;
  int64_t npatch;
  T sor_const;      // Poi_Coeff*dh*dh        (CPU_PoissonSolver_SOR.cpp:51)
  T omega_6;        // Omega/6                (CPU_PoissonSolver_SOR.cpp:52)
  T gra_const;      // dt/(2dh) or dt/(12dh)  (CPU_GravitySolver.cpp:23)
  T dh;
  T poi_coeff;
  T mg_tol;
  double sor_tol;   // relative L1 tolerance (GPG_STOP_TOLERANCE)
  int min_iter, max_iter;
  int mg_max_iter, mg_npre, mg_npost;
  int int_scheme;   // 4 CQUAD, 5 QUAD
  int init_mode;    // GPG_INIT_*
  int stop_mode;    // GPG_STOP_*
  int gra_ghost;    // 0..2
  int gra_acc;      // fused gravity update
  int p5;           // 5-point gradient
};

}  // namespace gpg
