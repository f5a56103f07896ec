// sor_kernel.cuh -- red-black SOR for one patch per team, fused with the
// coarse->fine interpolation, the L1 residual test, the output copy and
// (optionally) the gravity update.
//
// Semantics follow the reference CPU solver CPU_PoissonSolver_SOR.cpp:43-320:
//   a. interpolate the coarse potential into the cube (initial guess + ghosts)
//   b. sweeps: pass p updates interior cells whose rho index has parity p,
//        R = phi(z+1)+phi(z-1)+phi(y+1)+phi(y-1)+phi(x+1)+phi(x-1) - 6phi - Const rho
//        phi += Omega/6 R,   Total += |R|      (Total accumulated in double)
//      stop after the first sweep whose Total grows once Iter+1 >= Min_Iter
//      (or, in tolerance mode, once Total <= tol * sum|Const rho|); cap Max_Iter
//   c. copy the GRA_NXT^3 window of the cube to pot_out
//
// B200 layout.  A team of TEAM = ceil(M*M/2 / 32)*32 threads owns a patch;
// lane (y, h) owns the interior x-pair {2h+1, 2h+2} of row y at every height
// and keeps both columns in registers, split by colour: v[c][z] is the lane's
// colour-c cell at height z (one cell of each colour per pair and height).
// A pass of colour p therefore updates v[p][z] for all heights and reads
//   - z neighbours            v[1-p][z+-1]      (own registers)
//   - one x neighbour         v[1-p][z]         (own registers, the pair mate)
//   - other x and both y      shared memory     (3 loads)
// and publishes the new value with one store.  The shared copy of the cube is
// red/black split with a row pitch of HALF words, so a warp's 32 lanes touch
// 32 consecutive words per access.  Two team barriers per sweep (one per
// pass); the residual reduction rides on the second.
#pragma once

#include <cfloat>

#include "common.cuh"
#include "gravity.cuh"
#include "interp.cuh"

namespace gpg {

template <typename T, int G>
struct SorSmem {
  using g = Geo<G>;
  // per team: cube + coarse staging + double-buffered warp partial sums
  static constexpr int ALIGN = 16;
  static constexpr size_t cube_bytes = sizeof(T) * g::CUBE;
  static constexpr size_t coarse_bytes = sizeof(T) * g::PN3;
  static constexpr size_t part_bytes = sizeof(double) * 2 * g::NWARP;
  static constexpr size_t round(size_t b) { return (b + ALIGN - 1) / ALIGN * ALIGN; }
  static constexpr size_t team_bytes = round(cube_bytes) + round(coarse_bytes) + round(part_bytes);
};

template <typename T, int G, int PPC>
__global__ void __launch_bounds__(PPC *Geo<G>::TEAM)
    sor_kernel(const SolveArgs<T> a) {
  using g = Geo<G>;
  constexpr int N = g::N, M = g::M, HALF = g::HALF, TEAM = g::TEAM, NWARP = g::NWARP, PP = g::PP;
  constexpr int PN3 = g::PN3, NPAIR = g::NPAIR;
  using S = SorSmem<T, G>;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int team = threadIdx.x / TEAM, tid = threadIdx.x - team * TEAM;
  const int lane = tid & 31, warp = tid >> 5;
  unsigned char *tb = smem_raw + team * S::team_bytes;
  T *s_cube = reinterpret_cast<T *>(tb);
  T *s_coarse = reinterpret_cast<T *>(tb + S::round(S::cube_bytes));
  double *s_part = reinterpret_cast<double *>(tb + S::round(S::cube_bytes) + S::round(S::coarse_bytes));

  const int64_t P = int64_t(blockIdx.x) * PPC + team;
  if (P >= a.npatch) return;  // whole team leaves together

  // ---- stage the coarse potential and interpolate into the cube ----------
  {
    const T *src = a.pot_in + P * PN3;
    for (int t = tid; t < PN3; t += TEAM) s_coarse[t] = src[t];
  }
  team_sync<TEAM>(team);
  interpolate<T, G, TEAM>(s_coarse, tid, a.int_scheme,
                          [s_cube](int x, int y, int z, T v) { s_cube[cube_addr<G>(x, y, z)] = v; });
  team_sync<TEAM>(team);

  // ---- lane -> (y, h) pair, registers -------------------------------------
  const bool active = tid < NPAIR;
  const int q = active ? tid : 0;
  const int y = 1 + q / HALF, h = q - (y - 1) * HALF;
  const int own = y * HALF + h;  // in-plane offset of this lane's pair
  // in-plane offset of the x neighbour outside the pair, for the cell on the
  // left (x = 2h+1, neighbour x = 2h) and on the right (x = 2h+2, x = 2h+3)
  const int xo_left = (h == 0) ? N * HALF + y : own - 1;
  const int xo_right = (h == HALF - 1) ? N * HALF + N + y : own + 1;
  // colour-c cell at height z sits on the left iff (y + z + c) is even
  const int xo_even = (y & 1) ? xo_right : xo_left;  // used when (z + c) is even
  const int xo_odd = (y & 1) ? xo_left : xo_right;   // used when (z + c) is odd
  const bool left_even = !(y & 1);

  T v[2][N];
  T crho[2][M];
  double cr_sum = 0.0;
  {
    const T *rho = a.rho + P * g::RHO3;
    const T *guess = a.guess ? a.guess + P * g::RHO3 : nullptr;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
#pragma unroll
      for (int z = 0; z < N; ++z) v[c][z] = s_cube[(c * N + z) * PP + own];
#pragma unroll
      for (int z = 1; z <= M; ++z) {
        const bool left = (((z + c) & 1) == 0) == left_even;
        const int x = left ? 2 * h + 1 : 2 * h + 2;
        const int idx = ((z - 1) * M + (y - 1)) * M + (x - 1);
        crho[c][z - 1] = active ? mul(a.sor_const, rho[idx]) : T(0);
        cr_sum += (double)absval(crho[c][z - 1]);
        if (a.init_mode != 0) {
          const T init = (a.init_mode == 2 && active) ? guess[idx] : T(0);
          v[c][z] = init;
        }
      }
    }
  }
  if (a.init_mode != 0) {
    // the cube's interior must hold the new initial guess before any neighbour reads
    if (active) {
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int z = 1; z <= M; ++z) s_cube[(c * N + z) * PP + own] = v[c][z];
    }
  }
  double tol_abs = 0.0;
  if (a.stop_mode == 1) {
    cr_sum = warp_sum(cr_sum);
    if constexpr (NWARP > 1) {
      if (lane == 0) s_part[warp] = cr_sum;
    }
    team_sync<TEAM>(team);
    if constexpr (NWARP > 1) {
      cr_sum = s_part[0];
#pragma unroll
      for (int w = 1; w < NWARP; ++w) cr_sum += s_part[w];
    }
    tol_abs = a.sor_tol * cr_sum;
  }
  team_sync<TEAM>(team);

  // ---- SOR sweeps ---------------------------------------------------------
  const T omega_6 = a.omega_6;
  double total_old = (double)FLT_MAX, last = 0.0;
  int iter;
  for (iter = 0; iter < a.max_iter; ++iter) {
    double acc = 0.0;
#pragma unroll
    for (int p = 0; p < 2; ++p) {
      if (active) {
        const T *nb = s_cube + (1 - p) * N * PP;  // planes of the other colour
        T *mine = s_cube + p * N * PP;
#pragma unroll
        for (int z = 1; z <= M; ++z) {
          const bool even = ((z + p) & 1) == 0;
          const bool left = even == left_even;
          const T xo = nb[z * PP + (even ? xo_even : xo_odd)];
          const T yp = nb[z * PP + own + HALF];
          const T ym = nb[z * PP + own - HALF];
          const T mate = v[1 - p][z];
          const T xp = left ? mate : xo, xm = left ? xo : mate;
          const T s = add(add(add(add(add(v[1 - p][z + 1], v[1 - p][z - 1]), yp), ym), xp), xm);
          const T r = sub(sub(s, mul(T(6), v[p][z])), crho[p][z - 1]);
          v[p][z] = add(v[p][z], mul(omega_6, r));
          mine[z * PP + own] = v[p][z];
          acc += (double)absval(r);
        }
      }
      if (p == 0) team_sync<TEAM>(team);
    }
    acc = warp_sum(acc);
    if constexpr (NWARP > 1) {
      if (lane == 0) s_part[(iter & 1) * NWARP + warp] = acc;
    }
    team_sync<TEAM>(team);
    double total = acc;
    if constexpr (NWARP > 1) {
      const double *pp = s_part + (iter & 1) * NWARP;
      total = pp[0];
#pragma unroll
      for (int w = 1; w < NWARP; ++w) total += pp[w];
    }
    last = total;
    if (iter + 1 >= a.min_iter) {
      if (a.stop_mode == 0 ? (total > total_old) : (total <= tol_abs)) {
        ++iter;
        break;
      }
    }
    total_old = total;
  }
  if (tid == 0) {
    if (a.iters) a.iters[P] = iter;
    if (a.resid) a.resid[P] = last;
  }

  // ---- output window (CPU_PoissonSolver_SOR.cpp:305-311) ------------------
  {
    const int GN = 8 + 2 * a.gra_ghost, shift = G - a.gra_ghost, GN3 = GN * GN * GN;
    T *dst = a.pot_out + P * GN3;
    for (int t = tid; t < GN3; t += TEAM) {
      const int i = t % GN, j = (t / GN) % GN, k = t / (GN * GN);
      dst[t] = s_cube[cube_addr<G>(i + shift, j + shift, k + shift)];
    }
  }
  // ---- fused gravity update (CPU_GravitySolver.cpp:34-79) -----------------
  if (a.gra_acc) {
    gravity_patch<T, TEAM>(a.flu + P * 5 * 512, tid, a.gra_const, a.p5,
                           [s_cube](int i, int j, int k) { return s_cube[cube_addr<G>(i + G, j + G, k + G)]; });
  }
}

}  // namespace gpg
