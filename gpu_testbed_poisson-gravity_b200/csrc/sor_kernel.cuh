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
//      (or, in tolerance mode, once Total <= tol * sum|Const rho| -- or <= tol
//      in absolute-tolerance mode, or <= tol * sum|phi_interp| over the
//      updated cells in potential-tolerance mode); cap Max_Iter
//   c. copy the GRA_NXT^3 window of the cube to pot_out
//
// B200 layout.  A team of 1-8 warps owns a patch.  A lane owns the interior
// x-pair {2h+1, 2h+2} of Y rows (Y = 1: row y; Y = 2: rows y, y+1 with y odd)
// at every height, or at half of the heights in the column-split variants
// (Z = 2), and keeps those columns in registers, split by colour: v[c][z] is
// the lane's colour-c cell at height z (each pair has one cell of each colour
// per height).  A pass of colour p updates v[p][z] for all heights and reads
//   - z neighbours            v[1-p][z+-1]      (own registers)
//   - one x neighbour         v[1-p][z]         (own registers, the pair mate)
//   - Y = 1: other x and both y   shared memory (3 loads)
//   - Y = 2: the y neighbour inside the lane's two rows comes from registers
//            too, so each cell reads 2 values from shared memory
// and publishes the new value with one store.
//
// Shared cube: plane (colour c, height z) has N rows of pitch P; slot s of a
// row holds the colour-c cell among x = 2s-1, 2s (slot 0: x = 0 ghost, slot
// H+1: x = N-1 ghost), so every x-neighbour read is own slot +-1.  Y = 1 lanes
// are grouped by row parity (odd rows first, R lanes per row), which makes
// the read direction uniform inside a shared-memory wavefront; P is chosen per
// (precision, ghost size, layout) so that the accesses of a wavefront fall in
// distinct banks.  Two team barriers per sweep (one per pass); the residual
// reduction rides on the second.
#pragma once

#include <cfloat>
#include <type_traits>

#include "common.cuh"
#include "gravity.cuh"
#include "interp.cuh"
#include "tc_common.cuh"

namespace gpg {

// Lane mapping and row pitch per (precision, ghost size, layout).
// Z = 1: a lane owns its pair's whole column (heights 1..M).  Z = 2: the column
// is split in two halves owned by two lanes (heights 1..M/2 and M/2+1..M), so
// a team has twice the lanes with half the registers each, at one extra shared
// load per pass and row for the neighbour across the split.
// Y = 2: a lane owns the pair in two adjacent rows (odd y and y+1): 3 shared
// accesses per cell update instead of 4, at twice the registers per lane.
// R (lanes per row / row pair), P, the plane padding PADZ and the block
// rounding U come from an exhaustive search of a wavefront model of one sweep
// (per warp instruction, 32-bit: largest number of distinct words in one bank;
// 64-bit: the same per half-warp); e.g. FP64 g5 1024 wavefronts per
// patch-sweep (Y1 Z1) -> 800 (Y2 Z2), FP64 g3 576 (Y1 Z1) -> 480 (Y1 Z2) -> 380
// (Y2 Z2).
template <typename T, int G, int Z = 1, int Y = 1>
struct SorCfg {
  using g = Geo<G>;
  static constexpr bool F64 = sizeof(T) == 8;
  static_assert(Z == 1 || Z == 2, "a column is owned by one or two lanes");
  static_assert(Y == 1 || Y == 2, "a lane owns one or two rows");
  static constexpr int MH = g::M / Z;  // heights per lane
  // lanes per row (Y = 1) or row pair (Y = 2); R > HALF pads rows so that
  // wavefronts hold whole rows (FP64 g2, Y = 1: 6 lanes for 5 pairs makes
  // every 64-bit access of a half-warp conflict-free)
  static constexpr int R = Y == 1 ? ((G == 1) ? 4 : (G == 2 ? (F64 ? 6 : 5) : ((G == 3 && Z == 2) ? 6 : 8)))
                                  : ((G == 1) ? 4 : (G == 2 ? (F64 ? 6 : 5) : ((G == 3 && F64) ? 6 : 8)));
  // row pitch (words)
  static constexpr int P = Y == 1 ? ((G == 1) ? ((F64 || Z == 2) ? 6 : 12)
                                              : (G == 2 ? (F64 ? 11 : 13)
                                                        : (G == 3 ? (F64 ? 11 : (Z == 2 ? 19 : 12)) : 12)))
                                  : ((G == 1) ? 6
                                              : (G == 2 ? (F64 ? 11 : 13)
                                                        : (G == 3 ? (F64 ? 11 : (Z == 2 ? 13 : 12)) : 12)));
  // plane padding (words)
  static constexpr int PADZ = Z == 1 ? 0
                                     : (Y == 1 ? (G == 3 ? 2 : (G == 4 ? 1 : 0))
                                               : (G == 3 ? (F64 ? 2 : 14) : ((G == 4 && F64) ? 1 : 0)));
  // rounding of a lane block
  static constexpr int U = Y == 1 ? (Z == 1 ? 16 : (G == 2 ? (F64 ? 4 : 8) : (G == 3 ? 8 : 1)))
                                  : (Z == 1 ? 1
                                            : (G == 2 ? (F64 ? 4 : 8)
                                                      : (G == 3 ? (F64 ? 8 : 1) : (G == 4 ? (F64 ? 32 : 16) : 1))));
  static constexpr int ROWS = g::M / 2;  // rows per parity class (Y = 1) = row pairs (Y = 2)
  // lanes per block: (class, half) blocks for Y = 1, (half) blocks for Y = 2
  static constexpr int BLOCK = ((ROWS * R + U - 1) / U) * U;
  static constexpr int NBLOCK = (Y == 1 ? 2 : 1) * Z;
  static constexpr int TEAM = ((NBLOCK * BLOCK + 31) / 32) * 32;
  static constexpr int NWARP = TEAM / 32;
  // Y = 1, Z = 1: every warp holds lanes of one row-parity class only, so the
  // side of a lane's colour-c cell (left / right of its pair) is warp-uniform
  // and the passes are compiled per side.  FP64 only: there it frees registers
  // (FP64 g5 phased 202 -> 166, a third team per SM) and each x select is two
  // instructions; the FP32 kernels measured 9-15 % slower at g4/g5 with it.
  static constexpr bool UNIFORM = Y == 1 && Z == 1 && F64 && BLOCK % 32 == 0;
  // Y = 2 with an odd MH: the upper half's cells sit on the other side; with
  // whole warps per half that side is warp-uniform and compiled per half
  static constexpr bool HALF_UNIFORM = Y == 2 && Z == 2 && (MH & 1) && BLOCK % 32 == 0;
  static constexpr int PP = g::N * P + PADZ;  // plane pitch
  static constexpr int CUBE = 2 * g::N * PP;
  // register words of a lane's columns and Const*rho; layouts far beyond the
  // register file are not built
  static constexpr int STATE_WORDS = Y * 2 * (2 * MH + 2) * (F64 ? 2 : 1);
  static constexpr bool FITS = Y == 1 || STATE_WORDS <= 180;
  static_assert(R >= g::HALF && P >= g::HALF + 2, "row layout");
  static_assert(g::M % Z == 0, "column halves");

  __device__ static __forceinline__ int addr(int x, int y, int z) {
    return (colour(x, y, z) * g::N + z) * PP + y * P + ((x + 1) >> 1);
  }
};

template <typename T, int G, int Z = 1, int Y = 1>
struct SorSmem {
  using C = SorCfg<T, G, Z, Y>;
  static constexpr size_t round(size_t b) { return (b + 15) / 16 * 16; }
  static constexpr size_t cube_bytes = sizeof(T) * C::CUBE;
  static constexpr size_t part_bytes = sizeof(double) * 2 * C::NWARP;
  static constexpr size_t team_bytes = round(cube_bytes) + round(part_bytes);
};

// A lane's fixed addressing for the passes.  Heights are local to the lane's
// column half: local zz = 0..MH+1 is global z = zbase + zz, and `zoff` =
// zbase * PP.  left_even / xo_even / xo_odd refer to the parity of the LOCAL
// height (for an odd zbase the global parity flips, folded in here).
struct SorLane {
  int own;         // in-plane offset of the lane's pair slot (first row for Y = 2)
  int xo_even;     // Y = 1: outside x neighbour slot when (zz + c) is even
  int xo_odd;      // ... when odd
  int zoff;        // plane offset of the lane's column half
  int zh;          // column half (0 / 1); always 0 for Z = 1
  bool left_even;  // colour-c cell on the left of the pair iff (zz + c) even
                   // (Y = 2: of the lane's second, even row)
};

// Z = 2: reload the other-colour neighbour across the split (owned by the
// other half's lane, updated in the previous pass) for each of the lane's rows.
template <typename T, int MH, int PP, int P, int Y, int p>
__device__ __forceinline__ void sor_reload_split(T (&v)[Y][2][MH + 2], const T *nb, const SorLane &ln) {
#pragma unroll
  for (int r = 0; r < Y; ++r) {
    const T b = nb[(ln.zh ? 0 : MH + 1) * PP + ln.own + r * P];
    if (ln.zh)
      v[r][1 - p][0] = b;
    else
      v[r][1 - p][MH + 1] = b;
  }
}

// One pass of colour p over every height of the lane's column (half), Y = 1:
// reads the other colour (registers + 3 shared loads per cell), updates
// v[p][*] in registers, then publishes them.  SUM: accumulate |R| into acc4
// (skipped for sweeps whose residual total the stopping rule never looks at).
// SIDE: -1 = the lane's side (left_even) is a run-time value; 0 / 1 = it is
// known at compile time (warp-uniform layouts dispatch once per pass), which
// turns the x operand selects and the outside-neighbour address into
// constants.
template <typename T, int G, int Z, bool PHASED, int p, bool SUM, int SIDE>
__device__ __forceinline__ void sor_pass(T (&vv)[1][2][SorCfg<T, G, Z>::MH + 2],
                                         const T (&cr)[1][2][SorCfg<T, G, Z>::MH], T *s_cube, const SorLane &ln,
                                         T omega_6, double (&acc4)[4]) {
  using C = SorCfg<T, G, Z>;
  constexpr int N = Geo<G>::N, MH = C::MH, P = C::P, PP = C::PP;
  T(&v)[2][MH + 2] = vv[0];
  const T(&crho)[2][MH] = cr[0];
  const int own = ln.own;
  const T *nb = s_cube + (1 - p) * N * PP + ln.zoff;  // planes of the other colour
  T *mine = s_cube + p * N * PP + ln.zoff;
  const bool left_even = SIDE < 0 ? ln.left_even : SIDE == 1;
  // outside x neighbour: slot own-1 for a left cell, own+1 for a right one
  const int xo_even = SIDE < 0 ? ln.xo_even : (SIDE == 1 ? own - 1 : own + 1);
  const int xo_odd = SIDE < 0 ? ln.xo_odd : (SIDE == 1 ? own + 1 : own - 1);
  if constexpr (Z == 2) sor_reload_split<T, MH, PP, P, 1, p>(vv, nb, ln);
  // all reads of the pass come from the other colour's planes and all writes
  // go to this colour's planes, so the MH updates are independent; the stores
  // follow all of them
  if constexpr (PHASED) {
    // phase by phase across all heights, keeping the reference's operand
    // order within each cell
    T sum[MH];
#pragma unroll
    for (int z = 1; z <= MH; ++z) sum[z - 1] = add(v[1 - p][z + 1], v[1 - p][z - 1]);
#pragma unroll
    for (int z = 1; z <= MH; ++z) sum[z - 1] = add(sum[z - 1], nb[z * PP + own + P]);
#pragma unroll
    for (int z = 1; z <= MH; ++z) sum[z - 1] = add(sum[z - 1], nb[z * PP + own - P]);
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const bool even = ((z + p) & 1) == 0;
      const bool left = even == left_even;
      const T xo = nb[z * PP + (even ? xo_even : xo_odd)];
      const T mate = v[1 - p][z];
      const T xp = left ? mate : xo, xm = left ? xo : mate;
      sum[z - 1] = add(add(sum[z - 1], xp), xm);
    }
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const T res = sub(sub(sum[z - 1], mul(T(6), v[p][z])), crho[p][z - 1]);
      v[p][z] = add(v[p][z], mul(omega_6, res));
      if constexpr (SUM) acc4[z & 3] += (double)absval(res);
    }
  } else {
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const bool even = ((z + p) & 1) == 0;
      const bool left = even == left_even;
      const T xo = nb[z * PP + (even ? xo_even : xo_odd)];
      const T yp = nb[z * PP + own + P];
      const T ym = nb[z * PP + own - P];
      const T mate = v[1 - p][z];
      const T xp = left ? mate : xo, xm = left ? xo : mate;
      const T sm = add(add(add(add(add(v[1 - p][z + 1], v[1 - p][z - 1]), yp), ym), xp), xm);
      const T res = sub(sub(sm, mul(T(6), v[p][z])), crho[p][z - 1]);
      v[p][z] = add(v[p][z], mul(omega_6, res));
      if constexpr (SUM) acc4[z & 3] += (double)absval(res);
    }
  }
#pragma unroll
  for (int z = 1; z <= MH; ++z) mine[z * PP + own] = v[p][z];
}

// Y = 2 pass: rows y0 (odd) and y1 = y0+1 of the lane's pair.  Per height the
// colour-p cells are (x0, y0) and (x1, y1), x0 != x1 the two x of the pair;
// the other-colour cells the lane holds are (x1, y0) = v[0][1-p] and
// (x0, y1) = v[1][1-p]: the x mate of one cell and the in-lane y neighbour of
// the other.  Shared memory supplies the y0-1 / y1+1 neighbours and the two
// outside x neighbours.  Operand order per cell as the reference's.
template <typename T, int G, int Z, bool PHASED, int p, bool SUM, int SIDE>
__device__ __forceinline__ void sor_pass2(T (&v)[2][2][SorCfg<T, G, Z, 2>::MH + 2],
                                          const T (&crho)[2][2][SorCfg<T, G, Z, 2>::MH], T *s_cube,
                                          const SorLane &ln, T omega_6, double (&acc4)[4]) {
  using C = SorCfg<T, G, Z, 2>;
  constexpr int N = Geo<G>::N, MH = C::MH, P = C::P, PP = C::PP;
  const int own0 = ln.own, own1 = ln.own + P;
  const T *nb = s_cube + (1 - p) * N * PP + ln.zoff;
  T *mine = s_cube + p * N * PP + ln.zoff;
  if constexpr (Z == 2) sor_reload_split<T, MH, PP, P, 2, p>(v, nb, ln);
  // row y1's colour-c cell is on the left iff ((zz + c) even) == left_even and
  // row y0's is then on the right; left_even is true at compile time unless an
  // odd MH makes it depend on the column half
  constexpr bool RT = (Z == 2) && (MH & 1);
  const bool le = SIDE >= 0 ? SIDE == 1 : (RT ? ln.left_even : true);
  // sum of the six neighbours of row r's colour-p cell at height z; yreg is
  // the y neighbour held in registers (y0+1 for row 0, y1-1 for row 1), ysm
  // the one read from shared memory
  auto nbsum = [&](int z, int r, T yreg, T ysm, bool left, T xo) -> T {
    const T mate = v[r][1 - p][z];
    const T yp = r == 0 ? yreg : ysm, ym = r == 0 ? ysm : yreg;
    const T xp = left ? mate : xo, xm = left ? xo : mate;
    return add(add(add(add(add(v[r][1 - p][z + 1], v[r][1 - p][z - 1]), yp), ym), xp), xm);
  };
  if constexpr (PHASED) {
    T s0[MH], s1[MH];
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const bool left1 = (((z + p) & 1) == 0) == le, left0 = !left1;
      const T xo0 = nb[z * PP + own0 + (left0 ? -1 : 1)];
      const T ym0 = nb[z * PP + own0 - P];
      const T xo1 = nb[z * PP + own1 + (left1 ? -1 : 1)];
      const T yp1 = nb[z * PP + own1 + P];
      s0[z - 1] = nbsum(z, 0, v[1][1 - p][z], ym0, left0, xo0);
      s1[z - 1] = nbsum(z, 1, v[0][1 - p][z], yp1, left1, xo1);
    }
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const T r0 = sub(sub(s0[z - 1], mul(T(6), v[0][p][z])), crho[0][p][z - 1]);
      const T r1 = sub(sub(s1[z - 1], mul(T(6), v[1][p][z])), crho[1][p][z - 1]);
      v[0][p][z] = add(v[0][p][z], mul(omega_6, r0));
      v[1][p][z] = add(v[1][p][z], mul(omega_6, r1));
      if constexpr (SUM) {
        acc4[z & 3] += (double)absval(r0);
        acc4[(z + 2) & 3] += (double)absval(r1);
      }
    }
  } else {
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const bool left1 = (((z + p) & 1) == 0) == le, left0 = !left1;
      const T xo0 = nb[z * PP + own0 + (left0 ? -1 : 1)];
      const T ym0 = nb[z * PP + own0 - P];
      const T xo1 = nb[z * PP + own1 + (left1 ? -1 : 1)];
      const T yp1 = nb[z * PP + own1 + P];
      const T r0 = sub(sub(nbsum(z, 0, v[1][1 - p][z], ym0, left0, xo0), mul(T(6), v[0][p][z])), crho[0][p][z - 1]);
      const T r1 = sub(sub(nbsum(z, 1, v[0][1 - p][z], yp1, left1, xo1), mul(T(6), v[1][p][z])), crho[1][p][z - 1]);
      v[0][p][z] = add(v[0][p][z], mul(omega_6, r0));
      v[1][p][z] = add(v[1][p][z], mul(omega_6, r1));
      if constexpr (SUM) {
        acc4[z & 3] += (double)absval(r0);
        acc4[(z + 2) & 3] += (double)absval(r1);
      }
    }
  }
#pragma unroll
  for (int z = 1; z <= MH; ++z) {
    mine[z * PP + own0] = v[0][p][z];
    mine[z * PP + own1] = v[1][p][z];
  }
}

template <typename T, int G, int Z, int Y, bool PHASED, int p, bool SUM>
__device__ __forceinline__ void sor_pass_any(T (&v)[Y][2][SorCfg<T, G, Z, Y>::MH + 2],
                                             const T (&crho)[Y][2][SorCfg<T, G, Z, Y>::MH], T *s_cube,
                                             const SorLane &ln, T omega_6, double (&acc4)[4]) {
  if constexpr (Y == 2) {
    if constexpr (SorCfg<T, G, Z, Y>::HALF_UNIFORM) {
      if (ln.left_even)  // warp-uniform branch
        sor_pass2<T, G, Z, PHASED, p, SUM, 1>(v, crho, s_cube, ln, omega_6, acc4);
      else
        sor_pass2<T, G, Z, PHASED, p, SUM, 0>(v, crho, s_cube, ln, omega_6, acc4);
    } else {
      sor_pass2<T, G, Z, PHASED, p, SUM, -1>(v, crho, s_cube, ln, omega_6, acc4);
    }
  } else if constexpr (SorCfg<T, G, Z, Y>::UNIFORM) {
    if (ln.left_even)  // warp-uniform branch
      sor_pass<T, G, Z, PHASED, p, SUM, 1>(v, crho, s_cube, ln, omega_6, acc4);
    else
      sor_pass<T, G, Z, PHASED, p, SUM, 0>(v, crho, s_cube, ln, omega_6, acc4);
  } else {
    sor_pass<T, G, Z, PHASED, p, SUM, -1>(v, crho, s_cube, ln, omega_6, acc4);
  }
}

// What a start-value hook sees: the lane's columns (v) and Const*rho (crho)
// in registers, the team's shared cube and the lane's place in it.
template <typename T, int G, int Z, int Y>
struct SorLaneState {
  using C = SorCfg<T, G, Z, Y>;
  T (&v)[Y][2][C::MH + 2];
  const T (&crho)[Y][2][C::MH];
  T *s_cube;
  const SorLane &ln;
  bool active;  // the lane owns cells
  int y, h, zbase;
};

// Solve patch P_ with the team `team` (thread `tid` of TEAM) whose shared
// memory starts at `tb` (SorSmem::team_bytes).  Used by the per-ghost-size
// kernel below and by the mixed-size persistent kernel (batch_kernel.cuh),
// so both produce the same bits for a patch.  `hook(state)` runs once the
// start values and the stopping bound are set, before the first sweep; it
// may change the interior (registers and shared cube) and must leave the
// team synchronised.  store == false skips every global write (a team that
// only keeps a CTA-wide schedule going).  STAGED: the patch's coarse
// potential and density come from `staged` in shared memory ([POT_NXT]^3
// then [RHO_NXT]^3) instead of global memory.
template <typename T, int G, bool PHASED, int Z, int Y, bool STAGED = false, typename Hook>
__device__ __forceinline__ void sor_solve_patch_with(const SolveArgs<T> &a, int64_t P_, int team, int tid,
                                                     unsigned char *tb, bool store, Hook &&hook,
                                                     const T *staged = nullptr) {
  using g = Geo<G>;
  using C = SorCfg<T, G, Z, Y>;
  using S = SorSmem<T, G, Z, Y>;
  constexpr int N = g::N, M = g::M, HALF = g::HALF, TEAM = C::TEAM, NWARP = C::NWARP;
  constexpr int P = C::P, PP = C::PP, R = C::R, MH = C::MH, BLOCK = C::BLOCK;
  const int lane = tid & 31, warp = tid >> 5;
  T *s_cube = reinterpret_cast<T *>(tb);
  double *s_part = reinterpret_cast<double *>(tb + S::round(S::cube_bytes));

  // ---- interpolate the coarse potential into the cube (reads via L1) -----
  interpolate<T, G, TEAM, !STAGED>(STAGED ? staged : a.pot_in + P_ * g::PN3, tid, a.int_scheme,
                                   [s_cube](int x, int y, int z, T v) { s_cube[C::addr(x, y, z)] = v; });
  team_sync<TEAM>(team);

  // ---- lane -> (rows, half, h) --------------------------------------------
  // Y = 1: blocks of BLOCK lanes (odd rows, half 0), [(odd rows, half 1)],
  // (even rows, half 0), [(even rows, half 1)]; Y = 2: (row pairs, half 0),
  // [(row pairs, half 1)]
  const int blk = tid / BLOCK, li = tid - blk * BLOCK, r = li / R, h0 = li - r * R;
  const bool active = (blk < C::NBLOCK) && (r < M / 2) && (h0 < HALF);
  const int cls = Y == 1 ? blk / Z : 0;
  const int y = active ? 2 * r + 1 + cls : 1, h = active ? h0 : 0;
  const int zbase = active ? (blk - cls * Z) * MH : 0;
  // colour-c cell at height z of row y sits on the left (x = 2h+1) iff
  // (y + z + c) is even; its outside x neighbour is then slot own-1, else
  // own+1.  For Y = 1 the row parity is fixed per class, so the direction is
  // uniform in a wavefront; for Y = 2 left_even describes the second row.
  const bool left_even_g = !((y + Y - 1) & 1);
  SorLane ln;
  ln.own = y * P + h + 1;
  ln.left_even = left_even_g != bool(zbase & 1);
  ln.xo_even = ln.left_even ? ln.own - 1 : ln.own + 1;
  ln.xo_odd = ln.left_even ? ln.own + 1 : ln.own - 1;
  ln.zoff = zbase * PP;
  ln.zh = zbase != 0;

  T v[Y][2][MH + 2];
  T crho[Y][2][MH];
  double cr_sum = 0.0;
  {
    const T *rho = STAGED ? staged + g::PN3 : a.rho + P_ * g::RHO3;
    const T *guess = a.guess ? a.guess + P_ * g::RHO3 : nullptr;
#pragma unroll
    for (int rr = 0; rr < Y; ++rr) {
      const int yr = y + rr;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
#pragma unroll
        for (int zz = 0; zz < MH + 2; ++zz) v[rr][c][zz] = s_cube[(c * N + zbase + zz) * PP + ln.own + rr * P];
#pragma unroll
        for (int zz = 1; zz <= MH; ++zz) {
          const int z = zbase + zz;
          const bool left = ((yr + z + c) & 1) == 0;
          const int x = left ? 2 * h + 1 : 2 * h + 2;
          const int idx = ((z - 1) * M + (yr - 1)) * M + (x - 1);
          T rv = T(0);
          if (active) {
            if constexpr (STAGED) rv = rho[idx];
            else rv = __ldg(rho + idx);
          }
          crho[rr][c][zz - 1] = active ? mul(a.sor_const, rv) : T(0);
          // tolerance scale: sum |Const rho| (mode 1) or sum |interpolated
          // phi| over the updated cells, before a start mode replaces it (3)
          cr_sum += (double)absval(a.stop_mode == 3 ? (active ? v[rr][c][zz] : T(0)) : crho[rr][c][zz - 1]);
          if (a.init_mode != 0) v[rr][c][zz] = (a.init_mode == 2 && active) ? __ldg(guess + idx) : T(0);
        }
      }
    }
  }
  if (a.init_mode != 0 && active) {
    // publish the new interior guess before any neighbour read
#pragma unroll
    for (int rr = 0; rr < Y; ++rr)
#pragma unroll
      for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int zz = 1; zz <= MH; ++zz) s_cube[(c * N + zbase + zz) * PP + ln.own + rr * P] = v[rr][c][zz];
  }
  double tol_abs = 0.0;
  if (a.stop_mode == 1 || a.stop_mode == 3) {
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
  } else if (a.stop_mode == 2) {
    tol_abs = a.sor_tol;
  }
  team_sync<TEAM>(team);
  hook(SorLaneState<T, G, Z, Y>{v, crho, s_cube, ln, active, y, h, zbase});

  // ---- SOR sweeps ---------------------------------------------------------
  const T omega_6 = a.omega_6;
  double total_old = (double)FLT_MAX, last = 0.0;
  int iter;
  for (iter = 0; iter < a.max_iter; ++iter) {
    // The stopping rule reads the residual total from sweep Min_Iter-2 on
    // (the growth test compares with the previous sweep) and the final
    // report needs the last sweep's; earlier sweeps skip the sums.
    const bool need = (iter + 2 >= a.min_iter) || (iter + 1 == a.max_iter);
    // four partial sums keep the accumulation off the critical path; they are
    // combined in a fixed order, so the total is deterministic and identical
    // for a patch solved alone or in a batch
    double acc4[4] = {0.0, 0.0, 0.0, 0.0};
    if (!need) {
      if (active) sor_pass_any<T, G, Z, Y, PHASED, 0, false>(v, crho, s_cube, ln, omega_6, acc4);
      team_sync<TEAM>(team);
      if (active) sor_pass_any<T, G, Z, Y, PHASED, 1, false>(v, crho, s_cube, ln, omega_6, acc4);
      team_sync<TEAM>(team);
      continue;
    }
    if (active) sor_pass_any<T, G, Z, Y, PHASED, 0, true>(v, crho, s_cube, ln, omega_6, acc4);
    team_sync<TEAM>(team);
    if (active) sor_pass_any<T, G, Z, Y, PHASED, 1, true>(v, crho, s_cube, ln, omega_6, acc4);
    double acc = (acc4[0] + acc4[1]) + (acc4[2] + acc4[3]);
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
  if (!store) return;
  if (tid == 0) {
    if (a.iters) a.iters[P_] = iter;
    if (a.resid) a.resid[P_] = last;
  }

  // ---- output window (CPU_PoissonSolver_SOR.cpp:305-311) ------------------
  // (edge GN a compile-time constant per GRA_GHOST_SIZE: the index split is
  // then multiply-shift, not division)
  auto window = [&](auto gg) {
    constexpr int GG = decltype(gg)::value, GN = 8 + 2 * GG, shift = G - GG, GN3 = GN * GN * GN;
    T *dst = a.pot_out + P_ * GN3;
    for (int t = tid; t < GN3; t += TEAM) {
      const int i = t % GN, j = (t / GN) % GN, k = t / (GN * GN);
      dst[t] = s_cube[C::addr(i + shift, j + shift, k + shift)];
    }
  };
  if (a.gra_ghost == 0)
    window(std::integral_constant<int, 0>{});
  else if (a.gra_ghost == 1)
    window(std::integral_constant<int, 1>{});
  else
    window(std::integral_constant<int, 2>{});
  // ---- fused gravity update (CPU_GravitySolver.cpp:34-79) -----------------
  if (a.gra_acc) {
    gravity_patch<T, TEAM>(a.flu + P_ * 5 * 512, tid, a.gra_const, a.p5,
                           [s_cube](int i, int j, int k) { return s_cube[C::addr(i + G, j + G, k + G)]; });
  }
}

template <typename T, int G, bool PHASED, int Z = 1, int Y = 1>
__device__ __forceinline__ void sor_solve_patch(const SolveArgs<T> &a, int64_t P_, int team, int tid,
                                                unsigned char *tb) {
  sor_solve_patch_with<T, G, PHASED, Z, Y>(a, P_, team, tid, tb, true, [](const auto &) {});
}

// PPC: teams (patches) per CTA.  PHASED: form the MH independent updates of a
// pass phase by phase across heights (more updates in flight, more registers)
// instead of height by height.  Z: lanes per pair column (1 or 2); Y: rows
// per lane (1 or 2).  The Y = 1, Z = 1 variants give identical bits; the
// others sum the residual in another order (the fields are the same whenever
// the sweep counts are).  The autotuner (gpg_set_sor_variant) picks per
// (precision, ghost size).
template <typename T, int G, int PPC, bool PHASED, int Z = 1, int Y = 1>
__global__ void __launch_bounds__(PPC *SorCfg<T, G, Z, Y>::TEAM)
    sor_kernel(const SolveArgs<T> a) {
  constexpr int TEAM = SorCfg<T, G, Z, Y>::TEAM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int team = threadIdx.x / TEAM, tid = threadIdx.x - team * TEAM;
  const int64_t P_ = int64_t(blockIdx.x) * PPC + team;
  if (P_ >= a.npatch) return;  // whole team leaves together
  sor_solve_patch<T, G, PHASED, Z, Y>(a, P_, team, tid, smem_raw + team * SorSmem<T, G, Z, Y>::team_bytes);
}

// ---------------------------------------------------------------------------
// Staged persistent variant: TPC teams per CTA, each team loops over patches
// (team t of CTA c takes patches c*TPC + t, + gridDim.x*TPC, ...) and bulk-
// copies its next patch's coarse potential and density into its shared
// staging buffer while it solves the current one, so the interpolation and
// the Const*rho loads read shared memory.  Same per-patch code as sor_kernel
// (same bits).  A staging wait that gives up (about a second) leaves that
// patch's iteration count at -1 and its residual NaN.
// ---------------------------------------------------------------------------
template <typename T, int G, int Z, int Y, int TPC>
struct StagedSmem {
  using S = SorSmem<T, G, Z, Y>;
  static constexpr int stage_elems = Geo<G>::PN3 + Geo<G>::RHO3;
  static constexpr size_t stage_bytes = S::round(sizeof(T) * stage_elems);
  static constexpr size_t team_bytes = S::team_bytes + stage_bytes + 16;
  static constexpr size_t bytes = TPC * team_bytes;
  // CTAs that shared memory lets an SM hold (228 KB, 1 KB reserved per CTA);
  // the register budget is bounded to match
  static constexpr int ctas_per_sm = (228 * 1024) / (bytes + 1024) < 1    ? 1
                                     : (228 * 1024) / (bytes + 1024) > 16 ? 16
                                                                          : (228 * 1024) / (bytes + 1024);
};

template <typename T, int G, bool PHASED, int Z, int Y, int TPC>
__global__ void __launch_bounds__(TPC *SorCfg<T, G, Z, Y>::TEAM, (StagedSmem<T, G, Z, Y, TPC>::ctas_per_sm))
    staged_sor_kernel(const SolveArgs<T> a) {
  using g = Geo<G>;
  using SS = StagedSmem<T, G, Z, Y, TPC>;
  constexpr int TEAM = SorCfg<T, G, Z, Y>::TEAM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int team = threadIdx.x / TEAM, tid = threadIdx.x - team * TEAM;
  unsigned char *tb = smem_raw + team * SS::team_bytes;
  T *stg = reinterpret_cast<T *>(tb + SS::S::team_bytes);
  uint64_t *bar = reinterpret_cast<uint64_t *>(tb + SS::S::team_bytes + SS::stage_bytes);
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_fence_init();
  }
  __syncthreads();
  auto stage = [&](int64_t P) {  // one thread: patch P's inputs -> stg
    tc::mbar_arrive_expect_tx(bar, uint32_t(sizeof(T) * SS::stage_elems));
    tc::bulk_load(stg, a.pot_in + P * g::PN3, uint32_t(sizeof(T) * g::PN3), bar);
    tc::bulk_load(stg + g::PN3, a.rho + P * g::RHO3, uint32_t(sizeof(T) * g::RHO3), bar);
  };
  const int64_t stride = int64_t(gridDim.x) * TPC;
  int64_t P_ = int64_t(blockIdx.x) * TPC + team;
  if (P_ < a.npatch && tid == 0) stage(P_);
  uint32_t it = 0;
  for (; P_ < a.npatch; P_ += stride, ++it) {
    if (it) team_sync<TEAM>(team);  // the previous patch's output and gravity reads of the cube are done
    const bool arrived = tc::mbar_wait(bar, it & 1u, nullptr);
    const int64_t next = P_ + stride;
    sor_solve_patch_with<T, G, PHASED, Z, Y, true>(
        a, P_, team, tid, tb, true,
        [&](const auto &) {
          // the staged inputs are in the cube and registers: fetch the next patch
          if (tid == 0 && next < a.npatch) {
            tc::fence_proxy_async_smem();
            stage(next);
          }
        },
        stg);
    if (!arrived && tid == 0) {
      if (a.iters) a.iters[P_] = -1;
      if (a.resid) a.resid[P_] = __longlong_as_double(0x7ff8000000000000ll);
    }
  }
}

}  // namespace gpg
