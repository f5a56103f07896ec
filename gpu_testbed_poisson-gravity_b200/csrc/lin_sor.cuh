// lin_sor.cuh -- ghost-size-1 FP32 SOR whose start value is the interpolated
// coarse potential plus a learned linear correction, in one persistent kernel.
//
// The correction.  Let r0 = Lap(phi_i) - Const rho be the residual of the
// interpolated start phi_i on the 8^3 interior (the SOR's own residual
// expression, CPU_PoissonSolver_SOR.cpp:232-237).  The exact correction is
// linear in r0 (the interior inverse Laplacian with zero boundary values), and
// that operator commutes with the reflections of the cube, so the learned map
// is built equivariant:
//   fold    u_b = sum_s (-1)^(b.s) r0(s(o))   for each orbit o in [0,4)^3 of
//           the reflections x -> 7-x, y -> 7-y, z -> 7-z and each parity
//           b = (pz, py, px): a length-8 Walsh-Hadamard transform per orbit
//   apply   v_b = W_class(b) u_b              64 x 64 per block; blocks whose
//           parities are axis permutations of each other share one matrix
//           (classes by the number of odd axes: 1, 3, 3, 1 blocks), applied
//           to the orbit index permuted into the class representative's axes
//   unfold  delta(s(o)) = sum_b (-1)^(b.s) v_b(o)
//   start   phi = phi_i + delta
// 4 x 64 x 64 parameters (FP32 masters, BF16 in the kernel), 65,536 FLOP per
// patch (algorithmic).
//
// Kernel.  One persistent CTA per SM, 16 warps in two independent halves of
// 8 that share the weight tiles (each half has its own barrier, operand tile,
// TMEM columns and MMA barrier, so one half's batch synchronisation is hidden
// behind the other's work).  Each warp is one SOR team (the two-row,
// split-column lane layout of sor_kernel.cuh) and owns one patch of its
// half's batch of 8.  A warp's next patch (coarse potential and density,
// 4 KB) is prefetched into shared memory with bulk copies while the current
// one is solved.  Per batch, every team interpolates its patch from the
// staged copy into its shared cube, forms r0 for its cells, folds it and
// writes the 8 block vectors (BF16) into its half's MMA operand tile; one
// thread per half issues 16 tcgen05.mma (M 128 = two class matrices stacked,
// N 16 = the 8 patches of two blocks side by side, K 64) against the weight
// tiles, which stay in shared memory for the whole kernel; the teams read the
// FP32 results back from TMEM, unfold their own patch, add the correction to
// the cube and run the ordinary sweeps, stopping rule, output window and
// (optionally) gravity update of sor_solve_patch_with.
#pragma once

#include <cuda_bf16.h>

#include "sor_kernel.cuh"
#include "tc_common.cuh"

namespace gpg {
namespace lin {

constexpr int kHalfWarps = 8;         // teams (patches) per batch of one group of teams
constexpr int kN = 2 * kHalfWarps;    // MMA N: two blocks' patches side by side
constexpr int kGroups = 4;            // MMAs per K step: (c0 | c3), 3 x (c1 | c2)
constexpr int kK = 64;                // orbits per block
constexpr int kTileBytes = 128 * kK * 2;       // one A tile (BF16): 16 KB
// one B tile (BF16): 8 K chunks of kN rows x 16 B, chunks kChunkB apart (16 B
// of padding put consecutive chunks on different banks for the operand stores)
constexpr int kChunkB = kN * 16 + 16;
constexpr int kGroupBytes = (kK / 8) * kChunkB;
// team scratch: interior cell (z, y, x) at z * kScrPZ + y * 8 + x (plane pitch
// padded from 64 so that lane-cell and mirror-orbit accesses spread over the
// banks), block results at b * 64 + o
constexpr int kScrPZ = 66;
constexpr int kScrWords = 8 * kScrPZ;
constexpr int kHalfCols = kGroups * kN;        // TMEM columns of one group of teams: 64
constexpr int kParams = 4 * kK * kK;           // 16,384
constexpr int kFeatureGain = 17;               // log2 of the training features' extra scale
constexpr uint32_t kIdesc = tc::idesc_bf16(128, kN, false, false);

// block b = pz*4 + py*2 + px: MMA group, side (rows 0-63 / 64-127 of the
// stacked tile and the first / second 8 columns of the group) and the axis
// permutation that maps the block's orbit index into its class
// representative's (0 none, 1 x<->y, 2 x<->z, 3 y<->z)
__host__ __device__ constexpr int group_of(int b) { return b == 0 || b == 7 ? 0 : (b == 1 || b == 3 ? 1 : (b == 2 || b == 5 ? 2 : 3)); }
__host__ __device__ constexpr int side_of(int b) { return (b == 3 || b == 5 || b == 6 || b == 7) ? 1 : 0; }
__host__ __device__ constexpr int perm_of(int b) { return b == 2 ? 1 : (b == 4 || b == 6 ? 2 : (b == 5 ? 3 : 0)); }
// block of (group, side)
__host__ __device__ constexpr int block_of(int g, int side) {
  return g == 0 ? (side ? 7 : 0) : (g == 1 ? (side ? 3 : 1) : (g == 2 ? (side ? 5 : 2) : (side ? 6 : 4)));
}
// orbit index o = k*16 + j*4 + i (z, y, x in [0,4)) under an axis swap (an
// involution, so it is its own inverse)
__host__ __device__ constexpr int perm_orbit(int o, int t) {
  const int k = o >> 4, j = (o >> 2) & 3, i = o & 3;
  return t == 0 ? o : (t == 1 ? (k << 4) | (i << 2) | j : (t == 2 ? (i << 4) | (j << 2) | k : (j << 4) | (k << 2) | i));
}
// scratch word of interior cell (z, y, x)
__host__ __device__ constexpr int scr_cell(int z, int y, int x) { return z * kScrPZ + y * 8 + x; }
// scratch word of orbit o's image under mirror s = (sz, sy, sx)
__host__ __device__ constexpr int orbit_cell(int o, int s) {
  const int k = o >> 4, j = (o >> 2) & 3, i = o & 3;
  const int z = (s & 4) ? 7 - k : k, y = (s & 2) ? 7 - j : j, x = (s & 1) ? 7 - i : i;
  return scr_cell(z, y, x);
}

// In-place length-8 Walsh-Hadamard transform, stages x, y, z (index bit 0, 1,
// 2); out[b] = sum_s (-1)^popcount(b & s) in[s].  Fixed order, IEEE adds.
__device__ __forceinline__ void hadamard8(float (&a)[8]) {
#pragma unroll
  for (int hb = 1; hb < 8; hb <<= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & hb)) {
        const float p = a[i], q = a[i | hb];
        a[i] = __fadd_rn(p, q);
        a[i | hb] = __fsub_rn(p, q);
      }
}

// TMEM -> registers: 32 lanes x 8 columns of 32-bit
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// named barrier of one group of teams (ids 1.., 0 is __syncthreads)
__device__ __forceinline__ void half_bar(int half) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + half), "n"(kHalfWarps * 32) : "memory");
}

// Launch shape: HALVES groups of 8 teams share the weight tiles; STAGE: each
// team prefetches its next patch's inputs into shared memory (bulk copies).
// Shared memory allows 2 staged groups or 3 unstaged ones (registers then
// bounded to 80 per thread).
template <int HALVES, bool STAGE>
struct Shape {
  static constexpr int kHalves = HALVES;
  static constexpr int kWarps = HALVES * kHalfWarps;
  static constexpr int kThreads = kWarps * 32;
  static constexpr int kTmemCols = HALVES * kHalfCols <= 128 ? 128 : 256;  // a power of two
};

// Team shape: ghost 1, FP32, two rows per lane, split column (variant 10 of
// the per-ghost-size kernels): one warp per patch, every lane owns cells.
using Cfg = SorCfg<float, 1, 2, 2>;
using Smem = SorSmem<float, 1, 2, 2>;
static_assert(Cfg::TEAM == 32 && Cfg::NBLOCK * Cfg::BLOCK == 32, "one fully used warp per patch");

template <int HALVES, bool STAGE>
struct Layout {
  using SH = Shape<HALVES, STAGE>;
  static constexpr int kStage = Geo<1>::PN3 + Geo<1>::RHO3;               // floats per staged patch
  static constexpr size_t a_off = 0;                                      // 2 weight tiles
  static constexpr size_t b_off = a_off + 2 * kTileBytes;                 // per group 4 operand tiles
  static constexpr size_t scr_off = b_off + HALVES * kGroups * kGroupBytes;  // per team scratch
  static constexpr size_t stg_off = scr_off + SH::kWarps * kScrWords * 4;    // per team staged inputs
  static constexpr size_t cube_off = stg_off + (STAGE ? SH::kWarps * kStage * 4 : 0);  // per team cube
  static constexpr size_t bar_off = cube_off + SH::kWarps * Smem::team_bytes;
  // barriers: [0, HALVES) MMA done per group, then staged inputs per team, then the probe
  static constexpr int kBars = HALVES + SH::kWarps + 1;
  static constexpr size_t bytes = bar_off + kBars * 8 + 16;
  static_assert(bytes <= 227 * 1024, "shared memory");
};

struct LinArgs {
  SolveArgs<float> s;
  const __nv_bfloat16 *wtiles;  // [2][kTileBytes / 2], packed by the host
  float *u_out;                 // features mode: [P][8][64] folded residual (class axes), scaled
  float *t_out;                 // features mode: [P][8][64] folded (target - interpolation) / 8, scaled
  const float *target;          // features mode: [P][8]^3 or null
  int *err;                     // set when a tensor-core wait timed out
  int probe_polls;              // > 0: thread 0 also waits that many polls on a barrier nothing signals
};

// residual of the lane's cells on the unmodified interpolated cube: for
// colour p, rows r and heights z of the lane, the same neighbour reads and
// operand order as sor_pass2 (six neighbours summed z+, z-, y+, y-, x+, x-,
// then - 6 phi - Const rho)
__device__ __forceinline__ void lane_residual(const SorLaneState<float, 1, 2, 2> &st,
                                              float (&res)[2][2][Cfg::MH]) {
  constexpr int N = Geo<1>::N, MH = Cfg::MH, P = Cfg::P, PP = Cfg::PP;
  static_assert(!(MH & 1), "the side of each cell follows from the local height alone");
  const auto &v = st.v;
  const int own0 = st.ln.own, own1 = st.ln.own + P;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const float *nb = st.s_cube + (1 - p) * N * PP + st.ln.zoff;
#pragma unroll
    for (int z = 1; z <= MH; ++z) {
      const bool left1 = ((z + p) & 1) == 0, left0 = !left1;
      const float xo0 = nb[z * PP + own0 + (left0 ? -1 : 1)];
      const float ym0 = nb[z * PP + own0 - P];
      const float xo1 = nb[z * PP + own1 + (left1 ? -1 : 1)];
      const float yp1 = nb[z * PP + own1 + P];
      // row 0: y+ neighbour is row 1 (registers), y- from shared memory
      {
        const float mate = v[0][1 - p][z];
        const float xp = left0 ? mate : xo0, xm = left0 ? xo0 : mate;
        const float sm = add(add(add(add(add(v[0][1 - p][z + 1], v[0][1 - p][z - 1]), v[1][1 - p][z]), ym0), xp), xm);
        res[0][p][z - 1] = sub(sub(sm, mul(6.f, v[0][p][z])), st.crho[0][p][z - 1]);
      }
      {
        const float mate = v[1][1 - p][z];
        const float xp = left1 ? mate : xo1, xm = left1 ? xo1 : mate;
        const float sm = add(add(add(add(add(v[1][1 - p][z + 1], v[1][1 - p][z - 1]), yp1), v[0][1 - p][z]), xp), xm);
        res[1][p][z - 1] = sub(sub(sm, mul(6.f, v[1][p][z])), st.crho[1][p][z - 1]);
      }
    }
  }
}

// interior (z, y, x) of the lane's colour-p cell at local height z in row r
__device__ __forceinline__ void lane_xyz(const SorLaneState<float, 1, 2, 2> &st, int r, int p, int z, int &cz,
                                         int &cy, int &cx) {
  const int yr = st.y + r, zg = st.zbase + z;
  cx = (((yr + zg + p) & 1) == 0 ? 2 * st.h + 1 : 2 * st.h + 2) - 1;
  cy = yr - 1;
  cz = zg - 1;
}
// its scratch word
__device__ __forceinline__ int lane_cell(const SorLaneState<float, 1, 2, 2> &st, int r, int p, int z) {
  int cz, cy, cx;
  lane_xyz(st, r, p, z, cz, cy, cx);
  return scr_cell(cz, cy, cx);
}

template <bool FEATURES, int HALVES, bool STAGE>
__global__ void __launch_bounds__(Shape<HALVES, STAGE>::kThreads, 1) lin_sor_kernel(const LinArgs a) {
  using SH = Shape<HALVES, STAGE>;
  using Layout = gpg::lin::Layout<HALVES, STAGE>;
  constexpr int kHalves = SH::kHalves, kWarps = SH::kWarps, kThreads = SH::kThreads, kTmemCols = SH::kTmemCols;
  constexpr bool kStaged = STAGE && !FEATURES;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *sA = smem + Layout::a_off;
  float *s_scr = reinterpret_cast<float *>(smem + Layout::scr_off);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + Layout::bar_off);
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + Layout::kBars);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int half = warp / kHalfWarps, wl = warp - half * kHalfWarps;  // team index inside the half
  unsigned char *sB = smem + Layout::b_off + size_t(half) * kGroups * kGroupBytes;
  float *scr = s_scr + warp * kScrWords;
  float *stg = reinterpret_cast<float *>(smem + Layout::stg_off) + size_t(warp) * Layout::kStage;
  unsigned char *tb = smem + Layout::cube_off + size_t(warp) * Smem::team_bytes;
  uint64_t *bar_mma = bars + half, *bar_stg = bars + kHalves + warp, *bar_probe = bars + kHalves + kWarps;

  uint32_t tmem = 0;
  if constexpr (!FEATURES) {
    // weight tiles: resident for the whole kernel
    const uint4 *src = reinterpret_cast<const uint4 *>(a.wtiles);
    uint4 *dst = reinterpret_cast<uint4 *>(sA);
    for (int i = tid; i < 2 * kTileBytes / 16; i += kThreads) dst[i] = src[i];
    if (tid == 0) {
      for (int i = 0; i < Layout::kBars; ++i) tc::mbar_init(&bars[i], 1);
      tc::mbar_fence_init();
    }
    if (warp == 0) {
      tc::tmem_alloc(s_tmem, kTmemCols);
      tc::tmem_relinquish();
    }
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    tmem = *s_tmem + uint32_t(half * kHalfCols);
    if (a.probe_polls > 0 && tid == 0) {
      // test hook: a bounded wait on a barrier nothing arrives on gives up
      // after probe_polls polls, records the timeout and the kernel goes on
      tc::mbar_wait_polls(bar_probe, 0, a.err, uint32_t(a.probe_polls));
    }
  }
  const int64_t npatch = a.s.npatch;
  const int64_t nbatch = (npatch + kHalfWarps - 1) / kHalfWarps;
  const int64_t hstride = int64_t(gridDim.x) * kHalves;
  // the patch team wl solves in batch b; a team past the end solves the last
  // patch again without storing it, so that it takes part in the barriers
  auto patch_of = [&](int64_t b) {
    const int64_t m = b * kHalfWarps + wl;
    return m < npatch ? m : npatch - 1;
  };
  auto stage = [&](int64_t P) {  // lane 0: this team's inputs of patch P -> stg
    tc::mbar_arrive_expect_tx(bar_stg, uint32_t(Layout::kStage * 4));
    tc::bulk_load(stg, a.s.pot_in + P * Geo<1>::PN3, Geo<1>::PN3 * 4, bar_stg);
    tc::bulk_load(stg + Geo<1>::PN3, a.s.rho + P * Geo<1>::RHO3, Geo<1>::RHO3 * 4, bar_stg);
  };
  const int64_t first = int64_t(blockIdx.x) * kHalves + half;
  if constexpr (kStaged) {
    if (first < nbatch && lane == 0) stage(patch_of(first));
  }
  uint32_t it = 0, phase = 0, last_parity = 0;
  bool late = false;  // a bounded wait gave up
  for (int64_t batch = first; batch < nbatch; batch += hstride, ++it) {
    const int64_t mine = batch * kHalfWarps + wl;
    const bool real = mine < npatch;
    const int64_t P_ = patch_of(batch), next = batch + hstride;
    if constexpr (kStaged) {
      if (!tc::mbar_wait(bar_stg, it & 1u, a.err)) late = true;
    }
    auto hook = [&](const auto &st) {
      if constexpr (kStaged) {
        // the staged inputs are in the cube and registers: prefetch the
        // team's next patch while this one is corrected and solved
        __syncwarp();
        if (next < nbatch && lane == 0) {
          tc::fence_proxy_async_smem();
          stage(patch_of(next));
        }
      }
      float res[2][2][Cfg::MH];
      lane_residual(st, res);
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
          for (int z = 1; z <= Cfg::MH; ++z) scr[lane_cell(st, r, p, z)] = res[r][p][z - 1];
      __syncwarp();
      // fold: lane handles orbits lane and lane + 32
      float u[2][8];
#pragma unroll
      for (int oo = 0; oo < 2; ++oo) {
        const int o = lane + 32 * oo;
#pragma unroll
        for (int s = 0; s < 8; ++s) u[oo][s] = scr[orbit_cell(o, s)];
        hadamard8(u[oo]);
      }
      if constexpr (FEATURES) {
        // scale: 2^(kFeatureGain - e) with max|phi_i| over the interior =
        // m 2^e, m in [0.5, 1) -- exact, and a linear map is indifferent to
        // it; the training loss then weights patches by their potential, and
        // the gain puts the residuals (about 1e-5 of the potential) near one,
        // far above the optimizer's epsilon
        float vmax = 0.f;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int z = 1; z <= Cfg::MH; ++z) vmax = fmaxf(vmax, fabsf(st.v[r][p][z]));
#pragma unroll
        for (int m = 16; m >= 1; m >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, m));
        int ex = 0;
        frexpf(vmax, &ex);
        const float sc = ldexpf(1.f, (vmax > 0.f ? -ex : 0) + kFeatureGain);
        if (real) {
          float *uo = a.u_out + mine * 512;
#pragma unroll
          for (int oo = 0; oo < 2; ++oo)
#pragma unroll
            for (int b = 0; b < 8; ++b) uo[b * 64 + perm_orbit(lane + 32 * oo, perm_of(b))] = mul(sc, u[oo][b]);
        }
        if (a.target) {
          // folded (target - interpolation) / 8: the block-space target whose
          // unfold is the correction
          __syncwarp();
          const float *tg = a.target + P_ * 512;
#pragma unroll
          for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int p = 0; p < 2; ++p)
#pragma unroll
              for (int z = 1; z <= Cfg::MH; ++z) {
                int cz, cy, cx;
                lane_xyz(st, r, p, z, cz, cy, cx);
                scr[scr_cell(cz, cy, cx)] = sub(__ldg(tg + (cz * 8 + cy) * 8 + cx), st.v[r][p][z]);
              }
          __syncwarp();
          float t[2][8];
#pragma unroll
          for (int oo = 0; oo < 2; ++oo) {
            const int o = lane + 32 * oo;
#pragma unroll
            for (int s = 0; s < 8; ++s) t[oo][s] = scr[orbit_cell(o, s)];
            hadamard8(t[oo]);
          }
          if (real) {
            float *to = a.t_out + mine * 512;
#pragma unroll
            for (int oo = 0; oo < 2; ++oo)
#pragma unroll
              for (int b = 0; b < 8; ++b)
                to[b * 64 + perm_orbit(lane + 32 * oo, perm_of(b))] = mul(sc, mul(0.125f, t[oo][b]));
          }
        }
        return;
      } else {
        // operand rows: [K chunk][row][8 BF16], row = side * 8 + team
#pragma unroll
        for (int oo = 0; oo < 2; ++oo)
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            const int K = perm_orbit(lane + 32 * oo, perm_of(b));
            const int row = side_of(b) * kHalfWarps + wl;
            __nv_bfloat16 *dst = reinterpret_cast<__nv_bfloat16 *>(sB + group_of(b) * kGroupBytes +
                                                                   (K >> 3) * kChunkB + row * 16) + (K & 7);
            *dst = __float2bfloat16_rn(u[oo][b]);
          }
        tc::fence_proxy_async_smem();
        half_bar(half);  // operands complete; the previous batch's results were read
        if (wl == 0 && lane == 0) {
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
#pragma unroll
          for (int g = 0; g < kGroups; ++g)
#pragma unroll
            for (int ks = 0; ks < kK / 16; ++ks) {
              const uint64_t ad = tc::smem_desc(a0 + (g ? kTileBytes : 0) + 2 * ks * 2048, 2048, 128);
              const uint64_t bd = tc::smem_desc(b0 + g * kGroupBytes + 2 * ks * kChunkB, kChunkB, 128);
              tc::mma_bf16(tmem + uint32_t(g * kN), ad, bd, kIdesc, ks > 0 ? 1u : 0u);
            }
          tc::mma_commit(bar_mma);
        }
        if (!tc::mbar_wait(bar_mma, phase, a.err)) late = true;
        last_parity = phase;
        phase ^= 1u;
        tc::fence_after_sync();
        // results: warp w reads TMEM lanes 32 (w % 4) .. + 31, i.e. class
        // rows 32 (w & 1) .. of side (w & 3) >> 1, for groups wl / 4 and wl / 4 + 2
        {
          const int q = warp & 3, side = q >> 1, row = 32 * (q & 1) + lane;
#pragma unroll
          for (int gi = 0; gi < 2; ++gi) {
            const int g = (wl >> 2) + 2 * gi;
            float val[8];
            tmem_ld8(tmem + (uint32_t(32 * q) << 16) + uint32_t(g * kN + side * kHalfWarps), val);
            tc::tmem_wait_ld();
            const int b = block_of(g, side), o = perm_orbit(row, perm_of(b));
            float *dst = s_scr + size_t(half) * kHalfWarps * kScrWords + b * 64 + o;
#pragma unroll
            for (int n = 0; n < kHalfWarps; ++n) dst[n * kScrWords] = val[n];
          }
        }
        tc::fence_before_sync();
        half_bar(half);  // every team's block results are in its scratch
        // unfold the own patch and add the correction to the start value
        float d[2][8];
#pragma unroll
        for (int oo = 0; oo < 2; ++oo) {
          const int o = lane + 32 * oo;
#pragma unroll
          for (int b = 0; b < 8; ++b) d[oo][b] = scr[b * 64 + o];
          hadamard8(d[oo]);
        }
        __syncwarp();
#pragma unroll
        for (int oo = 0; oo < 2; ++oo)
#pragma unroll
          for (int s = 0; s < 8; ++s) scr[orbit_cell(lane + 32 * oo, s)] = d[oo][s];
        __syncwarp();
        constexpr int N = Geo<1>::N, PP = Cfg::PP, P = Cfg::P;
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int p = 0; p < 2; ++p)
#pragma unroll
            for (int z = 1; z <= Cfg::MH; ++z) {
              st.v[r][p][z] = add(st.v[r][p][z], scr[lane_cell(st, r, p, z)]);
              st.s_cube[(p * N + st.zbase + z) * PP + st.ln.own + r * P] = st.v[r][p][z];
            }
        __syncwarp();
      }
    };
    if constexpr (FEATURES) {
      // interpolation and residual only: no sweeps, nothing else stored
      SolveArgs<float> s = a.s;
      s.max_iter = 0;
      sor_solve_patch_with<float, 1, false, 2, 2>(s, P_, 0, lane, tb, false, hook);
    } else if constexpr (kStaged) {
      sor_solve_patch_with<float, 1, false, 2, 2, true>(a.s, P_, 0, lane, tb, real, hook, stg);
    } else {
      sor_solve_patch_with<float, 1, false, 2, 2>(a.s, P_, 0, lane, tb, real, hook);
    }
  }
  if constexpr (!FEATURES) {
    // after a timed-out wait the MMAs may still run: wait for the half's last
    // commit (bounded) before the accumulator columns are released
    if (__syncthreads_or(late) && wl == 0 && lane == 0 && it > 0) tc::mbar_wait(bar_mma, last_parity, a.err);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
      tc::fence_after_sync();
      tc::tmem_dealloc(*s_tmem, kTmemCols);
    }
  }
}

}  // namespace lin
}  // namespace gpg
