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
// Kernel.  CTA = 8 warps; each warp is one SOR team (the two-row, split-column
// lane layout of sor_kernel.cuh) and owns one patch of the CTA's batch of 8.
// Per batch, every team interpolates its patch into its shared cube, forms r0
// for its cells, folds it and writes the 8 block vectors (BF16) into the MMA
// operand tile; thread 0 issues 16 tcgen05.mma (M 128 = two class matrices
// stacked, N 16 = the 8 patches of two blocks side by side, K 64) against the
// weight tiles, which stay in shared memory for the whole kernel; the teams
// read the FP32 results back from TMEM, unfold their own patch, add the
// correction to the cube and run the ordinary sweeps, stopping rule, output
// window and (optionally) gravity update of sor_solve_patch_with.
#pragma once

#include <cuda_bf16.h>

#include "sor_kernel.cuh"
#include "tc_common.cuh"

namespace gpg {
namespace lin {

constexpr int kWarps = 8;             // teams (patches) per CTA batch
constexpr int kThreads = kWarps * 32;
constexpr int kN = 2 * kWarps;        // MMA N: two blocks' patches side by side
constexpr int kGroups = 4;            // MMAs per K step: (c0 | c3), 3 x (c1 | c2)
constexpr int kK = 64;                // orbits per block
constexpr int kTileBytes = 128 * kK * 2;       // one A tile (BF16): 16 KB
constexpr int kGroupBytes = kN * kK * 2;       // one B tile (BF16): 2 KB
constexpr int kTmemCols = kGroups * kN;        // 64
constexpr int kParams = 4 * kK * kK;           // 16,384
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
// interior index (z*8 + y)*8 + x of orbit o's image under mirror s = (sz, sy, sx)
__host__ __device__ constexpr int orbit_cell(int o, int s) {
  const int k = o >> 4, j = (o >> 2) & 3, i = o & 3;
  const int z = (s & 4) ? 7 - k : k, y = (s & 2) ? 7 - j : j, x = (s & 1) ? 7 - i : i;
  return (z * 8 + y) * 8 + x;
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

__device__ __forceinline__ void cta_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory"); }

// Team shape: ghost 1, FP32, two rows per lane, split column (variant 10 of
// the per-ghost-size kernels): one warp per patch, every lane owns cells.
using Cfg = SorCfg<float, 1, 2, 2>;
using Smem = SorSmem<float, 1, 2, 2>;
static_assert(Cfg::TEAM == 32 && Cfg::NBLOCK * Cfg::BLOCK == 32, "one fully used warp per patch");

struct Layout {
  static constexpr size_t a_off = 0;                                   // 2 weight tiles
  static constexpr size_t b_off = a_off + 2 * kTileBytes;              // 4 operand tiles
  static constexpr size_t scr_off = b_off + kGroups * kGroupBytes;     // per team 512 floats
  static constexpr size_t cube_off = scr_off + kWarps * 512 * 4;       // per team cube
  static constexpr size_t bar_off = cube_off + kWarps * Smem::team_bytes;
  static constexpr size_t bytes = bar_off + 64;
};

struct LinArgs {
  SolveArgs<float> s;
  const __nv_bfloat16 *wtiles;  // [2][kTileBytes / 2], packed by the host
  float *u_out;                 // features mode: [P][8][64] folded residual (class axes)
  float *t_out;                 // features mode: [P][8][64] folded (target - interpolation) / 8
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

// interior index of the lane's colour-p cell at local height z in row r
__device__ __forceinline__ int lane_cell(const SorLaneState<float, 1, 2, 2> &st, int r, int p, int z) {
  const int yr = st.y + r, zg = st.zbase + z;
  const int x = ((yr + zg + p) & 1) == 0 ? 2 * st.h + 1 : 2 * st.h + 2;
  return ((zg - 1) * 8 + (yr - 1)) * 8 + (x - 1);
}

template <bool FEATURES>
__global__ void __launch_bounds__(kThreads, 2) lin_sor_kernel(const LinArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *sA = smem + Layout::a_off;
  unsigned char *sB = smem + Layout::b_off;
  float *s_scr = reinterpret_cast<float *>(smem + Layout::scr_off);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + Layout::bar_off);  // [0] MMA done, [1] probe
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float *scr = s_scr + warp * 512;
  unsigned char *tb = smem + Layout::cube_off + size_t(warp) * Smem::team_bytes;

  uint32_t tmem = 0;
  if constexpr (!FEATURES) {
    // weight tiles: resident for the whole kernel
    const uint4 *src = reinterpret_cast<const uint4 *>(a.wtiles);
    uint4 *dst = reinterpret_cast<uint4 *>(sA);
    for (int i = tid; i < 2 * kTileBytes / 16; i += kThreads) dst[i] = src[i];
    if (tid == 0) {
      tc::mbar_init(&bars[0], 1);
      tc::mbar_init(&bars[1], 1);
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
    tmem = *s_tmem;
    if (a.probe_polls > 0 && tid == 0) {
      // test hook: a bounded wait on a barrier nothing arrives on gives up
      // after probe_polls polls, records the timeout and the kernel goes on
      tc::mbar_wait_polls(&bars[1], 0, a.err, uint32_t(a.probe_polls));
    }
  }
  const int64_t npatch = a.s.npatch;
  const int64_t nbatch = (npatch + kWarps - 1) / kWarps;
  uint32_t phase = 0, last_parity = 0;
  bool late = false;  // a wait for the MMAs gave up
  for (int64_t batch = blockIdx.x; batch < nbatch; batch += gridDim.x) {
    const int64_t mine = batch * kWarps + warp;
    const bool real = mine < npatch;
    // a team past the end solves the last patch again without storing it, so
    // that every team takes part in the batch's barriers
    const int64_t P_ = real ? mine : npatch - 1;
    auto hook = [&](const auto &st) {
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
        if (real) {
          float *uo = a.u_out + mine * 512;
#pragma unroll
          for (int oo = 0; oo < 2; ++oo)
#pragma unroll
            for (int b = 0; b < 8; ++b) uo[b * 64 + perm_orbit(lane + 32 * oo, perm_of(b))] = u[oo][b];
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
                const int c = lane_cell(st, r, p, z);
                scr[c] = sub(__ldg(tg + c), st.v[r][p][z]);
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
              for (int b = 0; b < 8; ++b) to[b * 64 + perm_orbit(lane + 32 * oo, perm_of(b))] = mul(0.125f, t[oo][b]);
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
            const int row = side_of(b) * kWarps + warp;
            __nv_bfloat16 *dst = reinterpret_cast<__nv_bfloat16 *>(sB + group_of(b) * kGroupBytes) +
                                 ((K >> 3) * kN + row) * 8 + (K & 7);
            *dst = __float2bfloat16_rn(u[oo][b]);
          }
        tc::fence_proxy_async_smem();
        cta_bar();  // operands complete; the previous batch's results were read
        if (tid == 0) {
          tc::fence_after_sync();
          const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
#pragma unroll
          for (int g = 0; g < kGroups; ++g)
#pragma unroll
            for (int ks = 0; ks < kK / 16; ++ks) {
              const uint64_t ad = tc::smem_desc(a0 + (g ? kTileBytes : 0) + 2 * ks * 2048, 2048, 128);
              const uint64_t bd = tc::smem_desc(b0 + g * kGroupBytes + 2 * ks * (kN * 16), kN * 16, 128);
              tc::mma_bf16(tmem + uint32_t(g * kN), ad, bd, kIdesc, ks > 0 ? 1u : 0u);
            }
          tc::mma_commit(&bars[0]);
        }
        if (!tc::mbar_wait(&bars[0], phase, a.err)) late = true;
        last_parity = phase;
        phase ^= 1u;
        tc::fence_after_sync();
        // results: warp w reads TMEM lanes 32 (w % 4) .. + 31, i.e. class
        // rows 32 (w & 1) .. of side (w & 3) >> 1, for groups w / 4 and w / 4 + 2
        {
          const int q = warp & 3, side = q >> 1, row = 32 * (q & 1) + lane;
#pragma unroll
          for (int gi = 0; gi < 2; ++gi) {
            const int g = (warp >> 2) + 2 * gi;
            float val[8];
            tmem_ld8(tmem + (uint32_t(32 * q) << 16) + uint32_t(g * kN + side * kWarps), val);
            tc::tmem_wait_ld();
            const int b = block_of(g, side), o = perm_orbit(row, perm_of(b));
#pragma unroll
            for (int n = 0; n < kWarps; ++n) s_scr[n * 512 + b * 64 + o] = val[n];
          }
        }
        tc::fence_before_sync();
        cta_bar();  // every team's block results are in its scratch
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
    } else {
      sor_solve_patch_with<float, 1, false, 2, 2>(a.s, P_, 0, lane, tb, real, hook);
    }
  }
  if constexpr (!FEATURES) {
    // after a timed-out wait the MMAs may still run: wait for the last commit
    // (bounded) before the accumulator columns are released
    if (__syncthreads_or(late) && tid == 0) tc::mbar_wait(&bars[0], last_parity, a.err);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
      tc::fence_after_sync();
      tc::tmem_dealloc(tmem, kTmemCols);
    }
  }
}

}  // namespace lin
}  // namespace gpg
