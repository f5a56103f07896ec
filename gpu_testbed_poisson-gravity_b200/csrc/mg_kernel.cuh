// mg_kernel.cuh -- per-patch multigrid V-cycle, one patch per CTA, all levels
// resident in shared memory (no device-side malloc).
//
// Semantics follow CPU_PoissonSolver_MG.cpp:46-377:
//   levels  N0 = 8+2G, N(l+1) = (N(l)+1)/2 while that is >= 3; dh(l) = dh (N0-1)/(N(l)-1)
//           (10-5-3, 12-6-3, 14-7-4, 16-8-4, 18-9-5-3), bottom smoothing 1 (3^3) or 7 (4^3)
//   cycle   per level down: NPre red-black Gauss-Seidel sweeps, defect, 27-point
//           restriction to the next RHS, zero correction; bottom smoothing; per level
//           up: trilinear prolongation added, NPost sweeps
//   error   dh^2 sum|defect| / sum|sol| on level 0 (sums in double), stop when
//           <= MG_Tolerated_Error or after Max_Iter cycles
// Operand order of every stencil follows the reference loops (bit-identical values).
#pragma once

#include <type_traits>

#include <cfloat>

#include "common.cuh"
#include "gravity.cuh"
#include "interp.cuh"

namespace gpg {

template <int G>
struct MgLevels {
  static constexpr int n0 = 8 + 2 * G;
  static constexpr int next(int n) { return (n + 1) / 2; }
  static constexpr int count() {
    int n = n0, c = 1;
    while (next(n) >= 3 && c < 10) { n = next(n); ++c; }
    return c;
  }
  static constexpr int L = count();  // number of levels, bottom = L-1
  static constexpr int size(int lv) {
    int n = n0;
    for (int i = 0; i < lv; ++i) n = next(n);
    return n;
  }
  static constexpr int cells(int lv) { return size(lv) * size(lv) * size(lv); }
  static constexpr int offset(int lv) {
    int o = 0;
    for (int i = 0; i < lv; ++i) o += cells(i);
    return o;
  }
  static constexpr int total = offset(L);
  static constexpr int nbottom = size(L - 1) == 3 ? 1 : 7;
  static_assert(size(L - 1) == 3 || size(L - 1) == 4, "bottom grid must be 3^3 or 4^3");
};

template <typename T, int G, int NT>
struct MgSmem {
  using LV = MgLevels<G>;
  static constexpr size_t round(size_t b) { return (b + 15) / 16 * 16; }
  static constexpr size_t level_bytes = round(sizeof(T) * LV::total);
  // sol, rhs, def for every level + reduction slots
  static constexpr size_t bytes = 3 * level_bytes + round(2 * sizeof(double) * (NT / 32));
};

// Red-black Gauss-Seidel (CPU_PoissonSolver_MG.cpp:392-441): pass 0 updates
// cells with (i+j+k) odd.  Ends with a barrier.
template <typename T, int NT>
__device__ __forceinline__ void mg_smooth(T *sol, const T *rhs, T dh, int n, int tid) {
  const T dh2 = mul(dh, dh), one_six = divide(T(1), T(6));
  const int m = n - 2, w = (m + 1) / 2, rows = m * m;
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    for (int t = tid; t < rows * w; t += NT) {
      const int row = t / w, s = t - row * w;
      const int j = 1 + row % m, k = 1 + row / m;
      const int i = 2 - ((1 + k + j + pass) & 1) + 2 * s;
      if (i >= n - 1) continue;
      const int id = (k * n + j) * n + i;
      const T sum = add(add(add(add(add(sol[id + n * n], sol[id - n * n]), sol[id + n]), sol[id - n]),
                            sol[id + 1]), sol[id - 1]);
      sol[id] = mul(one_six, sub(sum, mul(dh2, rhs[id])));
    }
    __syncthreads();
  }
}

// def = -(lap(sol) - rhs) on interior cells (CPU_PoissonSolver_MG.cpp:474-494);
// optionally accumulates sum|def| and sum|sol| in double.
template <typename T, int NT, bool SUMS>
__device__ __forceinline__ void mg_defect(const T *sol, const T *rhs, T *def, T dh, int n, int tid,
                                          double &sd, double &ss) {
  const T m_dh2 = divide(T(-1), mul(dh, dh));
  const int m = n - 2;
  for (int t = tid; t < m * m * m; t += NT) {
    const int i = 1 + t % m, j = 1 + (t / m) % m, k = 1 + t / (m * m);
    const int id = (k * n + j) * n + i;
    const T sum = add(add(add(add(add(sol[id + n * n], sol[id - n * n]), sol[id + n]), sol[id - n]),
                          sol[id + 1]), sol[id - 1]);
    const T d = add(mul(m_dh2, sub(sum, mul(T(6), sol[id]))), rhs[id]);
    def[id] = d;
    if constexpr (SUMS) {
      sd += (double)absval(d);
      ss += (double)absval(sol[id]);
    }
  }
}

// 27-point restriction (CPU_PoissonSolver_MG.cpp:533-616).
template <typename T, int NT>
__device__ __forceinline__ void mg_restrict(const T *f, T *c, int nf, int nc, int tid) {
  const T ratio = divide(T(nf - 1), T(nc - 1)), half = T(0.5);
  const int mc = nc - 2;
  for (int t = tid; t < mc * mc * mc; t += NT) {
    const int i = 1 + t % mc, j = 1 + (t / mc) % mc, k = 1 + t / (mc * mc);
    T w[3][3];  // [z/y/x][left/centre/right]
    int base[3];
    const int ijk[3] = {k, j, i};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T pos = mul(T(ijk[d]), ratio);
      const int cc = (int)add(pos, half);
      base[d] = cc - 1;
      w[d][0] = mul(half, sub(add(T(cc), half), pos));
      w[d][2] = sub(half, w[d][0]);
      w[d][1] = half;
    }
    T v = T(0);
    if constexpr (sizeof(T) == 8) {
      // FP64: one z plane of the 27 terms at a time (same accumulation order);
      // fully unrolled, the restriction alone held the kernel at 163 registers
#pragma unroll 1
      for (int tz = 0; tz < 3; ++tz) {
        const T wz = tz == 0 ? w[0][0] : (tz == 1 ? w[0][1] : w[0][2]);
#pragma unroll
        for (int ty = 0; ty < 3; ++ty)
#pragma unroll
          for (int tx = 0; tx < 3; ++tx) {
            const T term = mul(mul(mul(wz, w[1][ty]), w[2][tx]),
                               f[((base[0] + tz) * nf + base[1] + ty) * nf + base[2] + tx]);
            v = (tz | ty | tx) ? add(v, term) : term;
          }
      }
    } else {
#pragma unroll
      for (int tz = 0; tz < 3; ++tz)
#pragma unroll
        for (int ty = 0; ty < 3; ++ty)
#pragma unroll
          for (int tx = 0; tx < 3; ++tx) {
            const T term = mul(mul(mul(w[0][tz], w[1][ty]), w[2][tx]),
                               f[((base[0] + tz) * nf + base[1] + ty) * nf + base[2] + tx]);
            v = (tz | ty | tx) ? add(v, term) : term;
          }
    }
    c[(k * nc + j) * nc + i] = v;
  }
}

// Trilinear prolongation added to interior fine cells (CPU_PoissonSolver_MG.cpp:635-684);
// the eight corner terms in the reference's order 000,001,010,100,011,110,101,111 (z,y,x).
template <typename T, int NT>
__device__ __forceinline__ void mg_prolongate(const T *c, T *f, int nc, int nf, int tid) {
  const T ratio = divide(T(nc - 1), T(nf - 1));
  const int mf = nf - 2;
  for (int t = tid; t < mf * mf * mf; t += NT) {
    const int i = 1 + t % mf, j = 1 + (t / mf) % mf, k = 1 + t / (mf * mf);
    T w[3][2];
    int base[3];
    const int ijk[3] = {k, j, i};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T pos = mul(T(ijk[d]), ratio);
      const int cc = (int)pos;
      base[d] = cc;
      w[d][0] = sub(T(cc + 1), pos);
      w[d][1] = sub(T(1), w[d][0]);
    }
    constexpr int ord[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {1, 0, 0},
                               {0, 1, 1}, {1, 1, 0}, {1, 0, 1}, {1, 1, 1}};
    T v = T(0);
#pragma unroll
    for (int o = 0; o < 8; ++o) {
      const int oz = ord[o][0], oy = ord[o][1], ox = ord[o][2];
      const T term = mul(mul(mul(w[0][oz], w[1][oy]), w[2][ox]),
                         c[((base[0] + oz) * nc + base[1] + oy) * nc + base[2] + ox]);
      v = o ? add(v, term) : term;
    }
    const int id = (k * nf + j) * nf + i;
    f[id] = add(f[id], v);
  }
}

template <typename T, int NT>
__device__ __forceinline__ void block_sum2(double &a, double &b, double *s_red, int tid) {
  constexpr int NWARP = NT / 32;
  a = warp_sum(a);
  b = warp_sum(b);
  if ((tid & 31) == 0) {
    s_red[tid >> 5] = a;
    s_red[NWARP + (tid >> 5)] = b;
  }
  __syncthreads();
  a = s_red[0];
  b = s_red[NWARP];
#pragma unroll
  for (int w = 1; w < NWARP; ++w) {
    a += s_red[w];
    b += s_red[NWARP + w];
  }
  __syncthreads();
}

template <typename T, int G, int NT>
__global__ void __launch_bounds__(NT) mg_kernel(const SolveArgs<T> a) {
  using LV = MgLevels<G>;
  using g = Geo<G>;
  using S = MgSmem<T, G, NT>;
  constexpr int L = LV::L, N = g::N, M = g::M;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s_sol = reinterpret_cast<T *>(smem_raw);
  T *s_rhs = reinterpret_cast<T *>(smem_raw + S::level_bytes);
  T *s_def = reinterpret_cast<T *>(smem_raw + 2 * S::level_bytes);
  double *s_red = reinterpret_cast<double *>(smem_raw + 3 * S::level_bytes);
  const int tid = threadIdx.x;
  const int64_t P = blockIdx.x;
  if (P >= a.npatch) return;

  int nlv[L], off[L];
  T dhl[L];
#pragma unroll
  for (int l = 0; l < L; ++l) {
    nlv[l] = LV::size(l);
    off[l] = LV::offset(l);
    dhl[l] = l == 0 ? a.dh : divide(mul(a.dh, T(N - 1)), T(LV::size(l) - 1));
  }

  // level-0 solution = interpolated cube; rhs0 = Poi_Coeff * rho; def boundaries 0
  for (int t = tid; t < LV::total; t += NT) s_def[t] = T(0);
  interpolate<T, G, NT>(a.pot_in + P * g::PN3, tid, a.int_scheme,
                        [s_sol](int x, int y, int z, T v) { s_sol[(z * N + y) * N + x] = v; });
  {
    const T *rho = a.rho + P * g::RHO3;
    for (int t = tid; t < g::RHO3; t += NT) {
      const int i = t % M, j = (t / M) % M, k = t / (M * M);
      s_rhs[((k + 1) * N + (j + 1)) * N + (i + 1)] = mul(a.poi_coeff, rho[t]);
    }
  }
  __syncthreads();

  int iter = 0;
  double err = (double)FLT_MAX;
  const double tol = (double)a.mg_tol;
  while (iter < a.mg_max_iter && err > tol) {
#pragma unroll
    for (int l = 0; l < L - 1; ++l) {
      for (int s = 0; s < a.mg_npre; ++s) mg_smooth<T, NT>(s_sol + off[l], s_rhs + off[l], dhl[l], nlv[l], tid);
      double d0 = 0, d1 = 0;
      mg_defect<T, NT, false>(s_sol + off[l], s_rhs + off[l], s_def + off[l], dhl[l], nlv[l], tid, d0, d1);
      __syncthreads();
      mg_restrict<T, NT>(s_def + off[l], s_rhs + off[l + 1], nlv[l], nlv[l + 1], tid);
      for (int t = tid; t < nlv[l + 1] * nlv[l + 1] * nlv[l + 1]; t += NT) s_sol[off[l + 1] + t] = T(0);
      __syncthreads();
    }
    for (int s = 0; s < LV::nbottom; ++s)
      mg_smooth<T, NT>(s_sol + off[L - 1], s_rhs + off[L - 1], dhl[L - 1], nlv[L - 1], tid);
#pragma unroll
    for (int l = L - 2; l >= 0; --l) {
      mg_prolongate<T, NT>(s_sol + off[l + 1], s_sol + off[l], nlv[l + 1], nlv[l], tid);
      __syncthreads();
      for (int s = 0; s < a.mg_npost; ++s) mg_smooth<T, NT>(s_sol + off[l], s_rhs + off[l], dhl[l], nlv[l], tid);
    }
    double sd = 0, ss = 0;
    mg_defect<T, NT, true>(s_sol, s_rhs, s_def, dhl[0], N, tid, sd, ss);
    block_sum2<T, NT>(sd, ss, s_red, tid);  // includes the barriers
    err = ((double)mul(dhl[0], dhl[0]) * sd) / ss;
    ++iter;
  }
  if (tid == 0) {
    if (a.iters) a.iters[P] = iter;
    if (a.resid) a.resid[P] = err;
  }
  // output window, its edge a compile-time constant per GRA_GHOST_SIZE
  auto window = [&](auto gg) {
    constexpr int GG = decltype(gg)::value, GN = 8 + 2 * GG, shift = G - GG, GN3 = GN * GN * GN;
    T *dst = a.pot_out + P * GN3;
    for (int t = tid; t < GN3; t += NT) {
      const int i = t % GN, j = (t / GN) % GN, k = t / (GN * GN);
      dst[t] = s_sol[((k + shift) * N + (j + shift)) * N + (i + shift)];
    }
  };
  if (a.gra_ghost == 0)
    window(std::integral_constant<int, 0>{});
  else if (a.gra_ghost == 1)
    window(std::integral_constant<int, 1>{});
  else
    window(std::integral_constant<int, 2>{});
  if (a.gra_acc) {
    gravity_patch<T, NT>(a.flu + P * 5 * 512, tid, a.gra_const, a.p5, [s_sol](int i, int j, int k) {
      return s_sol[((k + G) * N + (j + G)) * N + (i + G)];
    });
  }
}

}  // namespace gpg
