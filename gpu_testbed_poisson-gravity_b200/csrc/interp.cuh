// interp.cuh -- coarse -> fine potential interpolation of one patch.
//
// Every interior coarse cell (i, j, k) in [1, POT_NXT-1)^3 produces its 8 fine
// children; children outside the solver cube (the POT_USELESS layers for odd
// ghost sizes) are dropped.  CQUAD is the conservative quadratic form of
// CPU_PoissonSolver_SOR.cpp:110-174 (13 slopes weighted 1/8, 1/64, 1/512);
// QUAD the 27-point tensor product of CPU_PoissonSolver_SOR.cpp:177-203.
// Operand order follows those loops so the values are bit-identical.
#pragma once

#include "common.cuh"

namespace gpg {

// `coarse` is one patch's [POT_NXT]^3 potential: in global memory, read
// through L1 (LDG; each value feeds up to 27 coarse cells), or a copy staged
// in shared memory (!LDG).
template <typename T, int G, int NT, bool LDG = true, typename Store>
__device__ __forceinline__ void interpolate(const T *__restrict__ coarse, int tid, int int_scheme,
                                            Store store) {
  using g = Geo<G>;
  constexpr int PN = g::PN, NC = PN - 2, N = g::N, U = g::U;
  for (int w = tid; w < NC * NC * NC; w += NT) {
    const int i = 1 + w % NC, j = 1 + (w / NC) % NC, k = 1 + w / (NC * NC);
    const T *c0 = coarse + (k * PN + j) * PN + i;
    auto C = [c0](int dk, int dj, int di) -> T {
      const T *q = c0 + (dk * PN + dj) * PN + di;
      if constexpr (LDG) return __ldg(q);
      else return *q;
    };
    T child[8];
    if (int_scheme == 4) {
      const T c8 = T(0.125), c64 = T(0.015625), c512 = T(0.001953125);
      T s[13];
      s[0] = mul(c8, sub(C(0, 0, 1), C(0, 0, -1)));
      s[1] = mul(c8, sub(C(0, 1, 0), C(0, -1, 0)));
      s[2] = mul(c8, sub(C(1, 0, 0), C(-1, 0, 0)));
      s[3] = mul(c64, sub(C(-1, 0, 1), C(-1, 0, -1)));
      s[4] = mul(c64, sub(C(-1, 1, 0), C(-1, -1, 0)));
      s[5] = mul(c64, sub(C(0, -1, 1), C(0, -1, -1)));
      s[6] = mul(c64, sub(C(0, 1, 1), C(0, 1, -1)));
      s[7] = mul(c64, sub(C(1, 0, 1), C(1, 0, -1)));
      s[8] = mul(c64, sub(C(1, 1, 0), C(1, -1, 0)));
      s[9] = mul(c512, sub(C(-1, -1, 1), C(-1, -1, -1)));
      s[10] = mul(c512, sub(C(-1, 1, 1), C(-1, 1, -1)));
      s[11] = mul(c512, sub(C(1, -1, 1), C(1, -1, -1)));
      s[12] = mul(c512, sub(C(1, 1, 1), C(1, 1, -1)));
      const T centre = C(0, 0, 0);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        // half-signs of child c along x, y, z; each slope's sign is their product
        const int sx = (c & 1) ? 1 : -1, sy = (c & 2) ? 1 : -1, sz = (c & 4) ? 1 : -1;
        const int sg[13] = {sx,      sy,      sz,           -sx * sz,      -sy * sz,
                            -sx * sy, sx * sy, sx * sz,      sy * sz,       sx * sy * sz,
                            -sx * sy * sz, -sx * sy * sz, sx * sy * sz};
        T v = sg[0] > 0 ? s[0] : -s[0];
#pragma unroll
        for (int t = 1; t < 13; ++t) v = sg[t] > 0 ? add(v, s[t]) : sub(v, s[t]);
        child[c] = add(v, centre);
      }
    } else {
      const T wm[3] = {T(0.15625), T(0.9375), T(-0.09375)};  // Mm = {5, 30, -3}/32
      const T wp[3] = {T(-0.09375), T(0.9375), T(0.15625)};  // Mp = {-3, 30, 5}/32
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const T *wx = (c & 1) ? wp : wm, *wy = (c & 2) ? wp : wm, *wz = (c & 4) ? wp : wm;
        T v = T(0);
#pragma unroll
        for (int dk = -1; dk <= 1; ++dk)
#pragma unroll
          for (int dj = -1; dj <= 1; ++dj)
#pragma unroll
            for (int di = -1; di <= 1; ++di)
              v = add(v, mul(mul(mul(C(dk, dj, di), wz[dk + 1]), wy[dj + 1]), wx[di + 1]));
        child[c] = v;
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int x = 2 * (i - 1) + (c & 1) - U, y = 2 * (j - 1) + ((c >> 1) & 1) - U,
                z = 2 * (k - 1) + ((c >> 2) & 1) - U;
      if (U == 0 || ((unsigned)x < (unsigned)N && (unsigned)y < (unsigned)N && (unsigned)z < (unsigned)N))
        store(x, y, z, child[c]);
    }
  }
}

}  // namespace gpg
