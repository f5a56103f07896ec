// gravity.cuh -- finite-difference acceleration and momentum/energy update of
// one patch (CPU_GravitySolver.cpp:34-79): with Gra_Const = dt/(2dh) (3-point)
// or dt/(12dh) (5-point, GRA_GHOST_SIZE == 2),
//   a     = Gra_Const * dphi
//   Eint  = E - 0.5/rho * |p|^2
//   p    -= rho * a
//   E     = Eint + 0.5/rho * |p|^2
// The density component is read, never written.
#pragma once

#include "common.cuh"

namespace gpg {

// `phi(i, j, k)` returns the potential at patch-cell offset (i, j, k), which
// ranges over [-2, 10) (x fastest).  flu points at one patch [5][8][8][8].
template <typename T, int NT, typename Phi>
__device__ __forceinline__ void gravity_patch(T *__restrict__ flu, int tid, T gra_const, int p5,
                                              Phi phi) {
  constexpr int PS3 = 512;
  const T c8 = T(8);
  for (int c = tid; c < PS3; c += NT) {
    const int i = c & 7, j = (c >> 3) & 7, k = c >> 6;
    T ax, ay, az;
    if (p5) {
      ax = mul(gra_const, sub(add(add(-phi(i + 2, j, k), phi(i - 2, j, k)), mul(c8, phi(i + 1, j, k))),
                              mul(c8, phi(i - 1, j, k))));
      ay = mul(gra_const, sub(add(add(-phi(i, j + 2, k), phi(i, j - 2, k)), mul(c8, phi(i, j + 1, k))),
                              mul(c8, phi(i, j - 1, k))));
      az = mul(gra_const, sub(add(add(-phi(i, j, k + 2), phi(i, j, k - 2)), mul(c8, phi(i, j, k + 1))),
                              mul(c8, phi(i, j, k - 1))));
    } else {
      ax = mul(gra_const, sub(phi(i + 1, j, k), phi(i - 1, j, k)));
      ay = mul(gra_const, sub(phi(i, j + 1, k), phi(i, j - 1, k)));
      az = mul(gra_const, sub(phi(i, j, k + 1), phi(i, j, k - 1)));
    }
    const T rho = flu[c];
    T px = flu[PS3 + c], py = flu[2 * PS3 + c], pz = flu[3 * PS3 + c];
    const T e = flu[4 * PS3 + c];
    const T temp = divide(T(0.5), rho);
    const T eint = sub(e, mul(temp, add(add(mul(px, px), mul(py, py)), mul(pz, pz))));
    px = sub(px, mul(rho, ax));
    py = sub(py, mul(rho, ay));
    pz = sub(pz, mul(rho, az));
    flu[PS3 + c] = px;
    flu[2 * PS3 + c] = py;
    flu[3 * PS3 + c] = pz;
    flu[4 * PS3 + c] = add(eint, mul(temp, add(add(mul(px, px), mul(py, py)), mul(pz, pz))));
  }
}

// Gravity alone (Poisson off): the potential comes from pot_out
// [P][GRA_NXT]^3.  One CTA of 256 threads per patch; the GRA window is staged
// in shared memory first.
template <typename T, int GG>
__global__ void __launch_bounds__(256) gravity_kernel(T *__restrict__ flu, const T *__restrict__ pot,
                                                      int64_t npatch, T gra_const, int p5) {
  constexpr int GN = 8 + 2 * GG, GN3 = GN * GN * GN;
  __shared__ T s_pot[GN3];
  const int64_t P = blockIdx.x;
  if (P >= npatch) return;
  const T *src = pot + P * GN3;
  for (int t = threadIdx.x; t < GN3; t += 256) s_pot[t] = src[t];
  __syncthreads();
  gravity_patch<T, 256>(flu + P * 5 * 512, threadIdx.x, gra_const, p5, [&](int i, int j, int k) {
    return s_pot[((k + GG) * GN + (j + GG)) * GN + (i + GG)];
  });
}

}  // namespace gpg
