// optim.cuh -- the Adam update shared by the trained models of libgpg.
#pragma once

#include <cstdint>

namespace gpg {

// one Adam step on n parameters: m, v moments (beta b1, b2), bias
// corrections c1 = 1 - b1^t, c2 = 1 - b2^t, step lr, epsilon eps
static __global__ void adam_kernel(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                                   const float *__restrict__ g, int64_t n, float lr, float b1, float b2, float eps,
                                   float c1, float c2) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

}  // namespace gpg
