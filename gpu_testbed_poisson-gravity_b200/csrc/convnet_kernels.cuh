// convnet_kernels.cuh -- tensor-core 3^3 convolutions of the learned
// initial-guess network (ghost-size-1 patches on their 10^3 solver cube).
//
// Activations are channels-last bfloat16, one row per cell: row m = patch *
// 1000 + (z*10 + y)*10 + x.  A convolution is an implicit GEMM
//     D[m][n] = sum_k A[m][k] B[n][k],   k = tap * CIN + c  (tap = 9(dz+1)+3(dy+1)+(dx+1))
// with A the im2col of the input (zero outside the patch cube).  A CTA of 128
// threads computes 128 rows (one per thread for the gather and the epilogue):
//   * the packed weights B (all K) sit in shared memory for the CTA's life;
//   * A is gathered 12 chunks (96 k) at a time into one of two buffers while
//     the tensor core works on the other;
//   * one thread issues tcgen05.mma (M=128, N=NOUT, K=16, BF16 -> FP32 in TMEM)
//     and commits each stage to that buffer's mbarrier;
//   * the epilogue reads the accumulators with tcgen05.ld (warp w owns TMEM
//     lanes 32w..32w+31 = its threads' rows), adds bias / applies ReLU or a
//     ReLU mask, and stores the row.
// Shared operand layout (no swizzle): chunk c (8 consecutive k) of row r at
// byte c*R*16 + r*16, i.e. 8-row x 16-byte core matrices, row groups 128 B
// apart.  The weight gradient reads the same im2col tile as an MN-major
// operand (k along MN, rows along K) against the gradient tile, also MN-major.
#pragma once

#include <cstdint>

#include "tc_common.cuh"

namespace gpg {
namespace net {

constexpr int kCells = 1000;  // 10^3 cube per patch
constexpr int kEdge = 10;
constexpr int kStageChunks = 12;

enum { EPI_RELU = 0, EPI_LINEAR_F32 = 1, EPI_MASK = 2 };

struct ConvArgs {
  const __nv_bfloat16 *x;     // [M][CIN]
  const __nv_bfloat16 *w;     // packed weights [KCH][NOUT][8]
  const float *bias;          // [NOUT] (EPI_RELU / EPI_LINEAR_F32)
  void *y;                    // [M][NOUT] bf16, or float for EPI_LINEAR_F32
  const __nv_bfloat16 *mask;  // [M][NOUT] previous activation (EPI_MASK)
  int64_t M;                  // rows = patches * 1000
  int *err;                   // set to 1 if a tensor-core wait timed out
};

template <int CIN>
struct KChunks {
  static constexpr int CPT = CIN / 8;                     // 8-k chunks per tap
  static constexpr int REAL = 27 * CPT;
  static constexpr int KCH = (REAL + 1) / 2 * 2;          // even: whole K=16 MMAs
};

// One im2col chunk (8 k values, 16 bytes) of row (patch base pb, cell v).
template <int CIN>
__device__ __forceinline__ uint4 gather_chunk(const __nv_bfloat16 *__restrict__ x, int64_t pb, int vx, int vy,
                                              int vz, bool valid, int c) {
  constexpr int CPT = KChunks<CIN>::CPT;
  uint4 val = make_uint4(0u, 0u, 0u, 0u);
  const int tap = c / CPT, cb = c - tap * CPT;
  if (valid && tap < 27) {
    const int nx = vx + (tap % 3) - 1, ny = vy + (tap / 3) % 3 - 1, nz = vz + tap / 9 - 1;
    if ((unsigned)nx < (unsigned)kEdge && (unsigned)ny < (unsigned)kEdge && (unsigned)nz < (unsigned)kEdge)
      val = __ldg(reinterpret_cast<const uint4 *>(x + (pb + (nz * kEdge + ny) * kEdge + nx) * CIN + cb * 8));
  }
  return val;
}

template <int CIN, int NOUT>
struct ConvSmem {
  static constexpr int KCH = KChunks<CIN>::KCH;
  static constexpr size_t b_bytes = size_t(KCH) * NOUT * 16;
  static constexpr size_t a_bytes = size_t(2) * kStageChunks * 128 * 16;
  static constexpr size_t bytes = b_bytes + a_bytes + 64;
};

template <int CIN, int NOUT, int EPI>
__global__ void __launch_bounds__(128) conv_fwd_kernel(const ConvArgs a) {
  using KC = KChunks<CIN>;
  using S = ConvSmem<CIN, NOUT>;
  constexpr int KCH = KC::KCH, SCH = kStageChunks;
  constexpr int NSTAGE = (KCH + SCH - 1) / SCH;
  constexpr uint32_t IDESC = tc::idesc_bf16(128, NOUT, false, false);
  static_assert(NOUT == 16 || NOUT == 32, "N");
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *sB = smem;
  unsigned char *sA = smem + S::b_bytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sA + S::a_bytes);
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + 2);
  const int tid = threadIdx.x, warp = tid >> 5;

  {
    const uint4 *src = reinterpret_cast<const uint4 *>(a.w);
    uint4 *dst = reinterpret_cast<uint4 *>(sB);
    for (int i = tid; i < KCH * NOUT; i += 128) dst[i] = src[i];
  }
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(s_tmem, 32);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;
  uint32_t issued[2] = {0u, 0u}, done[2] = {0u, 0u};

  const int64_t ntile = (a.M + 127) / 128;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t m = tile * 128 + tid;
    const bool valid = m < a.M;
    const int64_t pb = valid ? (m / kCells) * kCells : 0;
    const int v = valid ? int(m - pb) : 0;
    const int vx = v % kEdge, vy = (v / kEdge) % kEdge, vz = v / (kEdge * kEdge);
#pragma unroll 1
    for (int s = 0; s < NSTAGE; ++s) {
      const int b = s & 1;
      if (issued[b] > done[b]) {  // the stage that last used buffer b has finished reading it
        tc::mbar_wait(&bars[b], done[b] & 1u, a.err);
        ++done[b];
      }
      const int c0 = s * SCH, nch = (KCH - c0) < SCH ? (KCH - c0) : SCH;
      uint4 *dA = reinterpret_cast<uint4 *>(sA + b * SCH * 2048);
#pragma unroll 4
      for (int cc = 0; cc < nch; ++cc) dA[cc * 128 + tid] = gather_chunk<CIN>(a.x, pb, vx, vy, vz, valid, c0 + cc);
      tc::fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t aBase = tc::smem_u32(sA + b * SCH * 2048), bBase = tc::smem_u32(sB);
        for (int j = 0; j < nch / 2; ++j) {
          const uint64_t ad = tc::smem_desc(aBase + (2 * j) * 2048, 2048, 128);
          const uint64_t bd = tc::smem_desc(bBase + (c0 + 2 * j) * (NOUT * 16), NOUT * 16, 128);
          tc::mma_bf16(tmem, ad, bd, IDESC, (s > 0 || j > 0) ? 1u : 0u);
        }
        tc::mma_commit(&bars[b]);
      }
      ++issued[b];
    }
    for (int b = 0; b < 2; ++b)
      if (issued[b] > done[b]) {
        tc::mbar_wait(&bars[b], done[b] & 1u, a.err);
        ++done[b];
      }
    tc::fence_after_sync();
    float acc[NOUT];
#pragma unroll
    for (int h = 0; h < NOUT / 16; ++h) {
      float t[16];
      tc::tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(h * 16), t);
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[h * 16 + i] = t[i];
    }
    tc::tmem_wait_ld();
    if (valid) {
      if constexpr (EPI == EPI_LINEAR_F32) {
        float *y = reinterpret_cast<float *>(a.y) + m * NOUT;
#pragma unroll
        for (int n = 0; n < NOUT; n += 4)
          *reinterpret_cast<float4 *>(y + n) =
              make_float4(acc[n] + a.bias[n], acc[n + 1] + a.bias[n + 1], acc[n + 2] + a.bias[n + 2],
                          acc[n + 3] + a.bias[n + 3]);
      } else {
        __nv_bfloat16 *y = reinterpret_cast<__nv_bfloat16 *>(a.y) + m * NOUT;
#pragma unroll
        for (int n0 = 0; n0 < NOUT; n0 += 8) {
          __align__(16) __nv_bfloat16 o[8];
          if constexpr (EPI == EPI_MASK) {
            const uint4 mk = *reinterpret_cast<const uint4 *>(a.mask + m * NOUT + n0);
            const __nv_bfloat16 *mv = reinterpret_cast<const __nv_bfloat16 *>(&mk);
#pragma unroll
            for (int i = 0; i < 8; ++i)
              o[i] = __float2bfloat16_rn(__bfloat162float(mv[i]) > 0.f ? acc[n0 + i] : 0.f);
          } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) o[i] = __float2bfloat16_rn(fmaxf(acc[n0 + i] + a.bias[n0 + i], 0.f));
          }
          *reinterpret_cast<uint4 *>(y + n0) = *reinterpret_cast<const uint4 *>(o);
        }
      }
    }
    tc::fence_before_sync();
    __syncthreads();  // TMEM read by all before the next tile's MMAs overwrite it
  }
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 32);
  }
}

// ---------------------------------------------------------------------------
// weight gradient: dW[k][n] = sum_m A[m][k] G[m][n], per CTA over its row
// tiles, k in tiles of 128 (TMEM columns kt*NOUT..), written as partial sums
// partial[cta][k][n] (k < KT*128) for a deterministic second-stage reduction.
// ---------------------------------------------------------------------------
struct WgradArgs {
  const __nv_bfloat16 *x;  // [M][CIN]  layer input
  const __nv_bfloat16 *g;  // [M][NOUT] gradient wrt the layer's pre-activation
  float *partial;          // [gridDim.x][KT*128][NOUT]
  int64_t M;
  int *err;
};

template <int CIN, int NOUT>
struct WgradCfg {
  static constexpr int KCH = KChunks<CIN>::REAL;          // real chunks
  static constexpr int KT = (KCH + 15) / 16;              // k tiles of 128
  static constexpr int COLS0 = KT * NOUT;
  static constexpr int COLS = COLS0 <= 32 ? 32 : COLS0 <= 64 ? 64 : COLS0 <= 128 ? 128 : 256;
  static constexpr size_t bytes = size_t(16) * 2048 + size_t(NOUT / 8) * 2048 + 64;
  static_assert(COLS0 <= 256, "TMEM columns");
};

template <int CIN, int NOUT>
__global__ void __launch_bounds__(128) conv_wgrad_kernel(const WgradArgs a) {
  using W = WgradCfg<CIN, NOUT>;
  constexpr int KT = W::KT, KCHR = W::KCH;
  constexpr uint32_t IDESC = tc::idesc_bf16(128, NOUT, true, true);
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char *sA = smem;                    // 16 chunks x 128 rows
  unsigned char *sG = smem + 16 * 2048;        // NOUT/8 chunks x 128 rows
  uint64_t *bar = reinterpret_cast<uint64_t *>(sG + (NOUT / 8) * 2048);
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;

  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(s_tmem, W::COLS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *s_tmem;
  uint32_t issued = 0u, done = 0u;
  bool any = false;

  const int64_t ntile = (a.M + 127) / 128;
  for (int64_t tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
    const int64_t m = tile * 128 + tid;
    const bool valid = m < a.M;
    const int64_t pb = valid ? (m / kCells) * kCells : 0;
    const int v = valid ? int(m - pb) : 0;
    const int vx = v % kEdge, vy = (v / kEdge) % kEdge, vz = v / (kEdge * kEdge);
    if (issued > done) {  // previous MMAs read sA / sG
      tc::mbar_wait(bar, done & 1u, a.err);
      ++done;
    }
    {
      uint4 *dG = reinterpret_cast<uint4 *>(sG);
#pragma unroll
      for (int nc = 0; nc < NOUT / 8; ++nc)
        dG[nc * 128 + tid] = valid ? __ldg(reinterpret_cast<const uint4 *>(a.g + m * NOUT + nc * 8))
                                   : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll 1
    for (int kt = 0; kt < KT; ++kt) {
      if (issued > done) {
        tc::mbar_wait(bar, done & 1u, a.err);
        ++done;
      }
      uint4 *dA = reinterpret_cast<uint4 *>(sA);
#pragma unroll 4
      for (int cc = 0; cc < 16; ++cc) {
        const int c = kt * 16 + cc;
        dA[cc * 128 + tid] = c < KCHR ? gather_chunk<CIN>(a.x, pb, vx, vy, vz, valid, c) : make_uint4(0u, 0u, 0u, 0u);
      }
      tc::fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t aBase = tc::smem_u32(sA), gBase = tc::smem_u32(sG);
        for (int jj = 0; jj < 8; ++jj) {  // K = 16 rows per MMA
          const uint64_t ad = tc::smem_desc(aBase + jj * 256, 128, 2048);
          const uint64_t gd = tc::smem_desc(gBase + jj * 256, 128, 2048);
          tc::mma_bf16(tmem + uint32_t(kt * NOUT), ad, gd, IDESC, (any || jj > 0) ? 1u : 0u);
        }
        tc::mma_commit(bar);
      }
      ++issued;
    }
    any = true;
  }
  if (issued > done) {
    tc::mbar_wait(bar, done & 1u, a.err);
    ++done;
  }
  tc::fence_after_sync();
  float *out = a.partial + int64_t(blockIdx.x) * (KT * 128) * NOUT;
#pragma unroll 1
  for (int kt = 0; kt < KT; ++kt) {
    const int k = kt * 128 + warp * 32 + (tid & 31);
#pragma unroll
    for (int h = 0; h < NOUT / 16; ++h) {
      float t[16];
      tc::tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(kt * NOUT + h * 16), t);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 16; ++i) out[int64_t(k) * NOUT + h * 16 + i] = any ? t[i] : 0.f;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, W::COLS);
  }
}

}  // namespace net
}  // namespace gpg
