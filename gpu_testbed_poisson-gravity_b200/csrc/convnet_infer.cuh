// convnet_infer.cuh -- the whole forward pass of the learned initial guess in
// one persistent kernel: one patch at a time per CTA, its activations resident
// in shared memory from the interpolated input to the predicted interior.
//
// Layout.  A patch's 10^3 solver cube is stored as rows
// row = (z+1)*121 + (y+1)*11 + (x+1) for cube cell (x, y, z): lines of 11
// rows (10 cells and one zero halo column) and planes of 11 lines (10 and one
// zero halo line), with zero halo planes before and after.  A neighbour one
// step outside the cube in x (or y) wraps onto the halo column (line) that
// follows, so one zero slot serves both sides.  Each row holds the cell's
// channels as 16-byte chunks, chunk c of row r at c*1331*16 + r*16 (the
// no-swizzle K-major core-matrix layout: 8 rows x 16 bytes contiguous;
// consecutive chunks share their zero end planes, see kChunkRows).  Because
// rows are contiguous, the im2col operand of tap (dz, dy, dx) for a 128-row
// tile is the same buffer read from a start row shifted by
// off = 121 dz + 11 dy + dx: the convolution needs no gather at all, only one
// shared-memory descriptor per (tile, tap, K half).  The zero halo supplies the
// "same" padding; tile rows that are not cube cells produce values that the
// epilogue discards (their reads stay inside the kernel's shared memory).
//
// Roles (17 warps):
//   * producer warp (lane 0): streams the weights in 6 units per patch (up
//     to 28 KB: 14 taps of a 32 -> 32 layer) through a 2-slot ring with TMA bulk
//     copies (cp.async.bulk into this CTA alone), refilling a slot once the MMAs
//     that read it have completed (tcgen05.commit -> "empty" mbarrier).  The
//     stream runs across layers and patches, so the next layer's weights land
//     during the epilogue;
//   * 16 compute warps, per patch: interpolate the coarse potential (CQUAD,
//     same arithmetic as the SOR) into scratch, s = max |shell|, build the
//     8-channel input rows; then per layer thread 0 issues tcgen05.mma for
//     every tile as each unit lands (M=128, N=32 or 16, K=16, BF16 -> FP32 in
//     TMEM; all 10 tiles of a patch accumulate at once in 320 TMEM columns,
//     layer 4's 8 tiles in the next 128)
//     -- it waits only for weights, never for MMAs; one mbarrier wait per
//     unit of up to 280 MMAs -- and all 16 warps run the epilogue (tcgen05.ld; bias,
//     ReLU, BF16) into the other activation buffer; layer 4 writes (y + b) * s
//     of output channel 0 on the 8^3 interior straight to the guess array.
// Every operation and its order matches the per-layer kernels of
// convnet_kernels.cuh (same K order per output row, same epilogue
// arithmetic), so both paths produce the same guess.
#pragma once

#include <cstdint>

#include "convnet_kernels.cuh"
#include "interp.cuh"
#include "tc_common.cuh"

namespace gpg {
namespace net {

constexpr int kLine = 11;               // rows per y line: 10 cells + 1 shared halo column
constexpr int kPlane = 121;             // rows per z plane: 10 lines + 1 shared halo line
constexpr int kRowCube = 133;           // row of cube cell (0,0,0) = 121 + 11 + 1
constexpr int kRowInterior = 266;       // row of interior cell (1,1,1)
constexpr int kMaxOffset = 133;         // largest |tap offset|
constexpr int kTilesCube = 10;          // 128-row tiles over rows 133..1412 (cube rows end at 1330)
constexpr int kTilesInterior = 8;       // 128-row tiles over rows 266..1289 (interior rows end at 1197)
constexpr int kColsL4 = kTilesCube * 32;  // layer-4 accumulators follow those of layers 1-3 in TMEM
// Chunk regions are chained 1331 rows apart: the halo plane after a chunk's
// last cell plane (rows 1331..1451) is the halo plane before the next chunk's
// first (rows 0..120).  Both are zero for the kernel's life, so sharing them
// is exact.  The far corner's neighbour (+1, +1, +1) of cell (9, 9, 9) is row
// 1463, one plane further (the next chunk's halo line and column): the chain
// therefore ends with two zero planes after the last chunk, not one.
constexpr int kChunkRows = 11 * kPlane;
constexpr uint32_t kChunkBytes = kChunkRows * 16u;
constexpr uint32_t kChainBytes = (8u * kChunkRows + 2u * kPlane) * 16u;  // buffers A and B, 4 chunks each
// The issuing thread's wait for a weight unit slows the MMAs that follow it
// (about 1k cycles per wait measured on B200), so units are as large as the
// shared memory left by the activations allows: two 28 KB slots, 6 units per
// patch (layer 1's 14 tap pairs; 14 + 13 taps of each 32 -> 32 layer; layer
// 4's 27 taps).  While the tensor core works through one slot (>= 260 MMAs)
// the producer refills the other.
constexpr int kRing = 2;                // weight ring slots
constexpr uint32_t kSlotBytes = 14 * 2048;
__host__ __device__ constexpr int units_of_layer(int l) { return l == 0 || l == 3 ? 1 : 2; }
__host__ __device__ constexpr int first_unit(int l) { return l == 0 ? 0 : l == 1 ? 1 : l == 2 ? 3 : 5; }
constexpr int kUnitsPerPatch = 6;
constexpr int kComputeThreads = 512;                // 16 warps: input, MMA issue (thread 0), epilogues
constexpr int kInferThreads = kComputeThreads + 32; // + one producer warp for the weight ring
constexpr int kTileGroups = kComputeThreads / 128;  // warps sharing one TMEM lane quarter

struct InferSmem {
  static constexpr uint32_t buf_a = 0;
  static constexpr uint32_t buf_b = 4 * kChunkBytes;
  // control data in the gap between the activation chain and the ring (no
  // descriptor read reaches it)
  static constexpr uint32_t bias = kChainBytes;                 // 32 + 32 + 32 + 16 floats
  static constexpr uint32_t bars = bias + 112 * 4;             // full[kRing], empty[kRing], acc
  static constexpr uint32_t tmem_slot = bars + (2 * kRing + 1) * 8;
  static constexpr uint32_t red = tmem_slot + 16;              // one float per compute warp
  static constexpr uint32_t flag = red + 4 * (kComputeThreads / 32);  // abort flag
  static constexpr uint32_t probe = flag + 8;                  // test-hook barrier (never signalled)
  static constexpr uint32_t ring = (flag + 16 + 1023u) & ~1023u;
  static constexpr uint32_t bytes = ring + kRing * kSlotBytes;
};
static_assert(InferSmem::bytes <= 232448, "shared memory per CTA");
static_assert(InferSmem::bars % 8 == 0 && InferSmem::probe % 8 == 0, "mbarrier alignment");
// the farthest descriptor read: buffer B, chunk 3, rows up to 133 + 128*9 + 133 + 127 = 1545
static_assert(InferSmem::buf_b + 3 * kChunkBytes + (kRowCube + 128 * kTilesCube + kMaxOffset) * 16 <= kChainBytes,
              "shifted tile reads stay inside the activation chain");
static_assert(kColsL4 + kTilesInterior * 16 <= 512, "TMEM columns");
// every read of a kept (cube) row stays inside the zero-filled chain
static_assert(InferSmem::buf_b + 3 * kChunkBytes + (10 * kPlane + 10 * kLine + 10 + kMaxOffset + 1) * 16 <= kChainBytes,
              "kept rows read only the zero-filled chain");
static_assert(InferSmem::ring % 128 == 0, "ring alignment");

struct InferArgs {
  const float *rho;              // [P][8]^3
  const float *pot_in;           // [P][8]^3 coarse potential
  float *guess;                  // [P][8]^3
  const __nv_bfloat16 *w[4];     // packed forward operands (pack_kernel layout)
  const float *bias[4];          // FP32 biases (32, 32, 32, 16)
  float cnst;                    // Poi_Coeff * dh^2
  int64_t npatch;
  int *err;
  int probe_polls;               // > 0: thread 0 also waits that many polls on a barrier nothing signals
};

__host__ __device__ constexpr int tap_offset(int t) {
  return (t / 9 - 1) * kPlane + ((t / 3) % 3 - 1) * kLine + (t % 3 - 1);
}
static_assert(tap_offset(26) == kMaxOffset && tap_offset(0) == -kMaxOffset, "tap offsets");

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)), "r"(bytes)
               : "memory");
}

// TMA bulk copy global -> this CTA's shared memory, completion on `bar`
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   tc::smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ uint32_t tmem_ld1(uint32_t taddr) {
  uint32_t r;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr) : "memory");
  return r;
}

// weight unit u (0..5) of the per-patch stream: its layer, first tap (tap
// pair for layer 1), number of taps and bytes.  A tap's packed operand is
// 2 KB (32 -> 32) or 1 KB (layer 4, and a tap pair of layer 1).
struct Unit {
  int layer, t0, ntap;
  uint32_t tap_bytes;
};
__host__ __device__ constexpr Unit unit_info(int u) {
  return u < 1   ? Unit{0, 0, 14, 1024u}
         : u < 3 ? Unit{1, 14 * (u - 1), u == 1 ? 14 : 13, 2048u}
         : u < 5 ? Unit{2, 14 * (u - 3), u == 3 ? 14 : 13, 2048u}
                 : Unit{3, 0, 27, 1024u};
}
static_assert(unit_info(0).ntap == 14 && unit_info(2).t0 + unit_info(2).ntap == 27 &&
                  unit_info(4).t0 + unit_info(4).ntap == 27 && unit_info(5).ntap == 27 &&
                  unit_info(1).ntap * unit_info(1).tap_bytes <= kSlotBytes &&
                  unit_info(5).ntap * unit_info(5).tap_bytes <= kSlotBytes &&
                  first_unit(3) + units_of_layer(3) == kUnitsPerPatch,
              "units cover every tap and fit a slot");
__device__ __forceinline__ const unsigned char *unit_src(const InferArgs &a, int u, uint32_t &bytes) {
  const Unit un = unit_info(u);
  bytes = uint32_t(un.ntap) * un.tap_bytes;
  return reinterpret_cast<const unsigned char *>(a.w[un.layer]) + uint32_t(un.t0) * un.tap_bytes;
}

// one weight unit: NT tiles x KH K-halves of M=128 MMAs into TMEM columns
// i*NCOLS.  Descriptor steps are in units of the 16-byte start-address field.
template <int NT, int KH, int NCOLS>
__device__ __forceinline__ void issue_unit(uint32_t tmem, uint64_t a0, uint32_t a_step, uint64_t b0, uint32_t b_step,
                                           uint32_t idesc, uint32_t acc_first) {
#pragma unroll
  for (int i = 0; i < NT; ++i)
#pragma unroll
    for (int jj = 0; jj < KH; ++jj)
      tc::mma_bf16(tmem + uint32_t(i * NCOLS), a0 + uint64_t(i * 128 + jj * a_step), b0 + uint64_t(jj * b_step), idesc,
                   jj > 0 ? 1u : acc_first);
}

// named barrier over the compute warps (the producer warp never joins)
__device__ __forceinline__ void compute_sync() {
  asm volatile("bar.sync 1, %0;" ::"n"(kComputeThreads) : "memory");
}
// the same barrier, returning whether any compute thread passed `v` true
__device__ __forceinline__ bool compute_sync_or(bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"(v ? 1u : 0u), "n"(kComputeThreads)
      : "memory");
  return r != 0;
}

__global__ void __launch_bounds__(kInferThreads, 1) net_infer_kernel(const InferArgs a) {
  using S = InferSmem;
  extern __shared__ __align__(1024) unsigned char infer_smem[];
  unsigned char *smem = infer_smem;
  unsigned char *buf_a = smem + S::buf_a, *buf_b = smem + S::buf_b, *ring = smem + S::ring;
  float *s_bias = reinterpret_cast<float *>(smem + S::bias);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S::bars), *empty = full + kRing, *accb = full + 2 * kRing;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + S::tmem_slot);
  float *s_red = reinterpret_cast<float *>(smem + S::red);
  volatile int *s_abort = reinterpret_cast<volatile int *>(smem + S::flag);
  // scratch for the interpolated cube: buffer B chunk 1, rows 0..249 (the
  // first 121 are chunk 0's last halo plane); zeroed again before layer 1
  float *cube = reinterpret_cast<float *>(buf_b + kChunkBytes);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quarter = warp & 3, group = warp >> 2;  // TMEM lanes 32*quarter.., tiles group, group+4, ...

  // both activation buffers start at zero; the epilogues write cube rows only,
  // so the halo rows stay zero for the kernel's life
  for (uint32_t i = tid; i < kChainBytes / 16; i += kInferThreads)
    reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
  for (int i = tid; i < 112; i += kInferThreads)
    s_bias[i] = i < 32 ? a.bias[0][i] : i < 64 ? a.bias[1][i - 32] : i < 96 ? a.bias[2][i - 64] : a.bias[3][i - 96];
  if (tid == 0) {
    for (int s = 0; s < kRing; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(accb, 1);
    tc::mbar_init(reinterpret_cast<uint64_t *>(smem + S::probe), 1);
    *s_abort = 0;
    tc::mbar_fence_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(s_tmem, 512);
    tc::tmem_relinquish();
  }
  tc::fence_proxy_async_smem();
  tc::fence_before_sync();
  __syncthreads();  // the last barrier all 9 warps take
  tc::fence_after_sync();
  if (a.probe_polls > 0 && tid == 0) {
    // test hook: a bounded wait on a barrier nothing arrives on gives up
    // after probe_polls polls, records the timeout and the kernel goes on
    tc::mbar_wait_polls(reinterpret_cast<uint64_t *>(smem + S::probe), 0, a.err, uint32_t(a.probe_polls));
  }

  const int64_t my_patches = a.npatch > blockIdx.x ? (a.npatch - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int64_t total_units = my_patches * kUnitsPerPatch;

  // ---- producer warp: stream the weight units through the ring -------------
  if (warp == kComputeThreads / 32) {
    if (lane == 0) {
      int64_t q_load = 0;
      for (int64_t q = 0; q < total_units; ++q) {
        if (*s_abort) break;
        const int slot = int(q % kRing);
        // the slot is free once the MMAs of unit q - kRing have completed
        if (q >= kRing && !tc::mbar_wait(&empty[slot], uint32_t((q / kRing) - 1) & 1u, a.err)) {
          *s_abort = 1;
          break;
        }
        uint32_t bytes;
        const unsigned char *src = unit_src(a, int(q % kUnitsPerPatch), bytes);
        mbar_expect_tx(&full[slot], bytes);
        bulk_load(ring + slot * kSlotBytes, src, bytes, &full[slot]);
        q_load = q + 1;
      }
      // the last copies (one per slot) land before this warp leaves
      for (int64_t q = q_load > kRing ? q_load - kRing : 0; q < q_load; ++q)
        tc::mbar_wait(&full[q % kRing], uint32_t(q / kRing) & 1u, nullptr);
    }
    return;
  }

  // ---- compute warps --------------------------------------------------------
  const uint32_t tmem = *s_tmem;
  int64_t q_use = 0;  // thread 0: weight units consumed
  uint32_t acc_phase = 0;
  bool failed = false;

  constexpr uint32_t IDESC32 = tc::idesc_bf16(128, 32, false, false);
  constexpr uint32_t IDESC16 = tc::idesc_bf16(128, 16, false, false);
  constexpr uint32_t CH = kChunkBytes;  // chunk stride (leading byte offset)
  const uint32_t a_u32 = tc::smem_u32(buf_a), b_u32 = tc::smem_u32(buf_b), ring_u32 = tc::smem_u32(ring);

  // thread 0: all MMAs of one layer and the accumulator commit; it waits only
  // for weight units to land, never for MMAs to complete
  auto issue_layer = [&](int layer) {
    for (int u = first_unit(layer); u < first_unit(layer) + units_of_layer(layer); ++u) {
      if (failed) break;
      const int slot = int(q_use % kRing);
      if (!tc::mbar_wait(&full[slot], uint32_t(q_use / kRing) & 1u, a.err)) {
        failed = true;
        *s_abort = 1;
        break;
      }
      // the wait observed the copy's completion; this fence orders the
      // asynchronous MMAs below after it (without it they may read the slot
      // before the copy has landed)
      tc::fence_after_sync();
      const Unit un = unit_info(u);
      for (int k = 0; k < un.ntap; ++k) {
        const uint32_t wsl = ring_u32 + slot * kSlotBytes + uint32_t(k) * un.tap_bytes;
        const int t = un.t0 + k;
        // descriptors are built once per tap; a tile (128 rows of 16 bytes)
        // adds 128 to the 16-byte start-address field, a K half 2 chunks
        if (layer == 0) {  // t = tap pair (2t, 2t+1); pair 13 = tap 26 + a zero tap
          const uint32_t lbo = t < 13 ? uint32_t(tap_offset(2 * t + 1) - tap_offset(2 * t)) * 16u : 16u;
          issue_unit<kTilesCube, 1, 32>(tmem,
                                        tc::smem_desc(b_u32 + uint32_t(kRowCube + tap_offset(2 * t)) * 16u, lbo, 128),
                                        0, tc::smem_desc(wsl, 512, 128), 0, IDESC32, t > 0 ? 1u : 0u);
        } else if (layer < 3) {
          const uint32_t src = layer == 1 ? a_u32 : b_u32;
          issue_unit<kTilesCube, 2, 32>(tmem, tc::smem_desc(src + uint32_t(kRowCube + tap_offset(t)) * 16u, CH, 128),
                                        2 * CH / 16, tc::smem_desc(wsl, 512, 128), 1024 / 16, IDESC32,
                                        t > 0 ? 1u : 0u);
        } else {
          issue_unit<kTilesInterior, 2, 16>(
              tmem + kColsL4, tc::smem_desc(a_u32 + uint32_t(kRowInterior + tap_offset(t)) * 16u, CH, 128), 2 * CH / 16,
              tc::smem_desc(wsl, 256, 128), 512 / 16, IDESC16, t > 0 ? 1u : 0u);
        }
      }
      tc::mma_commit(&empty[slot]);  // the producer may refill the slot once these MMAs are done
      ++q_use;
    }
    tc::mma_commit(accb);  // also on failure, so that the other threads' wait ends
  };

  // wait for the layer's accumulators: thread 0 polls the mbarrier, the other
  // compute threads block on the named barrier (polling from 256 threads
  // would take shared-memory bandwidth from the tensor core's operand reads)
  auto wait_acc = [&]() {
    if (tid == 0 && !tc::mbar_wait(accb, acc_phase & 1u, a.err)) failed = true;
    ++acc_phase;
    tc::fence_before_sync();
    failed = compute_sync_or(failed);
    tc::fence_after_sync();
  };

  // epilogue of layers 1-3: bias + ReLU -> bf16 rows of `dst`
  auto epilogue_relu = [&](unsigned char *dst, const float *bias) {
    for (int i = group; i < kTilesCube; i += kTileGroups) {
      float v[32];
      float (&v0)[16] = *reinterpret_cast<float(*)[16]>(v);
      float (&v1)[16] = *reinterpret_cast<float(*)[16]>(v + 16);
      const uint32_t ta = tmem + (uint32_t(32 * quarter) << 16) + uint32_t(i * 32);
      tc::tmem_ld16(ta, v0);
      tc::tmem_ld16(ta + 16, v1);
      tc::tmem_wait_ld();
      const int row = kRowCube + 128 * i + 32 * quarter + lane;
      const int z = row / kPlane, r2 = row - z * kPlane, y = r2 / kLine, x = r2 - y * kLine;
      if (x >= 1 && y >= 1 && z >= 1 && z <= 10) {  // x, y <= 10 always
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          __align__(16) __nv_bfloat16 o[8];
#pragma unroll
          for (int e = 0; e < 8; ++e) o[e] = __float2bfloat16_rn(fmaxf(v[8 * c + e] + bias[8 * c + e], 0.f));
          *reinterpret_cast<uint4 *>(dst + c * CH + row * 16) = *reinterpret_cast<const uint4 *>(o);
        }
      }
    }
  };

  auto end_phase = [&]() -> bool {  // smem writes -> tensor core; true when any thread failed
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    const bool stop = compute_sync_or(failed);
    tc::fence_after_sync();
    return stop;
  };

  for (int64_t p = blockIdx.x; p < a.npatch; p += gridDim.x) {
    // ---- input rows (layer-1 operand, buffer B chunk 0) -------------------
    interpolate<float, 1, kComputeThreads>(a.pot_in + p * Geo<1>::PN3, tid, 4,
                                           [cube](int x, int y, int z, float v) { cube[(z * 10 + y) * 10 + x] = v; });
    compute_sync();
    float mx = 0.f;
    for (int v = tid; v < kCells; v += kComputeThreads) {
      const int x = v % 10, y = (v / 10) % 10, z = v / 100;
      if (x == 0 || y == 0 || z == 0 || x == 9 || y == 9 || z == 9) mx = fmaxf(mx, fabsf(cube[v]));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) s_red[warp] = mx;
    compute_sync();
    float s = s_red[0];
    for (int w = 1; w < kComputeThreads / 32; ++w) s = fmaxf(s, s_red[w]);
    if (!(s > 0.f)) s = 1.f;
    for (int v = tid; v < kCells; v += kComputeThreads) {
      const int x = v % 10, y = (v / 10) % 10, z = v / 100;
      const bool shell = x == 0 || y == 0 || z == 0 || x == 9 || y == 9 || z == 9;
      __align__(16) __nv_bfloat16 o[8];
      const float r = shell ? 0.f : __fmul_rn(a.cnst, a.rho[p * 512 + ((z - 1) * 8 + (y - 1)) * 8 + (x - 1)]) / s;
      o[0] = __float2bfloat16_rn(r);
      o[1] = __float2bfloat16_rn(shell ? cube[v] / s : 0.f);
      o[2] = __float2bfloat16_rn(shell ? 0.f : 1.f);
#pragma unroll
      for (int i = 3; i < 8; ++i) o[i] = __float2bfloat16_rn(0.f);
      const int row = (z + 1) * kPlane + (y + 1) * kLine + (x + 1);
      *reinterpret_cast<uint4 *>(buf_b + row * 16) = *reinterpret_cast<const uint4 *>(o);
    }
    compute_sync();
    for (int i = tid; i < kCells / 4; i += kComputeThreads) reinterpret_cast<uint4 *>(cube)[i] = make_uint4(0, 0, 0, 0);
    if (end_phase()) break;

    // ---- layers 1-3 -------------------------------------------------------
    unsigned char *dst[3] = {buf_a, buf_b, buf_a};
    bool stop = false;
    for (int l = 0; l < 3 && !stop; ++l) {
      if (warp == 0) {
        if (lane == 0) issue_layer(l);
        __syncwarp();
      }
      wait_acc();
      epilogue_relu(dst[l], s_bias + 32 * l);
      stop = end_phase();
    }
    if (stop) break;

    // ---- layer 4: channel 0 on the interior -> guess -----------------------
    if (warp == 0) {
      if (lane == 0) issue_layer(3);
      __syncwarp();
    }
    wait_acc();
    for (int i = group; i < kTilesInterior; i += kTileGroups) {
      const float y4 =
          __uint_as_float(tmem_ld1(tmem + (uint32_t(32 * quarter) << 16) + uint32_t(kColsL4 + i * 16)));
      tc::tmem_wait_ld();
      const int row = kRowInterior + 128 * i + 32 * quarter + lane;
      const int z = row / kPlane, r2 = row - z * kPlane, y = r2 / kLine, x = r2 - y * kLine;
      if (x >= 2 && x <= 9 && y >= 2 && y <= 9 && z >= 2 && z <= 9)
        a.guess[p * 512 + ((z - 2) * 8 + (y - 2)) * 8 + (x - 2)] = (y4 + s_bias[96]) * s;
    }
    if (end_phase()) break;
  }
  if (failed) *s_abort = 1;

  tc::fence_before_sync();
  compute_sync();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 512);
  }
}

}  // namespace net
}  // namespace gpg
