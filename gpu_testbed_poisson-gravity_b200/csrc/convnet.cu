// convnet.cu -- the learned initial guess for ghost-size-1 SOR: a 4-layer
// 3^3 convolution network (8 -> 32 -> 32 -> 32 -> 16 channels, ReLU, output
// channel 0 used) that maps a patch's density and interpolated boundary shell
// to its interior potential.  Forward, backward and the Adam update run on the
// tensor-core kernels of convnet_kernels.cuh and the small kernels below;
// weights are FP32 masters packed to BF16 for the MMAs.  C-ABI: gpg_net_* in
// include/gpg.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gpg.h"
#include "common.cuh"
#include "convnet_kernels.cuh"
#include "convnet_infer.cuh"
#include "interp.cuh"
#include "optim.cuh"

using gpg::net::ConvArgs;
using gpg::net::WgradArgs;
using gpg::net::kCells;

namespace {

thread_local std::string g_net_error;

int nfail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_net_error = buf;
  return status;
}

#define NET_CUDA(call)                                                                               \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return nfail(e_ == cudaErrorMemoryAllocation ? GPG_ERR_OOM : GPG_ERR_CUDA, "%s: %s (%s:%d)", #call, \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                                      \
  } while (0)

// layer shapes (input channels padded to 8, output channels of the last layer to 16)
constexpr int kLayers = 4;
constexpr int kCin[kLayers] = {8, 32, 32, 32};
constexpr int kCout[kLayers] = {32, 32, 32, 16};
constexpr int kRealCin0 = 3;   // density, boundary shell, interior mask
constexpr int kRealCout3 = 1;  // the potential

constexpr int64_t w_count(int l) { return int64_t(27) * kCin[l] * kCout[l]; }
constexpr int64_t param_offset_w(int l) {
  int64_t o = 0;
  for (int i = 0; i < l; ++i) o += w_count(i) + kCout[i];
  return o;
}
constexpr int64_t param_offset_b(int l) { return param_offset_w(l) + w_count(l); }
constexpr int64_t kParams = param_offset_w(kLayers);

// ---------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------

// interpolated 10^3 cube of a ghost-1 patch (the SOR's initial cube)
__global__ void __launch_bounds__(128) interp_cube_kernel(const float *__restrict__ pot_in, float *__restrict__ cube,
                                                          int64_t npatch) {
  const int64_t p = blockIdx.x;
  if (p >= npatch) return;
  float *dst = cube + p * kCells;
  gpg::interpolate<float, 1, 128>(pot_in + p * gpg::Geo<1>::PN3, threadIdx.x, 4,
                                  [dst](int x, int y, int z, float v) { dst[(z * 10 + y) * 10 + x] = v; });
}

// X0 [P*1000][8] bf16 and the per-patch scale s = max |shell potential|
__global__ void __launch_bounds__(256) prep_input_kernel(const float *__restrict__ rho, const float *__restrict__ cube,
                                                         __nv_bfloat16 *__restrict__ x0, float *__restrict__ scale,
                                                         float cnst, int64_t npatch) {
  const int64_t p = blockIdx.x;
  if (p >= npatch) return;
  __shared__ float red[8];
  float mx = 0.f;
  for (int v = threadIdx.x; v < kCells; v += 256) {
    const int x = v % 10, y = (v / 10) % 10, z = v / 100;
    const bool shell = x == 0 || y == 0 || z == 0 || x == 9 || y == 9 || z == 9;
    if (shell) mx = fmaxf(mx, fabsf(cube[p * kCells + v]));
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  float s = red[0];
  for (int w = 1; w < 8; ++w) s = fmaxf(s, red[w]);
  if (!(s > 0.f)) s = 1.f;
  if (threadIdx.x == 0) scale[p] = s;
  for (int v = threadIdx.x; v < kCells; v += 256) {
    const int x = v % 10, y = (v / 10) % 10, z = v / 100;
    const bool shell = x == 0 || y == 0 || z == 0 || x == 9 || y == 9 || z == 9;
    __align__(16) __nv_bfloat16 o[8];
    const float r = shell ? 0.f : __fmul_rn(cnst, rho[p * 512 + ((z - 1) * 8 + (y - 1)) * 8 + (x - 1)]) / s;
    o[0] = __float2bfloat16_rn(r);
    o[1] = __float2bfloat16_rn(shell ? cube[p * kCells + v] / s : 0.f);
    o[2] = __float2bfloat16_rn(shell ? 0.f : 1.f);
#pragma unroll
    for (int i = 3; i < 8; ++i) o[i] = __float2bfloat16_rn(0.f);
    *reinterpret_cast<uint4 *>(x0 + (p * kCells + v) * 8) = *reinterpret_cast<const uint4 *>(o);
  }
}

// loss partials and G4 = d loss / d y4 (channel 0 on interior cells)
__global__ void __launch_bounds__(256) loss_grad_kernel(const float *__restrict__ y4, const float *__restrict__ target,
                                                        const float *__restrict__ scale, __nv_bfloat16 *__restrict__ g4,
                                                        double *__restrict__ loss_part, int64_t npatch) {
  const int64_t M = npatch * kCells;
  const double inv = 1.0 / double(npatch * 512);
  double l = 0.0;
  for (int64_t m = blockIdx.x * 256 + threadIdx.x; m < M; m += int64_t(gridDim.x) * 256) {
    const int64_t p = m / kCells;
    const int v = int(m - p * kCells);
    const int x = v % 10, y = (v / 10) % 10, z = v / 100;
    const bool interior = x > 0 && y > 0 && z > 0 && x < 9 && y < 9 && z < 9;
    __align__(16) __nv_bfloat16 o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] = __float2bfloat16_rn(0.f);
    if (interior) {
      const float t = target[p * 512 + ((z - 1) * 8 + (y - 1)) * 8 + (x - 1)] / scale[p];
      const double d = double(y4[m * 16]) - double(t);
      l += d * d;
      o[0] = __float2bfloat16_rn(float(2.0 * d * inv));
    }
    uint4 *dst = reinterpret_cast<uint4 *>(g4 + m * 16);
    dst[0] = reinterpret_cast<const uint4 *>(o)[0];
    dst[1] = reinterpret_cast<const uint4 *>(o)[1];
  }
  __shared__ double red[8];
#pragma unroll
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    loss_part[blockIdx.x] = s * inv;
  }
}

// sum of the loss partials in a fixed order
__global__ void sum_kernel(const double *p, int n, float *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < n; ++i) t += p[i];
    *out = float(t);
  }
}

__global__ void guess_kernel(const float *__restrict__ y4, const float *__restrict__ scale, float *__restrict__ guess,
                             int64_t npatch) {
  const int64_t n = npatch * 512;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t p = i / 512;
    const int q = int(i - p * 512), x = q % 8 + 1, y = (q / 8) % 8 + 1, z = q / 64 + 1;
    guess[i] = y4[(p * kCells + (z * 10 + y) * 10 + x) * 16] * scale[p];
  }
}

// bias gradient partials: part[block][n] = sum over the block's rows of g[m][n]
template <int NOUT>
__global__ void __launch_bounds__(256) bias_grad_kernel(const __nv_bfloat16 *__restrict__ g, float *__restrict__ part,
                                                        int64_t M) {
  __shared__ float red[256][NOUT + 1];
  float acc[NOUT];
#pragma unroll
  for (int n = 0; n < NOUT; ++n) acc[n] = 0.f;
  for (int64_t m = blockIdx.x * 256 + threadIdx.x; m < M; m += int64_t(gridDim.x) * 256)
#pragma unroll
    for (int n = 0; n < NOUT; ++n) acc[n] += __bfloat162float(g[m * NOUT + n]);
#pragma unroll
  for (int n = 0; n < NOUT; ++n) red[threadIdx.x][n] = acc[n];
  __syncthreads();
  if (threadIdx.x < NOUT) {
    float s = 0.f;
    for (int t = 0; t < 256; ++t) s += red[t][threadIdx.x];
    part[blockIdx.x * NOUT + threadIdx.x] = s;
  }
}

// grad[i] = sum_c part[c][row(i)][col(i)] for one layer's weights (+ its bias)
__global__ void reduce_grad_kernel(const float *__restrict__ wpart, int nwpart, int wrows_stride, int kreal,
                                   int nout, const float *__restrict__ bpart, int nbpart, float *__restrict__ grad_w,
                                   float *__restrict__ grad_b) {
  const int nw = kreal * nout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nw + nout; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    if (i < nw) {
      for (int c = 0; c < nwpart; ++c) s += wpart[int64_t(c) * wrows_stride * nout + i];
      grad_w[i] = s;
    } else {
      const int n = i - nw;
      for (int c = 0; c < nbpart; ++c) s += bpart[c * nout + n];
      grad_b[n] = s;
    }
  }
}

// pack W[27][cin][cout] (FP32) into the forward operand [KCH][cout][8] (bf16,
// k = tap*cin + c) and, when bwd != nullptr, the backward-data operand
// [KCH'][cin][8] with k' = tap'*cout + n and W'[tap'][n][c] = W[26-tap'][c][n]
__global__ void pack_kernel(const float *__restrict__ w, int cin, int cout, int kch_f, __nv_bfloat16 *__restrict__ fwd,
                            int kch_b, __nv_bfloat16 *__restrict__ bwd) {
  const int nf = kch_f * cout * 8, nb = bwd ? kch_b * cin * 8 : 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf + nb; i += gridDim.x * blockDim.x) {
    if (i < nf) {
      const int chunk = i / (cout * 8), n = (i / 8) % cout, e = i % 8;
      const int k = chunk * 8 + e, tap = k / cin, c = k % cin;
      fwd[i] = __float2bfloat16_rn(tap < 27 ? w[(tap * cin + c) * cout + n] : 0.f);
    } else {
      const int j = i - nf;
      const int chunk = j / (cin * 8), c = (j / 8) % cin, e = j % 8;
      const int k = chunk * 8 + e, tap = k / cout, n = k % cout;
      bwd[j] = __float2bfloat16_rn(tap < 27 ? w[((26 - tap) * cin + c) * cout + n] : 0.f);
    }
  }
}

// kernel attributes belong to a device's context: set once per (kernel, device)
constexpr int kMaxDevices = 64;
struct DevOnce {
  std::once_flag once[kMaxDevices];
  cudaError_t err[kMaxDevices] = {};
};

int device_index() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -1;
  return dev;
}

template <typename F>
int set_attr_once(F *fn, size_t bytes, DevOnce &st) {
  const int dev = device_index();
  if (dev < 0) return nfail(GPG_ERR_UNSUPPORTED, "current device out of range");
  std::call_once(st.once[dev], [&] {
    cudaError_t &err = st.err[dev];
    err = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
  });
  if (st.err[dev] != cudaSuccess)
    return nfail(GPG_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(st.err[dev]));
  return GPG_OK;
}

// blocks of the bias-gradient and loss kernels = partial sums they leave
constexpr int kPartials = 148;

// SM count of the current device (cached per device)
int sm_count() {
  static int n[kMaxDevices] = {};
  const int dev = device_index();
  if (dev < 0) return 148;
  if (!n[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    n[dev] = v > 0 ? v : 148;
  }
  return n[dev];
}

template <int CIN, int NOUT, int EPI>
int launch_conv(const ConvArgs &a, cudaStream_t s) {
  static DevOnce once;
  constexpr size_t smem = gpg::net::ConvSmem<CIN, NOUT>::bytes;
  auto fn = gpg::net::conv_fwd_kernel<CIN, NOUT, EPI>;
  if (int rc = set_attr_once(fn, smem, once)) return rc;
  const int64_t ntile = (a.M + 127) / 128;
  // at most 512/32 TMEM column blocks per SM; shared memory bounds it earlier
  const int64_t grid = std::min<int64_t>(ntile, int64_t(sm_count()) * 4);
  if (grid <= 0) return GPG_OK;
  fn<<<(unsigned)grid, 128, smem, s>>>(a);
  NET_CUDA(cudaGetLastError());
  return GPG_OK;
}

template <int CIN, int NOUT>
int wgrad_grid(int64_t M) {
  using W = gpg::net::WgradCfg<CIN, NOUT>;
  const int per_sm = 512 / W::COLS;
  return (int)std::min<int64_t>((M + 127) / 128, int64_t(sm_count()) * (per_sm < 4 ? per_sm : 4));
}

template <int CIN, int NOUT>
int launch_wgrad(const WgradArgs &a, int grid, cudaStream_t s) {
  using W = gpg::net::WgradCfg<CIN, NOUT>;
  static DevOnce once;
  // shared memory sized so that the CTAs an SM holds never ask for more than
  // its 512 TMEM columns in total
  const int per_sm = 512 / W::COLS;
  const size_t smem = std::max<size_t>(W::bytes, per_sm >= 6 ? W::bytes : (220 * 1024) / per_sm);
  auto fn = gpg::net::conv_wgrad_kernel<CIN, NOUT>;
  if (int rc = set_attr_once(fn, smem, once)) return rc;
  if (grid <= 0) return GPG_OK;
  fn<<<(unsigned)grid, 128, smem, s>>>(a);
  NET_CUDA(cudaGetLastError());
  return GPG_OK;
}

}  // namespace

// ===========================================================================
// network object
// ===========================================================================
struct gpg_net {
  int device = 0;
  int max_batch = 0;
  int probe_polls = 0;  // test hook of the inference kernel (gpg_net_set_wait_probe)
  int64_t step = 0;
  float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  __nv_bfloat16 *wf[kLayers] = {}, *wb[kLayers] = {};
  __nv_bfloat16 *x0 = nullptr, *act[3] = {}, *g4 = nullptr, *ga = nullptr, *gb = nullptr;
  float *y4 = nullptr, *cube = nullptr, *scale = nullptr, *wpart = nullptr, *bpart = nullptr;
  double *loss_part = nullptr;
  int *err = nullptr;
};

namespace {

int kch_fwd(int l) { return (27 * (kCin[l] / 8) + 1) / 2 * 2; }
int kch_bwd(int l) { return (27 * (kCout[l] / 8) + 1) / 2 * 2; }

int repack(gpg_net *n, cudaStream_t s) {
  for (int l = 0; l < kLayers; ++l) {
    pack_kernel<<<64, 256, 0, s>>>(n->params + param_offset_w(l), kCin[l], kCout[l], kch_fwd(l), n->wf[l],
                                   kch_bwd(l), l > 0 ? n->wb[l] : nullptr);
  }
  NET_CUDA(cudaGetLastError());
  return GPG_OK;
}

int conv_forward_layer(gpg_net *n, int l, const __nv_bfloat16 *x, void *y, int64_t M, cudaStream_t s) {
  ConvArgs a{x, n->wf[l], n->params + param_offset_b(l), y, nullptr, M, n->err};
  switch (l) {
    case 0: return launch_conv<8, 32, gpg::net::EPI_RELU>(a, s);
    case 1:
    case 2: return launch_conv<32, 32, gpg::net::EPI_RELU>(a, s);
    default: return launch_conv<32, 16, gpg::net::EPI_LINEAR_F32>(a, s);
  }
}

// gradient wrt the input of layer l (> 0), masked by ReLU' of that input
int conv_backward_data(gpg_net *n, int l, const __nv_bfloat16 *g, __nv_bfloat16 *gout, int64_t M, cudaStream_t s) {
  ConvArgs a{g, n->wb[l], nullptr, gout, n->act[l - 1], M, n->err};
  if (l == 3) return launch_conv<16, 32, gpg::net::EPI_MASK>(a, s);
  return launch_conv<32, 32, gpg::net::EPI_MASK>(a, s);
}

int conv_weight_grad(gpg_net *n, int l, const __nv_bfloat16 *x, const __nv_bfloat16 *g, int64_t M, cudaStream_t s) {
  int grid, rows;
  WgradArgs a{x, g, n->wpart, M, n->err};
  int rc;
  if (l == 0) {
    grid = wgrad_grid<8, 32>(M);
    rows = gpg::net::WgradCfg<8, 32>::KT * 128;
    rc = launch_wgrad<8, 32>(a, grid, s);
  } else if (l < 3) {
    grid = wgrad_grid<32, 32>(M);
    rows = gpg::net::WgradCfg<32, 32>::KT * 128;
    rc = launch_wgrad<32, 32>(a, grid, s);
  } else {
    grid = wgrad_grid<32, 16>(M);
    rows = gpg::net::WgradCfg<32, 16>::KT * 128;
    rc = launch_wgrad<32, 16>(a, grid, s);
  }
  if (rc) return rc;
  const int nb = kPartials;
  if (kCout[l] == 32)
    bias_grad_kernel<32><<<nb, 256, 0, s>>>(g, n->bpart, M);
  else
    bias_grad_kernel<16><<<nb, 256, 0, s>>>(g, n->bpart, M);
  reduce_grad_kernel<<<32, 256, 0, s>>>(n->wpart, grid, rows, 27 * kCin[l], kCout[l], n->bpart, nb,
                                        n->grad + param_offset_w(l), n->grad + param_offset_b(l));
  NET_CUDA(cudaGetLastError());
  return GPG_OK;
}

int forward_all(gpg_net *n, int64_t npatch, const float *rho, const float *pot_in, float cnst, cudaStream_t s) {
  const int64_t M = npatch * kCells;
  interp_cube_kernel<<<(unsigned)npatch, 128, 0, s>>>(pot_in, n->cube, npatch);
  prep_input_kernel<<<(unsigned)npatch, 256, 0, s>>>(rho, n->cube, n->x0, n->scale, cnst, npatch);
  NET_CUDA(cudaGetLastError());
  const __nv_bfloat16 *x = n->x0;
  for (int l = 0; l < 3; ++l) {
    if (int rc = conv_forward_layer(n, l, x, n->act[l], M, s)) return rc;
    x = n->act[l];
  }
  return conv_forward_layer(n, 3, x, n->y4, M, s);
}

int gradients(gpg_net *n, int64_t npatch, const float *rho, const float *pot_in, const float *target, float cnst,
              float *loss, cudaStream_t s) {
  const int64_t M = npatch * kCells;
  if (int rc = forward_all(n, npatch, rho, pot_in, cnst, s)) return rc;
  const int nlp = kPartials;
  loss_grad_kernel<<<nlp, 256, 0, s>>>(n->y4, target, n->scale, n->g4, n->loss_part, npatch);
  NET_CUDA(cudaGetLastError());
  // layer 4, then 3, 2, 1
  if (int rc = conv_weight_grad(n, 3, n->act[2], n->g4, M, s)) return rc;
  if (int rc = conv_backward_data(n, 3, n->g4, n->ga, M, s)) return rc;
  if (int rc = conv_weight_grad(n, 2, n->act[1], n->ga, M, s)) return rc;
  if (int rc = conv_backward_data(n, 2, n->ga, n->gb, M, s)) return rc;
  if (int rc = conv_weight_grad(n, 1, n->act[0], n->gb, M, s)) return rc;
  if (int rc = conv_backward_data(n, 1, n->gb, n->ga, M, s)) return rc;
  if (int rc = conv_weight_grad(n, 0, n->x0, n->ga, M, s)) return rc;
  if (loss) {
    sum_kernel<<<1, 32, 0, s>>>(n->loss_part, nlp, loss);
    NET_CUDA(cudaGetLastError());
  }
  return GPG_OK;
}

void free_net(gpg_net *n) {
  cudaFree(n->params);
  cudaFree(n->grad);
  cudaFree(n->adam_m);
  cudaFree(n->adam_v);
  for (int l = 0; l < kLayers; ++l) {
    cudaFree(n->wf[l]);
    cudaFree(n->wb[l]);
  }
  cudaFree(n->x0);
  for (auto *p : n->act) cudaFree(p);
  cudaFree(n->g4);
  cudaFree(n->ga);
  cudaFree(n->gb);
  cudaFree(n->y4);
  cudaFree(n->cube);
  cudaFree(n->scale);
  cudaFree(n->wpart);
  cudaFree(n->bpart);
  cudaFree(n->loss_part);
  cudaFree(n->err);
}

}  // namespace

extern "C" const char *gpg_net_last_error(void) { return g_net_error.c_str(); }

extern "C" int gpg_net_param_count(int64_t *count) {
  if (!count) return nfail(GPG_ERR_INVALID, "count is NULL");
  *count = kParams;
  return GPG_OK;
}

extern "C" int gpg_net_create(gpg_net **out, int max_batch, uint64_t seed, int device_id) {
  if (!out) return nfail(GPG_ERR_INVALID, "net is NULL");
  *out = nullptr;
  if (max_batch < 1 || max_batch > (1 << 20)) return nfail(GPG_ERR_INVALID, "max_batch %d", max_batch);
  NET_CUDA(cudaSetDevice(device_id));
  cudaDeviceProp prop;
  NET_CUDA(cudaGetDeviceProperties(&prop, device_id));
  if (prop.major != 10) return nfail(GPG_ERR_UNSUPPORTED, "tensor-core kernels need sm_100 (found sm_%d%d)",
                                     prop.major, prop.minor);
  auto *n = new gpg_net;
  n->device = device_id;
  n->max_batch = max_batch;
  const int64_t M = int64_t(max_batch) * kCells;
  const int wrows = 7 * 128;  // most k rows a layer's weight gradient has
  const int max_grid = sm_count() * 4;
  cudaError_t e = cudaSuccess;
  auto al = [&](void **p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, b);
  };
  al((void **)&n->params, kParams * 4);
  al((void **)&n->grad, kParams * 4);
  al((void **)&n->adam_m, kParams * 4);
  al((void **)&n->adam_v, kParams * 4);
  for (int l = 0; l < kLayers; ++l) {
    al((void **)&n->wf[l], size_t(kch_fwd(l)) * kCout[l] * 16);
    if (l > 0) al((void **)&n->wb[l], size_t(kch_bwd(l)) * kCin[l] * 16);
  }
  al((void **)&n->x0, size_t(M) * 8 * 2);
  for (auto &p : n->act) al((void **)&p, size_t(M) * 32 * 2);
  al((void **)&n->g4, size_t(M) * 16 * 2);
  al((void **)&n->ga, size_t(M) * 32 * 2);
  al((void **)&n->gb, size_t(M) * 32 * 2);
  al((void **)&n->y4, size_t(M) * 16 * 4);
  al((void **)&n->cube, size_t(max_batch) * kCells * 4);
  al((void **)&n->scale, size_t(max_batch) * 4);
  al((void **)&n->wpart, size_t(max_grid) * wrows * 32 * 4);
  al((void **)&n->bpart, size_t(kPartials) * 32 * 4);
  al((void **)&n->loss_part, kPartials * 8);
  al((void **)&n->err, 4);
  if (e != cudaSuccess) {
    free_net(n);
    delete n;
    return nfail(e == cudaErrorMemoryAllocation ? GPG_ERR_OOM : GPG_ERR_CUDA, "allocation: %s",
                 cudaGetErrorString(e));
  }
  // He-normal initialisation of the real weights (fixed seed); padded input
  // channels of layer 1 and output channels 1..15 of layer 4 stay zero
  std::vector<float> h(kParams, 0.f);
  uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  for (int l = 0; l < kLayers; ++l) {
    const int cin_real = l == 0 ? kRealCin0 : kCin[l];
    const int cout_real = l == 3 ? kRealCout3 : kCout[l];
    const double sd = std::sqrt(2.0 / (27.0 * cin_real)) * (l == 3 ? 0.1 : 1.0);
    for (int t = 0; t < 27; ++t)
      for (int c = 0; c < cin_real; ++c)
        for (int o = 0; o < cout_real; ++o) {
          const double z = std::sqrt(-2.0 * std::log(uni())) * std::cos(6.283185307179586 * uni());
          h[param_offset_w(l) + (int64_t(t) * kCin[l] + c) * kCout[l] + o] = float(sd * z);
        }
  }
  e = cudaMemcpy(n->params, h.data(), kParams * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    free_net(n);
    delete n;
    return nfail(GPG_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
  }
  if (int rc = repack(n, 0)) {
    free_net(n);
    delete n;
    return rc;
  }
  *out = n;
  return GPG_OK;
}

extern "C" int gpg_net_destroy(gpg_net *n) {
  if (!n) return GPG_OK;
  cudaSetDevice(n->device);
  cudaDeviceSynchronize();
  free_net(n);
  delete n;
  return GPG_OK;
}

extern "C" int gpg_net_get_params(gpg_net *n, float *host) {
  if (!n || !host) return nfail(GPG_ERR_INVALID, "NULL argument");
  NET_CUDA(cudaSetDevice(n->device));
  NET_CUDA(cudaMemcpy(host, n->params, kParams * 4, cudaMemcpyDeviceToHost));
  return GPG_OK;
}

extern "C" int gpg_net_set_params(gpg_net *n, const float *host) {
  if (!n || !host) return nfail(GPG_ERR_INVALID, "NULL argument");
  NET_CUDA(cudaSetDevice(n->device));
  NET_CUDA(cudaMemcpy(n->params, host, kParams * 4, cudaMemcpyHostToDevice));
  NET_CUDA(cudaMemset(n->adam_m, 0, kParams * 4));
  NET_CUDA(cudaMemset(n->adam_v, 0, kParams * 4));
  n->step = 0;
  return repack(n, 0);
}

extern "C" int gpg_net_check(gpg_net *n) {
  if (!n) return nfail(GPG_ERR_INVALID, "net is NULL");
  NET_CUDA(cudaSetDevice(n->device));
  int flag = 0;
  NET_CUDA(cudaMemcpy(&flag, n->err, 4, cudaMemcpyDeviceToHost));
  if (flag) {
    NET_CUDA(cudaMemset(n->err, 0, 4));  // reported once
    return nfail(GPG_ERR_CUDA, "a tensor-core wait timed out");
  }
  return GPG_OK;
}

extern "C" int gpg_net_set_wait_probe(gpg_net *n, int polls) {
  if (!n) return nfail(GPG_ERR_INVALID, "net is NULL");
  if (polls < 0) return nfail(GPG_ERR_INVALID, "polls %d", polls);
  n->probe_polls = polls;
  return GPG_OK;
}

extern "C" int gpg_net_predict(gpg_net *n, int npatch, const float *d_rho, const float *d_pot_in, float *d_guess,
                               double cnst, void *stream) {
  if (!n) return nfail(GPG_ERR_INVALID, "net is NULL");
  if (npatch < 0) return nfail(GPG_ERR_INVALID, "npatch %d", npatch);
  if (npatch && (!d_rho || !d_pot_in || !d_guess)) return nfail(GPG_ERR_INVALID, "NULL array");
  if (!npatch) return GPG_OK;
  NET_CUDA(cudaSetDevice(n->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  static DevOnce once;
  using gpg::net::InferSmem;
  if (int rc = set_attr_once(gpg::net::net_infer_kernel, InferSmem::bytes, once)) return rc;
  gpg::net::InferArgs a{};
  a.rho = d_rho;
  a.pot_in = d_pot_in;
  a.guess = d_guess;
  for (int l = 0; l < kLayers; ++l) {
    a.w[l] = n->wf[l];
    a.bias[l] = n->params + param_offset_b(l);
  }
  a.cnst = float(cnst);
  a.npatch = npatch;
  a.probe_polls = n->probe_polls;
  a.err = n->err;
  const int grid = std::min(npatch, sm_count());  // persistent: one CTA per SM (shared memory bound)
  gpg::net::net_infer_kernel<<<grid, gpg::net::kInferThreads, InferSmem::bytes, s>>>(a);
  NET_CUDA(cudaGetLastError());
  return GPG_OK;
}

extern "C" int gpg_net_predict_layers(gpg_net *n, int npatch, const float *d_rho, const float *d_pot_in,
                                      float *d_guess, double cnst, void *stream) {
  if (!n) return nfail(GPG_ERR_INVALID, "net is NULL");
  if (npatch < 0) return nfail(GPG_ERR_INVALID, "npatch %d", npatch);
  if (npatch && (!d_rho || !d_pot_in || !d_guess)) return nfail(GPG_ERR_INVALID, "NULL array");
  NET_CUDA(cudaSetDevice(n->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  for (int64_t p0 = 0; p0 < npatch; p0 += n->max_batch) {
    const int64_t b = std::min<int64_t>(n->max_batch, npatch - p0);
    if (int rc = forward_all(n, b, d_rho + p0 * 512, d_pot_in + p0 * 512, float(cnst), s)) return rc;
    guess_kernel<<<296, 256, 0, s>>>(n->y4, n->scale, d_guess + p0 * 512, b);
    NET_CUDA(cudaGetLastError());
  }
  return GPG_OK;
}

extern "C" int gpg_net_gradients(gpg_net *n, int npatch, const float *d_rho, const float *d_pot_in,
                                 const float *d_target, double cnst, float *d_grad, float *d_loss, void *stream) {
  if (!n) return nfail(GPG_ERR_INVALID, "net is NULL");
  if (npatch < 1 || npatch > n->max_batch) return nfail(GPG_ERR_INVALID, "npatch %d (1..%d)", npatch, n->max_batch);
  if (!d_rho || !d_pot_in || !d_target) return nfail(GPG_ERR_INVALID, "NULL array");
  NET_CUDA(cudaSetDevice(n->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (int rc = gradients(n, npatch, d_rho, d_pot_in, d_target, float(cnst), d_loss, s)) return rc;
  if (d_grad) NET_CUDA(cudaMemcpyAsync(d_grad, n->grad, kParams * 4, cudaMemcpyDeviceToDevice, s));
  return GPG_OK;
}

namespace {
// one Adam step (beta 0.9 / 0.999, eps 1e-8) with gradient `grad`, then the
// BF16 operands are repacked from the updated FP32 masters
int adam_step(gpg_net *n, const float *grad, float lr, cudaStream_t s) {
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, float(n->step)), c2 = 1.f - std::pow(b2, float(n->step));
  gpg::adam_kernel<<<128, 256, 0, s>>>(n->params, n->adam_m, n->adam_v, grad, kParams, lr, b1, b2, 1e-8f, c1, c2);
  NET_CUDA(cudaGetLastError());
  return repack(n, s);
}
}  // namespace

extern "C" int gpg_net_train_step(gpg_net *n, int npatch, const float *d_rho, const float *d_pot_in,
                                  const float *d_target, double cnst, float lr, float *d_loss, void *stream) {
  if (int rc = gpg_net_gradients(n, npatch, d_rho, d_pot_in, d_target, cnst, nullptr, d_loss, stream)) return rc;
  return adam_step(n, n->grad, lr, static_cast<cudaStream_t>(stream));
}

extern "C" int gpg_net_apply_gradient(gpg_net *n, const float *d_grad, float lr, void *stream) {
  if (!n || !d_grad) return nfail(GPG_ERR_INVALID, "NULL argument");
  NET_CUDA(cudaSetDevice(n->device));
  return adam_step(n, d_grad, lr, static_cast<cudaStream_t>(stream));
}
