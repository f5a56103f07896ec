// linear.cu -- the learned linear correction of the interpolated SOR start
// (gpg_lin_* in include/gpg.h): the fused solve of lin_sor.cuh, the training
// features, and training by gradient descent (FP32 kernels below, Adam).
//
// Model (block space, see lin_sor.cuh): per patch the folded residual
// u[8][64] and, for training, the folded target t[8][64] = H(phi* - phi_i)/8,
// phi* the converged solution; the prediction of block b is
// v_b = W[class(b)] u_b with W[4][64][64] (row = output orbit, column = input
// orbit, both in the class representative's axes).  The features come scaled
// by the power of two that brings the patch's max|phi_i| into [2^16, 2^17): a
// linear model is indifferent to the scale, and the training loss, the mean
// over patches, blocks and rows of e^2 with e = v - t, then measures each
// patch's start error relative to its potential -- the quantity the solve is
// judged by.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gpg.h"
#include "args.cuh"
#include "lin_sor.cuh"
#include "optim.cuh"

namespace {

using gpg::lin::kK;
using gpg::lin::kParams;

thread_local std::string g_lin_error;

int lfail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_lin_error = buf;
  return status;
}

#define LIN_CUDA(call)                                                                                 \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess)                                                                             \
      return lfail(e_ == cudaErrorMemoryAllocation ? GPG_ERR_OOM : GPG_ERR_CUDA, "%s: %s (%s:%d)", #call, \
                   cudaGetErrorString(e_), __FILE__, __LINE__);                                        \
  } while (0)

// class of block b: number of odd axes
__host__ __device__ constexpr int class_of(int b) { return (b & 1) + ((b >> 1) & 1) + ((b >> 2) & 1); }

// W[4][64][64] (FP32) -> the two stacked A tiles [kc][row 0..127][8] (BF16):
// tile 0 = (class 0 ; class 3), tile 1 = (class 1 ; class 2)
__global__ void lin_pack_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ tiles) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * 128 * kK; i += gridDim.x * blockDim.x) {
    const int t = i / (128 * kK), rem = i - t * 128 * kK;
    const int kc = rem / (128 * 8), row = (rem / 8) % 128, e = rem % 8;
    const int cls = t == 0 ? (row < 64 ? 0 : 3) : (row < 64 ? 1 : 2);
    tiles[i] = __float2bfloat16_rn(w[(cls * kK + (row & 63)) * kK + kc * 8 + e]);
  }
}

// per patch (one CTA of 512 threads = 8 blocks x 64 rows): the errors
// e = W u - t and the patch's sum of e^2 (fixed-order tree)
__global__ void __launch_bounds__(512) lin_err_kernel(const float *__restrict__ u, const float *__restrict__ t,
                                                      const float *__restrict__ w, float *__restrict__ e,
                                                      float *__restrict__ loss_part) {
  __shared__ float su[512];
  __shared__ float red[512];
  const int p = blockIdx.x, tid = threadIdx.x, b = tid >> 6, r = tid & 63;
  su[tid] = u[int64_t(p) * 512 + tid];
  __syncthreads();
  const float *wr = w + (class_of(b) * kK + r) * kK;
  const float *ub = su + b * kK;
  float acc = 0.f;
#pragma unroll 8
  for (int k = 0; k < kK; ++k) acc = fmaf(__ldg(wr + k), ub[k], acc);
  const float err = acc - t[int64_t(p) * 512 + tid];
  e[int64_t(p) * 512 + tid] = err;
  red[tid] = err * err;
  __syncthreads();
  for (int h = 256; h > 0; h >>= 1) {
    if (tid < h) red[tid] += red[tid + h];
    __syncthreads();
  }
  if (tid == 0) loss_part[p] = red[0];
}

// grad[c][r][k] = 2 / (npatch 512) sum_p sum_{b in c} e[p][b][r] u[p][b][k]
// (CTA = class c, 4 rows; thread = (row, k); patches and blocks in order)
__global__ void __launch_bounds__(256) lin_grad_kernel(const float *__restrict__ us, const float *__restrict__ e,
                                                       int npatch, float *__restrict__ grad) {
  const int c = blockIdx.x / 16, r = (blockIdx.x % 16) * 4 + (threadIdx.x >> 6), k = threadIdx.x & 63;
  float acc = 0.f;
  for (int p = 0; p < npatch; ++p)
#pragma unroll
    for (int b = 0; b < 8; ++b)
      if (class_of(b) == c) acc = fmaf(e[(int64_t(p) * 8 + b) * kK + r], us[(int64_t(p) * 8 + b) * kK + k], acc);
  grad[(c * kK + r) * kK + k] = acc * (2.f / (float(npatch) * 512.f));
}

// loss = sum_p loss_part[p] / (npatch 512), fixed order (one CTA)
__global__ void __launch_bounds__(256) lin_loss_kernel(const float *__restrict__ part, int npatch,
                                                       float *__restrict__ loss) {
  __shared__ double red[256];
  double s = 0.0;
  for (int p = threadIdx.x; p < npatch; p += 256) s += part[p];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = float(red[0] / (double(npatch) * 512.0));
}

}  // namespace

struct gpg_lin {
  int device = 0;
  int max_batch = 0;
  int step = 0;
  int probe_polls = 0;
  float *params = nullptr, *grad = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  float *e = nullptr, *loss_part = nullptr, *loss = nullptr;
  __nv_bfloat16 *tiles = nullptr;
  int *err = nullptr;
  int variant = 0;                   // launch shape of the fused solve
  int grid[2] = {0, 0};              // persistent CTAs per shape (one per SM)
};

namespace {

int repack(gpg_lin *l, cudaStream_t s) {
  lin_pack_kernel<<<32, 256, 0, s>>>(l->params, l->tiles);
  LIN_CUDA(cudaGetLastError());
  return GPG_OK;
}

// Launch shapes of the fused solve (identical results): 0 = two groups of 8
// teams with staged inputs, 1 = three groups of 8 teams reading their inputs
// from global memory.
constexpr int kLinVariants = 2;

template <bool FEATURES, int HALVES, bool STAGE>
int prepare(int *grid) {
  auto fn = gpg::lin::lin_sor_kernel<FEATURES, HALVES, STAGE>;
  using L = gpg::lin::Layout<HALVES, STAGE>;
  LIN_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::bytes)));
  LIN_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                int(cudaSharedmemCarveoutMaxShared)));
  if (grid) {
    int dev = 0, sms = 0;
    LIN_CUDA(cudaGetDevice(&dev));
    LIN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *grid = sms;  // one CTA per SM: its shared memory and TMEM take the whole SM
  }
  return GPG_OK;
}

// persistent CTAs for npatch patches: HALVES batches of 8 per CTA at a time
int lin_grid(int halves, int grid_max, int npatch) {
  const int64_t nbatch = (int64_t(npatch) + gpg::lin::kHalfWarps - 1) / gpg::lin::kHalfWarps;
  const int64_t need = (nbatch + halves - 1) / halves;
  return int(need < grid_max ? need : grid_max);
}

int check_solve_params(const gpg_params *p) {
  if (int rc = gpg_validate_params(p)) return lfail(rc, "%s", gpg_last_error());
  if (p->real_size != 4 || p->ghost != 1 || p->scheme != GPG_SOR || !p->poisson)
    return lfail(GPG_ERR_UNSUPPORTED, "the learned start covers ghost-size-1 FP32 SOR (real_size %d, ghost %d, scheme %d)",
                 p->real_size, p->ghost, p->scheme);
  return GPG_OK;
}

}  // namespace

extern "C" const char *gpg_lin_last_error(void) { return g_lin_error.c_str(); }

extern "C" int gpg_lin_param_count(int64_t *count) {
  if (!count) return lfail(GPG_ERR_INVALID, "count is NULL");
  *count = kParams;
  return GPG_OK;
}

extern "C" int gpg_lin_create(gpg_lin **out, int max_batch, int device_id) {
  if (!out) return lfail(GPG_ERR_INVALID, "lin is NULL");
  *out = nullptr;
  if (max_batch < 1 || max_batch > (1 << 22)) return lfail(GPG_ERR_INVALID, "max_batch %d", max_batch);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device_id < 0 || device_id >= count)
    return lfail(GPG_ERR_NO_DEVICE, "device %d of %d", device_id, count);
  LIN_CUDA(cudaSetDevice(device_id));
  cudaDeviceProp prop;
  LIN_CUDA(cudaGetDeviceProperties(&prop, device_id));
  if (prop.major != 10)
    return lfail(GPG_ERR_UNSUPPORTED, "tensor-core kernels need sm_100 (found sm_%d%d)", prop.major, prop.minor);
  gpg_lin *l = new gpg_lin;
  l->device = device_id;
  l->max_batch = max_batch;
  cudaError_t e = cudaSuccess;
  auto al = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  al((void **)&l->params, kParams * 4);
  al((void **)&l->grad, kParams * 4);
  al((void **)&l->adam_m, kParams * 4);
  al((void **)&l->adam_v, kParams * 4);
  al((void **)&l->tiles, 2 * gpg::lin::kTileBytes);
  al((void **)&l->e, size_t(max_batch) * 512 * 4);
  al((void **)&l->loss_part, size_t(max_batch) * 4);
  al((void **)&l->loss, 4);
  al((void **)&l->err, 4);
  if (e == cudaSuccess) e = cudaMemset(l->params, 0, kParams * 4);
  if (e == cudaSuccess) e = cudaMemset(l->adam_m, 0, kParams * 4);
  if (e == cudaSuccess) e = cudaMemset(l->adam_v, 0, kParams * 4);
  if (e == cudaSuccess) e = cudaMemset(l->err, 0, 4);
  if (e != cudaSuccess) {
    gpg_lin_destroy(l);
    return lfail(e == cudaErrorMemoryAllocation ? GPG_ERR_OOM : GPG_ERR_CUDA, "allocation: %s", cudaGetErrorString(e));
  }
  // attributes here, so that a stream capture never sees first-use set-up
  int rc = prepare<false, 2, true>(&l->grid[0]);
  if (!rc) rc = prepare<false, 3, false>(&l->grid[1]);
  if (!rc) rc = prepare<true, 2, false>(nullptr);
  if (rc) {
    gpg_lin_destroy(l);
    return rc;
  }
  if (int rc = repack(l, 0)) {
    gpg_lin_destroy(l);
    return rc;
  }
  LIN_CUDA(cudaDeviceSynchronize());
  *out = l;
  return GPG_OK;
}

extern "C" int gpg_lin_destroy(gpg_lin *l) {
  if (!l) return GPG_OK;
  cudaSetDevice(l->device);
  for (void *p : {(void *)l->params, (void *)l->grad, (void *)l->adam_m, (void *)l->adam_v, (void *)l->tiles,
                  (void *)l->e, (void *)l->loss_part, (void *)l->loss, (void *)l->err})
    cudaFree(p);
  delete l;
  return GPG_OK;
}

extern "C" int gpg_lin_get_params(gpg_lin *l, float *host) {
  if (!l || !host) return lfail(GPG_ERR_INVALID, "NULL argument");
  LIN_CUDA(cudaSetDevice(l->device));
  LIN_CUDA(cudaMemcpy(host, l->params, kParams * 4, cudaMemcpyDeviceToHost));
  return GPG_OK;
}

extern "C" int gpg_lin_set_params(gpg_lin *l, const float *host) {
  if (!l || !host) return lfail(GPG_ERR_INVALID, "NULL argument");
  LIN_CUDA(cudaSetDevice(l->device));
  LIN_CUDA(cudaMemcpy(l->params, host, kParams * 4, cudaMemcpyHostToDevice));
  LIN_CUDA(cudaMemset(l->adam_m, 0, kParams * 4));
  LIN_CUDA(cudaMemset(l->adam_v, 0, kParams * 4));
  l->step = 0;
  if (int rc = repack(l, 0)) return rc;
  LIN_CUDA(cudaDeviceSynchronize());
  return GPG_OK;
}

extern "C" int gpg_lin_solve_device(gpg_lin *l, const gpg_params *p, int npatch, const float *d_rho,
                                    const float *d_pot_in, float *d_pot_out, float *d_flu, int32_t *d_iters,
                                    double *d_resid, void *stream) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  if (int rc = check_solve_params(p)) return rc;
  if (npatch < 0) return lfail(GPG_ERR_INVALID, "npatch %d", npatch);
  if (npatch == 0) return GPG_OK;
  if (!d_rho || !d_pot_in || !d_pot_out || (p->gra_acc && !d_flu)) return lfail(GPG_ERR_INVALID, "NULL array");
  LIN_CUDA(cudaSetDevice(l->device));
  // the inputs are staged with bulk copies of whole patches
  if ((reinterpret_cast<uintptr_t>(d_rho) | reinterpret_cast<uintptr_t>(d_pot_in)) & 15)
    return lfail(GPG_ERR_INVALID, "d_rho and d_pot_in must be 16-byte aligned");
  gpg_params q = *p;
  q.init_mode = GPG_INIT_INTERP;  // the correction is added to the interpolated start
  gpg::lin::LinArgs a{};
  a.s = gpg::make_args<float>(q, npatch, d_rho, d_pot_in, d_pot_out, d_flu, nullptr, d_iters, d_resid);
  a.wtiles = l->tiles;
  a.err = l->err;
  a.probe_polls = l->probe_polls;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (l->variant == 0) {
    using SH = gpg::lin::Shape<2, true>;
    gpg::lin::lin_sor_kernel<false, 2, true><<<lin_grid(2, l->grid[0], npatch), SH::kThreads,
                                               gpg::lin::Layout<2, true>::bytes, s>>>(a);
  } else {
    using SH = gpg::lin::Shape<3, false>;
    gpg::lin::lin_sor_kernel<false, 3, false><<<lin_grid(3, l->grid[1], npatch), SH::kThreads,
                                                gpg::lin::Layout<3, false>::bytes, s>>>(a);
  }
  LIN_CUDA(cudaGetLastError());
  return GPG_OK;
}

extern "C" int gpg_lin_features(gpg_lin *l, const gpg_params *p, int npatch, const float *d_rho,
                                const float *d_pot_in, const float *d_target, float *d_u, float *d_t,
                                void *stream) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  if (int rc = check_solve_params(p)) return rc;
  if (npatch < 0) return lfail(GPG_ERR_INVALID, "npatch %d", npatch);
  if (npatch == 0) return GPG_OK;
  if (!d_rho || !d_pot_in || !d_u || (d_target && !d_t)) return lfail(GPG_ERR_INVALID, "NULL array");
  LIN_CUDA(cudaSetDevice(l->device));
  gpg_params q = *p;
  q.init_mode = GPG_INIT_INTERP;
  q.gra_acc = 0;
  gpg::lin::LinArgs a{};
  a.s = gpg::make_args<float>(q, npatch, d_rho, d_pot_in, nullptr, nullptr, nullptr, nullptr, nullptr);
  a.u_out = d_u;
  a.t_out = d_t;
  a.target = d_target;
  a.err = l->err;
  gpg::lin::lin_sor_kernel<true, 2, false>
      <<<lin_grid(2, l->grid[0], npatch), gpg::lin::Shape<2, false>::kThreads, gpg::lin::Layout<2, false>::bytes,
         static_cast<cudaStream_t>(stream)>>>(a);
  LIN_CUDA(cudaGetLastError());
  return GPG_OK;
}

extern "C" int gpg_lin_gradients(gpg_lin *l, int npatch, const float *d_u, const float *d_t, float *d_grad,
                                 float *d_loss, void *stream) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  if (npatch < 1 || npatch > l->max_batch) return lfail(GPG_ERR_INVALID, "npatch %d (1..%d)", npatch, l->max_batch);
  if (!d_u || !d_t) return lfail(GPG_ERR_INVALID, "NULL array");
  LIN_CUDA(cudaSetDevice(l->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  lin_err_kernel<<<npatch, 512, 0, s>>>(d_u, d_t, l->params, l->e, l->loss_part);
  lin_grad_kernel<<<64, 256, 0, s>>>(d_u, l->e, npatch, d_grad ? d_grad : l->grad);
  lin_loss_kernel<<<1, 256, 0, s>>>(l->loss_part, npatch, d_loss ? d_loss : l->loss);
  LIN_CUDA(cudaGetLastError());
  return GPG_OK;
}

namespace {
int lin_adam(gpg_lin *l, const float *grad, float lr, cudaStream_t s) {
  l->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, float(l->step)), c2 = 1.f - std::pow(b2, float(l->step));
  gpg::adam_kernel<<<64, 256, 0, s>>>(l->params, l->adam_m, l->adam_v, grad, kParams, lr, b1, b2, 1e-8f, c1, c2);
  LIN_CUDA(cudaGetLastError());
  return repack(l, s);
}
}  // namespace

extern "C" int gpg_lin_train_step(gpg_lin *l, int npatch, const float *d_u, const float *d_t, float lr,
                                  float *d_loss, void *stream) {
  if (int rc = gpg_lin_gradients(l, npatch, d_u, d_t, nullptr, d_loss, stream)) return rc;
  return lin_adam(l, l->grad, lr, static_cast<cudaStream_t>(stream));
}

extern "C" int gpg_lin_apply_gradient(gpg_lin *l, const float *d_grad, float lr, void *stream) {
  if (!l || !d_grad) return lfail(GPG_ERR_INVALID, "NULL argument");
  LIN_CUDA(cudaSetDevice(l->device));
  return lin_adam(l, d_grad, lr, static_cast<cudaStream_t>(stream));
}

extern "C" int gpg_lin_check(gpg_lin *l) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  LIN_CUDA(cudaSetDevice(l->device));
  int flag = 0;
  LIN_CUDA(cudaMemcpy(&flag, l->err, 4, cudaMemcpyDeviceToHost));
  if (flag) {
    LIN_CUDA(cudaMemset(l->err, 0, 4));
    return lfail(GPG_ERR_CUDA, "a tensor-core wait timed out");
  }
  return GPG_OK;
}

extern "C" int gpg_lin_variant_count(void) { return kLinVariants; }

extern "C" int gpg_lin_set_variant(gpg_lin *l, int variant) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  if (variant < 0 || variant >= kLinVariants) return lfail(GPG_ERR_INVALID, "variant %d", variant);
  l->variant = variant;
  return GPG_OK;
}

extern "C" int gpg_lin_set_wait_probe(gpg_lin *l, int polls) {
  if (!l) return lfail(GPG_ERR_INVALID, "lin is NULL");
  if (polls < 0) return lfail(GPG_ERR_INVALID, "polls %d", polls);
  l->probe_polls = polls;
  return GPG_OK;
}
