/*
 * gpg.h -- C-ABI of the B200 per-patch Poisson-gravity library (libgpg.so).
 *
 * The library replaces the reference testbed's GPU_API/ and GPU_Solver/
 * (gamer-project/gpu_testbed_poisson-gravity).  Every entry point takes plain
 * pointers and sizes, returns an int status (GPG_OK == 0) and never exits the
 * process; gpg_last_error() returns the message of the last failure on the
 * calling thread.
 *
 * Array layouts are the reference's (Header/Prototype.h:6-35), C order, x fastest:
 *   rho     [P][RHO_NXT][RHO_NXT][RHO_NXT]       RHO_NXT = 8 + 2*(ghost-1)
 *   pot_in  [P][POT_NXT][POT_NXT][POT_NXT]       POT_NXT = 4 + 2*((ghost+3)/2)
 *   pot_out [P][GRA_NXT][GRA_NXT][GRA_NXT]       GRA_NXT = 8 + 2*gra_ghost
 *   flu     [P][5][8][8][8]                      density, px, py, pz, energy
 * with P = 8 * NPatchGroup in the reference-shaped calls.  Element type is
 * float when params.real_size == 4 and double when it is 8 (the reference's
 * `real`, Header/Macro.h:35-39).
 */
#ifndef GPG_H
#define GPG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GPG_API __attribute__((visibility("default")))
#else
#define GPG_API
#endif

#define GPG_NULL_INT 2147483647 /* NULL_INT, Header/Macro.h:73-75 */
#define GPG_ABI_VERSION 1

typedef enum gpg_status {
  GPG_OK = 0,
  GPG_ERR_INVALID = 1,     /* bad argument (sizes, schemes, null pointers) */
  GPG_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  GPG_ERR_NO_DEVICE = 3,   /* no CUDA device / device id out of range */
  GPG_ERR_OOM = 4,         /* device or pinned host allocation failed */
  GPG_ERR_UNSUPPORTED = 5, /* valid request this build does not implement */
  GPG_ERR_STATE = 6        /* call out of order (e.g. solve before allocate) */
} gpg_status;

/* Poisson schemes, Header/Macro.h:11-14. */
enum { GPG_SOR = 1, GPG_MG = 2 };
/* Interpolation schemes, Header/Typedef.h:7-8 (only CQUAD and QUAD exist). */
enum { GPG_INT_CQUAD = 4, GPG_INT_QUAD = 5 };
/* SOR initial guess for the patch interior.
 *   INTERP: interpolated coarse potential (the reference, CPU_PoissonSolver_SOR.cpp:80-209)
 *   ZERO:   zero interior, interpolated ghost shell
 *   GUESS:  interior taken from a caller array [P][RHO_NXT]^3 */
enum { GPG_INIT_INTERP = 0, GPG_INIT_ZERO = 1, GPG_INIT_GUESS = 2 };
/* SOR stopping rule.
 *   REFERENCE:     stop after the first sweep whose L1 residual grows, once
 *                  Iter+1 >= Min_Iter; cap Max_Iter (CPU_PoissonSolver_SOR.cpp:273-283)
 *   TOLERANCE:     stop once Iter+1 >= Min_Iter and the sweep's L1 residual
 *                  <= sor_tolerance * sum|Poi_Coeff*dh^2*rho|; cap Max_Iter
 *   ABS_TOLERANCE: the same with the L1 residual <= sor_tolerance
 *   POT_TOLERANCE: the same with the L1 residual <= sor_tolerance * sum|phi_i|
 *                  over the updated cells, phi_i the interpolated coarse
 *                  potential there (taken before the initial guess replaces
 *                  it, so every start mode gets the same bound).  The SOR
 *                  residual stagnates at a multiple of the potential's
 *                  rounding error, so this bound is reachable for every patch
 *                  at any density contrast; GPG_STOP_TOLERANCE's source-scaled
 *                  bound is not where the potential dwarfs Const*rho. */
enum { GPG_STOP_REFERENCE = 0, GPG_STOP_TOLERANCE = 1, GPG_STOP_ABS_TOLERANCE = 2,
       GPG_STOP_POT_TOLERANCE = 3 };

/* Runtime form of the reference's compile-time shape (Makefile:13-85) plus the
 * argument list of CUAPI_Asyn_PoissonGravitySolver (Header/Prototype.h:25-34).
 * Fields are converted to `real` exactly where the reference converts them. */
typedef struct gpg_params {
  int32_t real_size;       /* 4 or 8 */
  int32_t ghost;           /* POT_GHOST_SIZE, 1..5 */
  int32_t gra_ghost;       /* GRA_GHOST_SIZE, 0..2, <= ghost */
  int32_t scheme;          /* GPG_SOR | GPG_MG */
  int32_t int_scheme;      /* GPG_INT_CQUAD | GPG_INT_QUAD */
  int32_t p5_gradient;     /* 5-point gradient; needs gra_ghost == 2 */
  int32_t poisson;         /* run the Poisson solver */
  int32_t gra_acc;         /* run the gravity update */
  double dt;
  double dh;
  int32_t sor_min_iter;
  int32_t sor_max_iter;
  double sor_omega;
  int32_t mg_max_iter;
  int32_t mg_npre_smooth;
  int32_t mg_npost_smooth;
  int32_t init_mode;       /* GPG_INIT_* (SOR only) */
  double mg_tolerated_error;
  double poi_coeff;        /* 4*pi*G*a */
  int32_t stop_mode;       /* GPG_STOP_* (SOR only) */
  int32_t reserved0;
  double sor_tolerance;    /* L1 tolerance for GPG_STOP_TOLERANCE (relative) / _ABS_TOLERANCE */
} gpg_params;

/* Fill `p` with the reference defaults for (real_size, ghost, scheme):
 * omega / Min_Iter / Max_Iter of Main.cpp:1142-1157, MG settings of
 * Main.cpp:1173-1223, dt = 1e-2, dh = 1, Poi_Coeff = 4*pi*1e-5, CQUAD,
 * gra_ghost = 1, Poisson and GraAcc on. */
GPG_API int gpg_default_params(gpg_params *p, int real_size, int ghost, int scheme);

/* The calibrated fixed residual for GPG_STOP_POT_TOLERANCE at (real_size,
 * ghost): 2 x the 90th percentile of L1 residual / sum|interpolated phi| at
 * the reference's own stopping point (CPU_PoissonSolver_SOR.cpp:275-281) of
 * zero-start SOR on seeded power-law inputs -- the round-off floor the
 * reference rule stops at, reachable by every patch.  FP32: 9.8e-7 (ghost 1)
 * ... 1.4e-6 (ghost 5); FP64: 1.8e-15 ... 2.5e-15.  No reference counterpart. */
GPG_API int gpg_pot_tolerance(int real_size, int ghost, double *tol);

/* Check a parameter block (same checks as CUAPI_Asyn_PoissonGravitySolver.cu:116-140). */
GPG_API int gpg_validate_params(const gpg_params *p);

/* Element counts per patch of each array for the shape in `p`. */
GPG_API int gpg_patch_sizes(const gpg_params *p, int64_t *rho, int64_t *pot_in, int64_t *pot_out,
                    int64_t *flu);

GPG_API const char *gpg_last_error(void);
GPG_API int gpg_abi_version(void);

/* ---------------------------------------------------------------------------
 * Stream-ordered device API.  All pointers are device pointers the caller owns;
 * the call only enqueues work on `stream` (a cudaStream_t, NULL = legacy default).
 *   d_guess  : [P][RHO_NXT]^3, read when init_mode == GPG_INIT_GUESS, else may be NULL
 *   d_iters  : [P] int32, per-patch SOR sweeps / MG V-cycles (may be NULL)
 *   d_resid  : [P] double, final SOR L1 residual / MG error estimate (may be NULL)
 * Replaces the kernel launches of CUAPI_Asyn_PoissonGravitySolver.cu:204-249
 * (CUPOT_PoissonSolver_SOR_10to14cube / _16to18cube / _MG and CUPOT_GravitySolver).
 * With poisson && gra_acc the gravity update is fused into the Poisson kernel
 * (one launch); with only gra_acc, d_pot_out is the input potential.
 * ------------------------------------------------------------------------- */
GPG_API int gpg_poisson_gravity_device(const gpg_params *p, int npatch, const void *d_rho,
                               const void *d_pot_in, void *d_pot_out, void *d_flu,
                               const void *d_guess, int32_t *d_iters, double *d_resid,
                               void *stream);

/* ---------------------------------------------------------------------------
 * Reference-shaped host API (Header/Prototype.h:15-35).  One context holds the
 * device buffers, pinned host buffers and streams that the reference keeps in
 * module globals (GPU_API/CUAPI_Asyn_PoissonGravitySolver.cu:32-39).
 * ------------------------------------------------------------------------- */
typedef struct gpg_context gpg_context;

/* CUAPI_Set_Diagnose_Device (GPU_API/CUAPI_Set_Diagnose_Device.cu:45-292):
 * select the device and replace GPG_NULL_INT in *npgroup / *nstream with
 * defaults (streams: 4; patch groups: 32 * SM count). */
GPG_API int gpg_set_diagnose_device(int *npgroup, int *nstream, int device_id);

GPG_API int gpg_context_create(gpg_context **ctx, int device_id, int nstream);
GPG_API int gpg_context_destroy(gpg_context *ctx);

/* CUAPI_MemAllocate_PoissonGravity (GPU_API/CUAPI_MemAllocate_PoissonGravity.cu:27-80):
 * device buffers for npatch_group*8 patches of the shape in `shape`, plus pinned
 * host buffers returned through the four out-pointers. */
GPG_API int gpg_mem_allocate(gpg_context *ctx, const gpg_params *shape, int npatch_group,
                     void **h_rho, void **h_pot_in, void **h_pot_out, void **h_flu);

/* CUAPI_MemFree_PoissonGravity (GPU_API/CUAPI_MemFree_PoissonGravity.cu:27-70). */
GPG_API int gpg_mem_free(gpg_context *ctx, void **h_rho, void **h_pot_in, void **h_pot_out,
                 void **h_flu);

/* CUAPI_Asyn_PoissonGravitySolver (GPU_API/CUAPI_Asyn_PoissonGravitySolver.cu:85-275):
 * per stream, H2D of rho / pot_in (and pot_out when !poisson) / flu, the solve,
 * D2H of pot_out / flu.  Returns before the GPU finishes; call gpg_synchronize()
 * before reading h_pot_out / h_flu.  h_flu is in/out. */
GPG_API int gpg_asyn_poisson_gravity_solver(gpg_context *ctx, const void *h_rho, void *h_pot_in,
                                    void *h_pot_out, void *h_flu, int npatch_group,
                                    const gpg_params *p, int nstream);

/* CUAPI_Synchronize (GPU_API/CUAPI_Synchronize.cu:10-13). */
GPG_API int gpg_synchronize(gpg_context *ctx);

/* Per-patch iteration counts / residuals of the last solve, read from the
 * device on request (the call waits for the context's streams).  No
 * reference counterpart: the reference only prints them
 * (CPU_PoissonSolver_SOR.cpp:288). */
GPG_API int gpg_last_iterations(gpg_context *ctx, int32_t *iters, double *resid, int npatch);

/* ---------------------------------------------------------------------------
 * Batched SOR over patches of mixed ghost sizes, one persistent launch.
 * No single reference counterpart: the reference compiles one ghost size per
 * build and launches one kernel per stream (CUAPI_Asyn_PoissonGravitySolver.cu:
 * 206-249).  A group is a set of patches of one ghost size in the reference
 * layout; `p` supplies everything else (p->ghost is ignored, p->scheme must be
 * GPG_SOR).  Each patch gives the same bits as gpg_poisson_gravity_device.
 * ------------------------------------------------------------------------- */
typedef struct gpg_batch_group {
  int32_t ghost;        /* POT_GHOST_SIZE of the group, 1..5 */
  int32_t npatch;
  const void *d_rho;    /* [npatch][RHO_NXT]^3 */
  const void *d_pot_in; /* [npatch][POT_NXT]^3 */
  void *d_pot_out;      /* [npatch][GRA_NXT]^3 */
  void *d_flu;          /* [npatch][5][8]^3 when p->gra_acc, else may be NULL */
  const void *d_guess;  /* [npatch][RHO_NXT]^3 when init_mode == GPG_INIT_GUESS */
  int32_t *d_iters;     /* [npatch] or NULL */
  double *d_resid;      /* [npatch] or NULL */
  double sor_omega;     /* omega of the group; <= 0 selects the reference default */
} gpg_batch_group;

#define GPG_BATCH_MAX_GROUPS 8

/* Stream-ordered.  d_counter: one uint32 of device memory the call resets and
 * uses as the work-queue counter (calls that overlap need separate counters). */
GPG_API int gpg_solve_batch_device(const gpg_params *p, int ngroup, const gpg_batch_group *groups,
                                   uint32_t *d_counter, void *stream);

/* Allocation-free variant of gpg_solve_batch_device.  No counterpart in the
 * reference.  Some callers cannot allocate device memory at the point where
 * they solve -- a code that gives all device memory to its own pool at start-
 * up, one whose allocator belongs to another runtime, or one that must keep a
 * fixed memory footprint between time steps -- so this entry point needs no
 * buffer beyond the caller's inputs and outputs and calls no cudaMalloc or
 * cudaFree: the work-queue counter lives in a static device array inside
 * libgpg (GPG_BATCH_NOALLOC_SCRATCH_WORDS words, 256-byte aligned, held on
 * every GPU that loads the library until the process exits).
 *  - The first call on a device looks up that array's device address
 *    (cudaGetSymbolAddress) and caches it; make that first call before any
 *    stream capture on the device.
 *  - The counter is reset on `stream` at the start of every call, but all
 *    calls on a device share it: calls whose work overlaps on the GPU (other
 *    streams, other host threads) race and must be serialised by the caller.
 *  - At most GPG_BATCH_NOALLOC_MAX_PATCHES patches per call; larger batches
 *    are rejected with GPG_ERR_INVALID. */
#define GPG_BATCH_NOALLOC_SCRATCH_WORDS 1
#define GPG_BATCH_NOALLOC_MAX_PATCHES (1LL << 30)
GPG_API int gpg_solve_batch_device_noalloc(const gpg_params *p, int ngroup, const gpg_batch_group *groups,
                                           void *stream);

/* The same batch captured once into a CUDA graph; gpg_batch_plan_launch
 * replays it on `stream`.  mode GPG_PLAN_PERSISTENT: counter reset + the
 * persistent work-queue kernel.  mode GPG_PLAN_CONCURRENT: one per-ghost-size
 * kernel per group as parallel branches of the graph, so the hardware block
 * scheduler interleaves their CTAs (same bits either way).  The plan owns its
 * counter; the group buffers must outlive the plan. */
enum { GPG_PLAN_PERSISTENT = 0, GPG_PLAN_CONCURRENT = 1 };
typedef struct gpg_batch_plan gpg_batch_plan;
GPG_API int gpg_batch_plan_create(gpg_batch_plan **plan, const gpg_params *p, int ngroup,
                                  const gpg_batch_group *groups, int device_id, int mode);
GPG_API int gpg_batch_plan_launch(gpg_batch_plan *plan, void *stream);
GPG_API int gpg_batch_plan_destroy(gpg_batch_plan *plan);

/* ---------------------------------------------------------------------------
 * SOR kernel variants.  No reference counterpart (the reference fixes its
 * launch shape per ghost size with macros, Header/CUPOT.h:44-90).  A variant
 * is (patches per CTA, phased pass order, lanes per pair column, rows per
 * lane): variants 0-5 give each lane a whole column of one row, 6-9 split the
 * column between two lanes (twice the threads, half the registers each),
 * 10-11 give a lane two rows and half a column, 12-13 two rows and a whole
 * column (not built where that exceeds the register file: GPG_ERR_UNSUPPORTED);
 * 14-16 run the layouts of 10, 11 and 13 in a staged persistent kernel: each
 * team loops over patches and bulk-copies its next patch's coarse potential
 * and density into shared memory while it solves the current one (patches per
 * CTA reported as 0; inputs that are not 16-byte aligned run unstaged; a
 * staging wait that gives up after about a second leaves that patch's
 * iteration count at -1 and its residual NaN).
 * Variants 0-5 return identical bits; the others sum the residual in another
 * order, so a stop decision can differ only where two sweeps' totals tie.  The table starts from the library's defaults, then an optional
 * tuning file ($GPG_TUNE_FILE, else sor_tune.txt beside libgpg.so, lines
 * "f32|f64 <ghost> <variant>") written by autotune.py.  Unless a variant was
 * chosen (by gpg_set_sor_variant or the tuning file), launches of up to a
 * stated number of patches (256 or 2048, per precision and ghost size) run a
 * small-batch variant instead, one that gives each patch more threads;
 * gpg_get_sor_variant reports the large-batch choice.
 * ------------------------------------------------------------------------- */
GPG_API int gpg_sor_variant_count(void);
GPG_API int gpg_sor_variant_info(int variant, int *patches_per_cta, int *phased);
GPG_API int gpg_sor_variant_layout(int variant, int *lanes_per_column, int *rows_per_lane);
GPG_API int gpg_sor_variant_staged(int variant, int *staged);
/* The lane layout a variant uses at (real_size, ghost), for tools and tests
 * that check its indexing on the host: fields[GPG_SOR_LAYOUT_FIELDS] =
 * {lanes per column Z, rows per lane Y, heights per lane MH, lanes per row R,
 *  row pitch P, plane padding PADZ, block rounding U, lanes per block BLOCK,
 *  threads per team TEAM, plane pitch PP, built (1) or beyond the register
 *  file (0)}.  The shared cube of a team is 2 * (8 + 2 ghost) * PP elements;
 * cell (x, y, z) of colour c = (x + y + z + 1) & 1 sits at
 * (c * (8 + 2 ghost) + z) * PP + y * P + (x + 1) / 2. */
#define GPG_SOR_LAYOUT_FIELDS 11
GPG_API int gpg_sor_layout(int real_size, int ghost, int variant, int *fields);
/* variant -1 returns (real_size, ghost) to the library's built-in choice */
GPG_API int gpg_set_sor_variant(int real_size, int ghost, int variant);
GPG_API int gpg_get_sor_variant(int real_size, int ghost, int *variant);
/* the variant a solve of npatch patches (one launch) at (real_size, ghost)
 * runs now: the small-launch or large-launch choice, or the one set */
GPG_API int gpg_sor_variant_for_launch(int real_size, int ghost, int64_t npatch, int *variant);

/* ---------------------------------------------------------------------------
 * Learned initial guess for ghost-size-1 SOR (GPG_INIT_GUESS).  No reference
 * counterpart.  A 4-layer 3^3 convolution network (8 -> 32 -> 32 -> 32 -> 16
 * channels, ReLU; BF16 weights and activations, FP32 accumulation on the
 * tcgen05 tensor cores) maps a patch's density and interpolated boundary shell
 * to its 8^3 interior potential.  Inputs are FP32 ghost-1 arrays: rho
 * [P][8]^3 and pot_in [P][8]^3; `cnst` is Poi_Coeff*dh^2.  Parameters are one
 * FP32 vector: per layer W[27][cin][cout] then b[cout] (cin 8 for layer 1 of
 * which 3 used, cout 16 for layer 4 of which 1 used).
 * ------------------------------------------------------------------------- */
typedef struct gpg_net gpg_net;
/* every call on a net makes the net's device current, as the gpg_context
 * calls do; device arrays and streams passed to it belong to that device */
GPG_API int gpg_net_create(gpg_net **net, int max_batch, uint64_t seed, int device_id);
GPG_API int gpg_net_destroy(gpg_net *net);
GPG_API int gpg_net_param_count(int64_t *count);
GPG_API int gpg_net_get_params(gpg_net *net, float *host_params);
GPG_API int gpg_net_set_params(gpg_net *net, const float *host_params);
/* interior guess [P][8]^3 for GPG_INIT_GUESS (stream-ordered): one
 * persistent kernel runs all four layers with the activations in shared
 * memory; no size limit from max_batch */
GPG_API int gpg_net_predict(gpg_net *net, int npatch, const float *d_rho, const float *d_pot_in, float *d_guess,
                            double cnst, void *stream);
/* the same guess through the per-layer kernels of the training pass (chunks
 * of max_batch patches); identical results, kept for checking */
GPG_API int gpg_net_predict_layers(gpg_net *net, int npatch, const float *d_rho, const float *d_pot_in,
                                   float *d_guess, double cnst, void *stream);
/* loss = mean (net / s - target / s)^2 over interior cells and its gradient
 * wrt every parameter (d_grad, same layout as the parameters; may be NULL) */
GPG_API int gpg_net_gradients(gpg_net *net, int npatch, const float *d_rho, const float *d_pot_in,
                              const float *d_target, double cnst, float *d_grad, float *d_loss, void *stream);
/* gradients + one Adam step (beta 0.9 / 0.999, eps 1e-8) */
GPG_API int gpg_net_train_step(gpg_net *net, int npatch, const float *d_rho, const float *d_pot_in,
                               const float *d_target, double cnst, float lr, float *d_loss, void *stream);
/* one Adam step with a caller-supplied gradient [param_count] on the device
 * (stream-ordered): data-parallel training computes per-rank gradients with
 * gpg_net_gradients, averages them across ranks (an all-reduce), and applies
 * the average here on every rank; gradients + this call = gpg_net_train_step */
GPG_API int gpg_net_apply_gradient(gpg_net *net, const float *d_grad, float lr, void *stream);
/* GPG_ERR_CUDA when a tensor-core wait timed out in an earlier call; reading
 * the flag clears it */
GPG_API int gpg_net_check(gpg_net *net);
/* Test hook: with polls > 0 every later gpg_net_predict also makes one
 * bounded wait of that many polls on a barrier nothing signals, so the
 * timeout path runs (the prediction itself completes normally); 0 = off. */
GPG_API int gpg_net_set_wait_probe(gpg_net *net, int polls);
GPG_API const char *gpg_net_last_error(void);

/* ---------------------------------------------------------------------------
 * Learned linear correction of the interpolated start, fused into ghost-size-1
 * FP32 SOR.  No reference counterpart (the reference starts from the
 * interpolated coarse potential, CPU_PoissonSolver_SOR.cpp:80-209, and runs
 * SOR from there).  The start value is phi_i + delta: phi_i the interpolated
 * coarse potential, delta a learned linear function of the residual
 * r0 = Lap(phi_i) - Const*rho of that start on the 8^3 interior.  The map is
 * equivariant under the reflections of the cube: r0 is folded by a length-8
 * Walsh-Hadamard transform per mirror orbit into 8 parity blocks of 64, block
 * b is multiplied by the 64 x 64 matrix of its class (number of odd axes,
 * 0..3; blocks of one class share it through an axis permutation of the orbit
 * index) and the result unfolded.  Parameters: W[4][64][64] FP32, row =
 * output orbit, column = input orbit, orbit o = k*16 + j*4 + i (z, y, x in
 * [0,4), the class representative's axes).  The solve runs the fold, the BF16
 * tcgen05 MMAs (FP32 accumulation), the unfold and the SOR sweeps in one
 * persistent kernel; the correction never leaves the chip.
 * ------------------------------------------------------------------------- */
typedef struct gpg_lin gpg_lin;
/* every call on a lin makes its device current (as for gpg_net) */
/* max_batch bounds npatch of gpg_lin_gradients / gpg_lin_train_step only;
 * parameters start at zero (delta = 0: the plain interpolated start) */
GPG_API int gpg_lin_create(gpg_lin **lin, int max_batch, int device_id);
GPG_API int gpg_lin_destroy(gpg_lin *lin);
GPG_API int gpg_lin_param_count(int64_t *count);
GPG_API int gpg_lin_get_params(gpg_lin *lin, float *host_params);
GPG_API int gpg_lin_set_params(gpg_lin *lin, const float *host_params);
/* Stream-ordered solve with the learned start: the arguments and outputs of
 * gpg_poisson_gravity_device for p->ghost == 1, p->real_size == 4, SOR (any
 * stopping rule, output window and fused gravity update; p->init_mode is
 * ignored).  d_pot_out [P][GRA_NXT]^3, d_flu [P][5][8]^3 when p->gra_acc. */
GPG_API int gpg_lin_solve_device(gpg_lin *lin, const gpg_params *p, int npatch, const float *d_rho,
                                 const float *d_pot_in, float *d_pot_out, float *d_flu, int32_t *d_iters,
                                 double *d_resid, void *stream);
/* Training features (stream-ordered): d_u [P][8][64] the folded residual of
 * each patch (block b at b*64, orbit index in its class's axes); when
 * d_target [P][8]^3 (a converged interior potential) is given, d_t [P][8][64]
 * the folded (target - interpolated start) / 8, so that the unfold of
 * W u ~ t is the correction.  Both are scaled by the power of two 2^(17 - e)
 * with the patch's largest |interpolated potential| = m 2^e, m in [0.5, 1):
 * exact, immaterial to a linear map; it makes the training loss measure each
 * patch's start error relative to its potential, with the features near one. */
GPG_API int gpg_lin_features(gpg_lin *lin, const gpg_params *p, int npatch, const float *d_rho,
                             const float *d_pot_in, const float *d_target, float *d_u, float *d_t, void *stream);
/* loss = mean over patches, blocks and rows of (W u - t)^2; its gradient wrt
 * W into d_grad [16384] (may be NULL: kept inside) and the loss into d_loss
 * (may be NULL) */
GPG_API int gpg_lin_gradients(gpg_lin *lin, int npatch, const float *d_u, const float *d_t, float *d_grad,
                              float *d_loss, void *stream);
/* gradients + one Adam step (beta 0.9 / 0.999, eps 1e-8) */
GPG_API int gpg_lin_train_step(gpg_lin *lin, int npatch, const float *d_u, const float *d_t, float lr,
                               float *d_loss, void *stream);
/* one Adam step with a caller-supplied gradient (data-parallel training) */
GPG_API int gpg_lin_apply_gradient(gpg_lin *lin, const float *d_grad, float lr, void *stream);
/* Launch shape of the fused solve: 0 (default) = per SM two groups of 8 teams
 * whose inputs are prefetched into shared memory by bulk copies, 1 = three
 * groups of 8 teams reading their inputs from global memory.  Every shape
 * gives the same bits. */
GPG_API int gpg_lin_variant_count(void);
GPG_API int gpg_lin_set_variant(gpg_lin *lin, int variant);
/* GPG_ERR_CUDA when a tensor-core wait of an earlier solve timed out; reading
 * the flag clears it */
GPG_API int gpg_lin_check(gpg_lin *lin);
/* Test hook: with polls > 0 every later solve also makes one bounded wait of
 * that many polls on a barrier nothing signals, so the timeout path runs
 * (the solve itself completes normally); 0 switches it off. */
GPG_API int gpg_lin_set_wait_probe(gpg_lin *lin, int polls);
GPG_API const char *gpg_lin_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* GPG_H */
