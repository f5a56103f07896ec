// cuapi_compat.cpp -- the reference's CUAPI_* functions (Header/Prototype.h:15-35)
// implemented on libgpg's C-ABI (include/gpg.h).
//
// Compile with the caller's macros (see include/gpg_cuapi.h), plain C++, no
// CUDA compiler needed; link with libgpg.so.  When the caller's build already
// provides `real` and IntScheme_t through the reference headers, pass
// -DGPG_CUAPI_NO_TYPES and include them first.
//
// The reference keeps its device buffers and streams in module globals
// (GPU_API/CUAPI_Asyn_PoissonGravitySolver.cu:32-39) and reads the caller's
// GPU_NSTREAM (GPU_API/CUAPI_MemAllocate_PoissonGravity.cu:11,76-77); here a
// single gpg_context plays that role, created by MemAllocate with the stream
// count CUAPI_Set_Diagnose_Device settled on.  Failures print the library's
// message and end the process with exit(-1), as Header/CUAPI.h:10-21 does.
#include <cstdio>
#include <cstdlib>

#include "../../../include/gpg_cuapi.h"
#include "../../../include/gpg.h"

namespace {

gpg_context *g_ctx = nullptr;
int g_device = 0;
int g_nstream = 1;

[[noreturn]] void die(const char *func, int status) {
  std::fprintf(stderr, "ERROR : %s failed (gpg status %d): %s !!\n", func, status, gpg_last_error());
  std::fflush(stderr);
  std::exit(-1);
}

#define GPG_CUAPI_CHECK(call)                     \
  do {                                            \
    int rc_ = (call);                             \
    if (rc_ != GPG_OK) die(__func__, rc_);        \
  } while (0)

gpg_params shape_params() {
  gpg_params p;
  GPG_CUAPI_CHECK(gpg_default_params(&p, (int)sizeof(real), POT_GHOST_SIZE, POT_SCHEME));
  p.gra_ghost = GRA_GHOST_SIZE;
  p.gra_acc = GRA_GHOST_SIZE > 0;
  return p;
}

}  // namespace

void CUAPI_Set_Diagnose_Device(int &FLU_GPU_NPGroup, int &GPU_NStream, const int InputID) {
  GPG_CUAPI_CHECK(gpg_set_diagnose_device(&FLU_GPU_NPGroup, &GPU_NStream, InputID));
  g_device = InputID;
  g_nstream = GPU_NStream;
}

void CUAPI_MemAllocate_PoissonGravity(const int Pot_NPatchGroup,
                                      real (**Rho_Array_P)[RHO_NXT][RHO_NXT][RHO_NXT],
                                      real (**Pot_Array_P_In)[POT_NXT][POT_NXT][POT_NXT],
                                      real (**Pot_Array_P_Out)[GRA_NXT][GRA_NXT][GRA_NXT],
                                      real (**Flu_Array_G)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE]) {
  if (!g_ctx) GPG_CUAPI_CHECK(gpg_context_create(&g_ctx, g_device, g_nstream));
  const gpg_params shape = shape_params();
  void *rho = nullptr, *pin = nullptr, *pout = nullptr, *flu = nullptr;
  GPG_CUAPI_CHECK(gpg_mem_allocate(g_ctx, &shape, Pot_NPatchGroup, &rho, &pin, &pout, &flu));
  const long npatch = 8L * Pot_NPatchGroup;
  const long mb = (long)sizeof(real) * npatch *
                  (RHO_NXT * RHO_NXT * RHO_NXT + POT_NXT * POT_NXT * POT_NXT + GRA_NXT * GRA_NXT * GRA_NXT +
                   NCOMP * PATCH_SIZE * PATCH_SIZE * PATCH_SIZE) / (1 << 20);
  std::fprintf(stdout, "NOTE : total memory requirement in GPU gravity solver = %ld MB\n", mb);
  std::fflush(stdout);
  *Rho_Array_P = reinterpret_cast<real(*)[RHO_NXT][RHO_NXT][RHO_NXT]>(rho);
  *Pot_Array_P_In = reinterpret_cast<real(*)[POT_NXT][POT_NXT][POT_NXT]>(pin);
  *Pot_Array_P_Out = reinterpret_cast<real(*)[GRA_NXT][GRA_NXT][GRA_NXT]>(pout);
  *Flu_Array_G = reinterpret_cast<real(*)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE]>(flu);
}

void CUAPI_MemFree_PoissonGravity(real (**Rho_Array_P)[RHO_NXT][RHO_NXT][RHO_NXT],
                                  real (**Pot_Array_P_In)[POT_NXT][POT_NXT][POT_NXT],
                                  real (**Pot_Array_P_Out)[GRA_NXT][GRA_NXT][GRA_NXT],
                                  real (**Flu_Array_G)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE]) {
  if (!g_ctx) return;
  void *p[4] = {*Rho_Array_P, *Pot_Array_P_In, *Pot_Array_P_Out, *Flu_Array_G};
  GPG_CUAPI_CHECK(gpg_mem_free(g_ctx, &p[0], &p[1], &p[2], &p[3]));
  *Rho_Array_P = nullptr;
  *Pot_Array_P_In = nullptr;
  *Pot_Array_P_Out = nullptr;
  *Flu_Array_G = nullptr;
  GPG_CUAPI_CHECK(gpg_context_destroy(g_ctx));
  g_ctx = nullptr;
}

void CUAPI_Asyn_PoissonGravitySolver(const real h_Rho_Array[][RHO_NXT][RHO_NXT][RHO_NXT],
                                     real h_Pot_Array_In[][POT_NXT][POT_NXT][POT_NXT],
                                     real h_Pot_Array_Out[][GRA_NXT][GRA_NXT][GRA_NXT],
                                     real h_Flu_Array[][5][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE],
                                     const int NPatchGroup, const real dt, const real dh,
                                     const int SOR_Min_Iter, const int SOR_Max_Iter, const real SOR_Omega,
                                     const int MG_Max_Iter, const int MG_NPre_Smooth,
                                     const int MG_NPost_Smooth, const real MG_Tolerated_Error,
                                     const real Poi_Coeff, const IntScheme_t IntScheme,
                                     const bool P5_Gradient, const bool Poisson, const bool GraAcc,
                                     const int GPU_NStream) {
  if (!g_ctx) die(__func__, GPG_ERR_STATE);
  gpg_params p = shape_params();
  p.dt = dt;
  p.dh = dh;
  p.sor_min_iter = SOR_Min_Iter;
  p.sor_max_iter = SOR_Max_Iter;
  p.sor_omega = SOR_Omega;
  p.mg_max_iter = MG_Max_Iter;
  p.mg_npre_smooth = MG_NPre_Smooth;
  p.mg_npost_smooth = MG_NPost_Smooth;
  p.mg_tolerated_error = MG_Tolerated_Error;
  p.poi_coeff = Poi_Coeff;
  p.int_scheme = (int)IntScheme;
  p.p5_gradient = P5_Gradient;
  p.poisson = Poisson;
  p.gra_acc = GraAcc;
  GPG_CUAPI_CHECK(gpg_asyn_poisson_gravity_solver(g_ctx, h_Rho_Array, h_Pot_Array_In, h_Pot_Array_Out,
                                                  h_Flu_Array, NPatchGroup, &p, GPU_NStream));
}

void CUAPI_Synchronize() { GPG_CUAPI_CHECK(gpg_synchronize(g_ctx)); }
