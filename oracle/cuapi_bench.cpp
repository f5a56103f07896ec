// cuapi_bench.cpp -- TEST INFRASTRUCTURE ONLY: times one Poisson-gravity
// configuration through the reference's CUAPI interface (Header/Prototype.h:15-35)
// and writes the first call's outputs, so that two builds can be compared on
// the same inputs:
//   * linked on the reference's own GPU_API/ and GPU_Solver/ sources
//     (recompiled for sm_100a by oracle/build.py), built with -DREF_GPU;
//   * linked on this library's CUAPI shim and libgpg.
// The reference's CUAPI_Set_Diagnose_Device stops on any GPU that is not the
// architecture named by GPU_ARCH (CUAPI_Set_Diagnose_Device.cu:134-167, major
// revision 2/3/5/6), so the REF_GPU build does its remaining set-up itself:
// device selection, the shared-memory cache preference it asks for
// (CUAPI_Set_Diagnose_Device.cu:277-287, here device-wide) and the constant
// memory of the interpolation weights (CUPOT_PoissonSolver_SetConstMem).
//
//   cuapi_bench --in FILE --out FILE --npg N --nstream S --reps R --warm W
//               --min-iter A --max-iter B --omega W --mg-max-iter M --mg-npre a
//               --mg-npost b --mg-tol T --int-scheme I --p5 P
// The input file holds rho [8N][RHO_NXT^3], pot_in [8N][POT_NXT^3] and
// flu [8N][5][PS^3] in `real`; the output file pot_out [8N][GRA_NXT^3] and
// flu after the first call.  One JSON line on stdout: per-call wall times
// (host clock around CUAPI_Asyn_PoissonGravitySolver + CUAPI_Synchronize).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "Macro.h"
#include "Typedef.h"
#include "Prototype.h"

#ifdef REF_GPU
#include <cuda_runtime.h>
int CUPOT_PoissonSolver_SetConstMem();
#endif

// read by the reference's CUAPI_MemAllocate_PoissonGravity (extern there)
int GPU_NSTREAM = 1;

namespace {

struct Args {
  std::string in, out;
  int npg = 32, nstream = 1, reps = 10, warm = 2, min_iter = 10, max_iter = 60;
  double omega = 1.5, mg_tol = 1e-6;
  int mg_max_iter = 10, mg_npre = 3, mg_npost = 3, int_scheme = 4, p5 = 0;
};

bool parse(int argc, char **argv, Args &a) {
  for (int i = 1; i + 1 < argc; i += 2) {
    const std::string k = argv[i], v = argv[i + 1];
    if (k == "--in") a.in = v;
    else if (k == "--out") a.out = v;
    else if (k == "--npg") a.npg = std::atoi(v.c_str());
    else if (k == "--nstream") a.nstream = std::atoi(v.c_str());
    else if (k == "--reps") a.reps = std::atoi(v.c_str());
    else if (k == "--warm") a.warm = std::atoi(v.c_str());
    else if (k == "--min-iter") a.min_iter = std::atoi(v.c_str());
    else if (k == "--max-iter") a.max_iter = std::atoi(v.c_str());
    else if (k == "--omega") a.omega = std::atof(v.c_str());
    else if (k == "--mg-max-iter") a.mg_max_iter = std::atoi(v.c_str());
    else if (k == "--mg-npre") a.mg_npre = std::atoi(v.c_str());
    else if (k == "--mg-npost") a.mg_npost = std::atoi(v.c_str());
    else if (k == "--mg-tol") a.mg_tol = std::atof(v.c_str());
    else if (k == "--int-scheme") a.int_scheme = std::atoi(v.c_str());
    else if (k == "--p5") a.p5 = std::atoi(v.c_str());
    else return false;
  }
  return !a.in.empty() && !a.out.empty() && a.npg > 0 && a.nstream > 0 && a.reps > 0;
}

}  // namespace

int main(int argc, char **argv) {
  Args a;
  if (!parse(argc, argv, a)) {
    std::fprintf(stderr, "usage: see the header of cuapi_bench.cpp\n");
    return 2;
  }
  const int np = 8 * a.npg;
  const size_t nrho = size_t(np) * RHO_NXT * RHO_NXT * RHO_NXT, npin = size_t(np) * POT_NXT * POT_NXT * POT_NXT,
               npout = size_t(np) * GRA_NXT * GRA_NXT * GRA_NXT, nflu = size_t(np) * NCOMP * PATCH_SIZE * PATCH_SIZE * PATCH_SIZE;

  int npg = a.npg, nstream = a.nstream;
  GPU_NSTREAM = nstream;
#ifdef REF_GPU
  if (cudaSetDevice(0) != cudaSuccess || cudaDeviceSetCacheConfig(cudaFuncCachePreferShared) != cudaSuccess ||
      CUPOT_PoissonSolver_SetConstMem() != 0) {
    std::fprintf(stderr, "device set-up failed\n");
    return 1;
  }
#else
  CUAPI_Set_Diagnose_Device(npg, nstream, 0);
#endif
  real(*rho)[RHO_NXT][RHO_NXT][RHO_NXT] = nullptr;
  real(*pin)[POT_NXT][POT_NXT][POT_NXT] = nullptr;
  real(*pout)[GRA_NXT][GRA_NXT][GRA_NXT] = nullptr;
  real(*flu)[NCOMP][PATCH_SIZE][PATCH_SIZE][PATCH_SIZE] = nullptr;
  CUAPI_MemAllocate_PoissonGravity(npg, &rho, &pin, &pout, &flu);

  std::vector<real> flu0(nflu);
  {
    FILE *f = std::fopen(a.in.c_str(), "rb");
    if (!f) {
      std::fprintf(stderr, "cannot read %s\n", a.in.c_str());
      return 1;
    }
    const bool ok = std::fread(&rho[0][0][0][0], sizeof(real), nrho, f) == nrho &&
                    std::fread(&pin[0][0][0][0], sizeof(real), npin, f) == npin &&
                    std::fread(flu0.data(), sizeof(real), nflu, f) == nflu;
    std::fclose(f);
    if (!ok) {
      std::fprintf(stderr, "short input file %s\n", a.in.c_str());
      return 1;
    }
  }
  const real dt = real(DT), dh = real(DH), poi = real(4.0 * M_PI * NEWTON_G);
  auto call = [&]() {
    CUAPI_Asyn_PoissonGravitySolver(rho, pin, pout, flu, npg, dt, dh, a.min_iter, a.max_iter, real(a.omega),
                                    a.mg_max_iter, a.mg_npre, a.mg_npost, real(a.mg_tol), poi,
                                    IntScheme_t(a.int_scheme), a.p5 != 0, true, GRA_GHOST_SIZE > 0, nstream);
    CUAPI_Synchronize();
  };
  // first call: the outputs to compare (fluid restored before it)
  std::memcpy(&flu[0][0][0][0][0], flu0.data(), nflu * sizeof(real));
  call();
  {
    FILE *f = std::fopen(a.out.c_str(), "wb");
    if (!f || std::fwrite(&pout[0][0][0][0], sizeof(real), npout, f) != npout ||
        std::fwrite(&flu[0][0][0][0][0], sizeof(real), nflu, f) != nflu) {
      std::fprintf(stderr, "cannot write %s\n", a.out.c_str());
      return 1;
    }
    std::fclose(f);
  }
  // timed calls: the fluid is restored before each (outside the timed region)
  for (int w = 0; w < a.warm; ++w) call();
  std::vector<double> ms;
  for (int r = 0; r < a.reps; ++r) {
    std::memcpy(&flu[0][0][0][0][0], flu0.data(), nflu * sizeof(real));
    const auto t0 = std::chrono::steady_clock::now();
    call();
    const auto t1 = std::chrono::steady_clock::now();
    ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
  }
  std::sort(ms.begin(), ms.end());
  std::printf("{\"npatch\": %d, \"nstream\": %d, \"reps\": %d, \"ms_min\": %.6f, \"ms_median\": %.6f}\n", np, nstream,
              a.reps, ms.front(), ms[ms.size() / 2]);
  CUAPI_MemFree_PoissonGravity(&rho, &pin, &pout, &flu);
  return 0;
}
