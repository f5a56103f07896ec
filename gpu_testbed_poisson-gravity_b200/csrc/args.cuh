// args.cuh -- host-side conversion of a gpg_params block into the kernels'
// argument struct, shared by the solver entry points of libgpg.
#pragma once

#include <cstdint>

#include "../../include/gpg.h"
#include "common.cuh"

namespace gpg {

template <typename T>
inline SolveArgs<T> make_args(const gpg_params &p, int64_t npatch, const void *rho, const void *pin, void *pout,
                            void *flu, const void *guess, int32_t *iters, double *resid) {
  SolveArgs<T> a{};
  a.rho = static_cast<const T *>(rho);
  a.pot_in = static_cast<const T *>(pin);
  a.pot_out = static_cast<T *>(pout);
  a.flu = static_cast<T *>(flu);
  a.guess = static_cast<const T *>(guess);
  a.iters = iters;
  a.resid = resid;
  a.npatch = npatch;
  // rounding exactly where the reference rounds: its CPU_* functions take
  // `real` arguments and form these constants in `real`
  // (CPU_PoissonSolver_SOR.cpp:51-52, CPU_GravitySolver.cpp:23)
  const T dh = (T)p.dh, dt = (T)p.dt, poi = (T)p.poi_coeff, omega = (T)p.sor_omega;
  volatile T c = poi;  // volatile: keep each product rounded to T on the host
  c = c * dh;
  c = c * dh;
  a.sor_const = c;
  volatile T o6 = omega;
  o6 = o6 / (T)6.0;
  a.omega_6 = o6;
  a.gra_const = p.p5_gradient ? (T)((double)dt / (12.0 * (double)dh)) : (T)((double)dt / (2.0 * (double)dh));
  a.dh = dh;
  a.poi_coeff = poi;
  a.mg_tol = (T)p.mg_tolerated_error;
  a.sor_tol = p.sor_tolerance;
  a.min_iter = p.sor_min_iter;
  a.max_iter = p.sor_max_iter;
  a.mg_max_iter = p.mg_max_iter;
  a.mg_npre = p.mg_npre_smooth;
  a.mg_npost = p.mg_npost_smooth;
  a.int_scheme = p.int_scheme;
  a.init_mode = p.init_mode;
  a.stop_mode = p.stop_mode;
  a.gra_ghost = p.gra_ghost;
  a.gra_acc = p.gra_acc;
  a.p5 = p.p5_gradient;
  return a;
}

}  // namespace gpg
