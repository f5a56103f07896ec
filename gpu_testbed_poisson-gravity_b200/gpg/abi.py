"""ctypes mirror of include/gpg.h (the library's C-ABI) and parameter helpers."""
from __future__ import annotations

import ctypes as C
import math

GPG_OK = 0
GPG_ERR_INVALID = 1
GPG_ERR_CUDA = 2
GPG_ERR_NO_DEVICE = 3
GPG_ERR_OOM = 4
GPG_ERR_UNSUPPORTED = 5
GPG_ERR_STATE = 6

GPG_SOR, GPG_MG = 1, 2
GPG_INT_CQUAD, GPG_INT_QUAD = 4, 5
GPG_INIT_INTERP, GPG_INIT_ZERO, GPG_INIT_GUESS = 0, 1, 2
GPG_STOP_REFERENCE, GPG_STOP_TOLERANCE, GPG_STOP_ABS_TOLERANCE, GPG_STOP_POT_TOLERANCE = 0, 1, 2, 3
NULL_INT = 2147483647


class GpgParams(C.Structure):
    """Field-for-field copy of ``struct gpg_params`` in include/gpg.h."""

    _fields_ = [
        ("real_size", C.c_int32),
        ("ghost", C.c_int32),
        ("gra_ghost", C.c_int32),
        ("scheme", C.c_int32),
        ("int_scheme", C.c_int32),
        ("p5_gradient", C.c_int32),
        ("poisson", C.c_int32),
        ("gra_acc", C.c_int32),
        ("dt", C.c_double),
        ("dh", C.c_double),
        ("sor_min_iter", C.c_int32),
        ("sor_max_iter", C.c_int32),
        ("sor_omega", C.c_double),
        ("mg_max_iter", C.c_int32),
        ("mg_npre_smooth", C.c_int32),
        ("mg_npost_smooth", C.c_int32),
        ("init_mode", C.c_int32),
        ("mg_tolerated_error", C.c_double),
        ("poi_coeff", C.c_double),
        ("stop_mode", C.c_int32),
        ("reserved0", C.c_int32),
        ("sor_tolerance", C.c_double),
    ]

    def copy(self, **kw) -> "GpgParams":
        p = GpgParams()
        C.pointer(p)[0] = self
        for k, v in kw.items():
            if not hasattr(p, k):
                raise AttributeError(k)
            setattr(p, k, v)
        return p

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}

    @property
    def dtype(self):
        import numpy as np
        return np.float32 if self.real_size == 4 else np.float64


class GpgBatchGroup(C.Structure):
    """Field-for-field copy of ``struct gpg_batch_group`` in include/gpg.h."""

    _fields_ = [
        ("ghost", C.c_int32),
        ("npatch", C.c_int32),
        ("d_rho", C.c_void_p),
        ("d_pot_in", C.c_void_p),
        ("d_pot_out", C.c_void_p),
        ("d_flu", C.c_void_p),
        ("d_guess", C.c_void_p),
        ("d_iters", C.c_void_p),
        ("d_resid", C.c_void_p),
        ("sor_omega", C.c_double),
    ]


SOR_OMEGA = {1: 1.49, 2: 1.57, 3: 1.62, 4: 1.65, 5: 1.69}

# The fixed residual of GPG_STOP_POT_TOLERANCE per (sizeof(real), ghost):
# 2 x the 90th percentile of L1 residual / sum|interpolated phi| at the
# reference stopping point (CPU_PoissonSolver_SOR.cpp:275-281) of zero-start
# SOR on the seeded power-law inputs (oracle/calibrate_tol.py, 1024 patches,
# seed 11); gpg_pot_tolerance() in the C library returns the same values.
POT_TOL = {(4, 1): 9.8e-7, (4, 2): 1.1e-6, (4, 3): 1.2e-6, (4, 4): 1.3e-6, (4, 5): 1.4e-6,
           (8, 1): 1.8e-15, (8, 2): 2.1e-15, (8, 3): 2.3e-15, (8, 4): 2.4e-15, (8, 5): 2.5e-15}


def default_params(real_size: int = 4, ghost: int = 1, scheme: int = GPG_SOR, **kw) -> GpgParams:
    """Reference defaults (Main.cpp:1142-1223, Makefile:41-48) in Python;
    identical to gpg_default_params() of the C library."""
    if real_size not in (4, 8):
        raise ValueError("real_size must be 4 or 8")
    p = GpgParams()
    p.real_size = real_size
    p.ghost = ghost
    p.gra_ghost = 1
    p.scheme = scheme
    p.int_scheme = GPG_INT_CQUAD
    p.p5_gradient = 0
    p.poisson = 1
    p.gra_acc = 1
    p.dt = 1.0e-2
    p.dh = 1.0
    p.sor_min_iter = 10
    p.sor_max_iter = 60 if real_size == 4 else 100
    p.sor_omega = SOR_OMEGA[ghost]
    p.mg_max_iter = 10 if real_size == 4 else 20
    p.mg_npre_smooth = 3
    p.mg_npost_smooth = 3
    p.init_mode = GPG_INIT_INTERP
    p.mg_tolerated_error = 1.0e-6 if real_size == 4 else 1.0e-15
    p.poi_coeff = 4.0 * math.pi * 1.0e-5
    p.stop_mode = GPG_STOP_REFERENCE
    p.reserved0 = 0
    p.sor_tolerance = 0.0
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def patch_sizes(p: GpgParams) -> dict:
    g, G = p.ghost, p.gra_ghost
    m = 8 + 2 * (g - 1)
    pn = 4 + 2 * ((g + 3) // 2)
    gn = 8 + 2 * G
    return {"rho": m ** 3, "pot_in": pn ** 3, "pot_out": gn ** 3, "flu": 5 * 512,
            "rho_nxt": m, "pot_nxt": pn, "gra_nxt": gn, "cube": 8 + 2 * g}


def fixed_residual_params(real_size: int, ghost: int, init_mode: int = GPG_INIT_ZERO, max_iter: int = 300,
                          **kw) -> GpgParams:
    """SOR to the calibrated fixed residual: stop at the first sweep whose L1
    residual is <= POT_TOL x sum|interpolated phi| (Min_Iter 1, Max_Iter
    `max_iter`), Poisson only, interior output (gra_ghost 0)."""
    d = dict(gra_acc=0, gra_ghost=0, init_mode=init_mode, stop_mode=GPG_STOP_POT_TOLERANCE,
             sor_tolerance=POT_TOL[(real_size, ghost)], sor_min_iter=1, sor_max_iter=max_iter)
    d.update(kw)
    return default_params(real_size, ghost, GPG_SOR, **d)

