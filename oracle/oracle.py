"""Python access to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

* ``run_oracle``    -> oracle/liboracle.so, the C restatement of the reference
                       CPU solvers (runtime sizes; f32 and f64).
* ``run_reference`` -> oracle/_ref/libref_*.so, the reference's own CPU code
                       compiled per configuration by oracle/build.py.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the library itself never does.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "gpu_testbed_poisson-gravity_b200"))

from gpg.abi import GpgParams  # noqa: E402

_lib = None
_ref_libs: dict = {}


def oracle_lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if os.path.exists(os.path.join(HERE, "gpg_oracle.c")):
            from oracle.build import build_oracle  # rebuilds only when out of date
            path = build_oracle()
        lib = C.CDLL(path)
        for sfx in ("f32", "f64"):
            f = getattr(lib, f"oracle_poisson_gravity_{sfx}")
            f.restype = C.c_int
            f.argtypes = [C.POINTER(GpgParams), C.c_int] + [C.c_void_p] * 5 + [
                C.c_int, C.c_int, C.c_void_p, C.c_void_p]
            g = getattr(lib, f"oracle_interp_cube_{sfx}")
            g.restype = None
            g.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        lib.oracle_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(a, dtype, name):
    if a is None:
        return None
    if a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"{name} must be a C-contiguous {np.dtype(dtype).name} array")
    return a


def run_oracle(p: GpgParams, rho, pot_in, pot_out=None, flu=None, guess=None, *,
               accum_f64: bool = True, nthreads: int = 0):
    """Run the restated CPU solver in place; returns (pot_out, flu, iters, resid).

    accum_f64=True accumulates the SOR residual / MG error sums in double (the
    CUDA library's arithmetic); False keeps the reference's `real` sums."""
    dt = np.float32 if p.real_size == 4 else np.float64
    n = (rho if rho is not None else pot_out).shape[0]
    gn = 8 + 2 * p.gra_ghost
    if pot_out is None:
        pot_out = np.zeros((n, gn, gn, gn), dtype=dt)
    for a, nm in ((rho, "rho"), (pot_in, "pot_in"), (pot_out, "pot_out"), (flu, "flu"),
                  (guess, "guess")):
        _check(a, dt, nm)
    if p.gra_acc and flu is None:
        raise ValueError("gra_acc needs flu")
    iters = np.zeros(n, dtype=np.int32)
    resid = np.zeros(n, dtype=np.float64)
    f = getattr(oracle_lib(), "oracle_poisson_gravity_" + ("f32" if p.real_size == 4 else "f64"))
    rc = f(C.byref(p), n, _ptr(rho), _ptr(pot_in), _ptr(pot_out), _ptr(flu), _ptr(guess),
           int(accum_f64), int(nthreads), _ptr(iters), _ptr(resid))
    if rc != 0:
        raise RuntimeError(f"oracle returned status {rc}")
    return pot_out, flu, iters, resid


def interp_cube(pot_in: np.ndarray, ghost: int, int_scheme: int) -> np.ndarray:
    """Interpolated N^3 cube of one patch (coarse [POT_NXT]^3 input)."""
    n = 8 + 2 * ghost
    out = np.zeros((n, n, n), dtype=pot_in.dtype)
    sfx = "f32" if pot_in.dtype == np.float32 else "f64"
    getattr(oracle_lib(), "oracle_interp_cube_" + sfx)(
        _ptr(np.ascontiguousarray(pot_in)), _ptr(out), ghost, int_scheme)
    return out


# --------------------------------------------------------------------------
# the reference's own CPU code (oracle/_ref)
# --------------------------------------------------------------------------

def ref_available(scheme: str = "sor", g: int = 1, G: int = 1, prec: str = "f32") -> bool:
    from oracle.build import ref_lib_path
    return os.path.exists(ref_lib_path(scheme, g, G, prec))


def ref_lib(scheme: str, g: int, G: int, prec: str):
    from oracle.build import ref_lib_path
    key = (scheme, g, G, prec)
    if key not in _ref_libs:
        path = ref_lib_path(*key)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run python oracle/build.py where the reference "
                                    "sources are present)")
        lib = C.CDLL(path, mode=os.RTLD_LOCAL)
        lib.ref_run.restype = C.c_int
        lib.ref_run.argtypes = ([C.c_void_p] * 4 + [C.c_int, C.c_double, C.c_double, C.c_int,
                                C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                                C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                C.c_void_p])
        lib.ref_config.argtypes = [C.POINTER(C.c_int)] * 5
        lib.ref_max_threads.restype = C.c_int
        vals = [C.c_int() for _ in range(5)]
        lib.ref_config(*[C.byref(v) for v in vals])
        want = (g, G, 4 if prec == "f32" else 8, 1 if scheme == "sor" else 2, 8)
        got = tuple(v.value for v in vals)
        if got != want:
            raise RuntimeError(f"{path}: configuration {got} != {want}")
        _ref_libs[key] = lib
    return _ref_libs[key]


def run_reference(p: GpgParams, rho, pot_in, pot_out=None, flu=None, *, nthreads: int = 0):
    """Run the reference CPU_PoissonGravitySolver in place (npatch % 8 == 0);
    returns (pot_out, flu, iters) where iters are the SOR counts it printed."""
    scheme = "sor" if p.scheme == 1 else "mg"
    prec = "f32" if p.real_size == 4 else "f64"
    G = p.gra_ghost if p.gra_ghost > 0 else 1
    lib = ref_lib(scheme, p.ghost, G, prec)
    dt = np.float32 if p.real_size == 4 else np.float64
    n = rho.shape[0]
    if n % 8:
        raise ValueError("the reference works on patch groups of 8")
    gn = 8 + 2 * G
    if pot_out is None:
        pot_out = np.zeros((n, gn, gn, gn), dtype=dt)
    if flu is None:
        flu = np.ones((n, 5, 8, 8, 8), dtype=dt)
    for a, nm in ((rho, "rho"), (pot_in, "pot_in"), (pot_out, "pot_out"), (flu, "flu")):
        _check(a, dt, nm)
    iters = np.full(n, -1, dtype=np.int32)
    rc = lib.ref_run(_ptr(rho), _ptr(pot_in), _ptr(pot_out), _ptr(flu), n // 8, p.dt, p.dh,
                     p.sor_min_iter, p.sor_max_iter, p.sor_omega, p.mg_max_iter,
                     p.mg_npre_smooth, p.mg_npost_smooth, p.mg_tolerated_error, p.poi_coeff,
                     p.int_scheme, p.p5_gradient, p.poisson, p.gra_acc, int(nthreads),
                     _ptr(iters))
    if rc != 0:
        raise RuntimeError("reference run failed")
    return pot_out, flu, iters
