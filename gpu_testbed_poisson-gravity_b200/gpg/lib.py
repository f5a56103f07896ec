"""ctypes binding of libgpg.so (include/gpg.h).

The CUDA library is the only compute path: if lib/libgpg.so is missing or a
CUDA call fails, the functions here raise; nothing falls back to the CPU.

Two API levels, as in the reference (Header/Prototype.h:15-35):

* device level  ``solve_device`` -- torch CUDA tensors in, stream-ordered;
* host level    ``Context``      -- the CUAPI_* flow: allocate pinned host
  buffers + device buffers, ``asyn_solve`` (H2D, kernels, D2H per stream,
  returns early), ``synchronize``, ``free``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .abi import GPG_OK, GPG_SOR, GpgBatchGroup, GpgParams, default_params, patch_sizes  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libgpg.so")

_lib = None


class GpgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"gpg status {status}: {message}")
        self.status = status


def library(path: str | None = None):
    """Load libgpg.so once (build it with gpu_testbed_poisson-gravity_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built; run python gpu_testbed_poisson-gravity_b200/build.py")
    lib = C.CDLL(path)
    P = C.POINTER(GpgParams)
    vp = C.c_void_p
    sig = {
        "gpg_abi_version": (C.c_int, []),
        "gpg_last_error": (C.c_char_p, []),
        "gpg_default_params": (C.c_int, [P, C.c_int, C.c_int, C.c_int]),
        "gpg_validate_params": (C.c_int, [P]),
        "gpg_pot_tolerance": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
        "gpg_patch_sizes": (C.c_int, [P] + [C.POINTER(C.c_int64)] * 4),
        "gpg_poisson_gravity_device": (C.c_int, [P, C.c_int] + [vp] * 8),
        "gpg_set_diagnose_device": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
        "gpg_context_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int]),
        "gpg_context_destroy": (C.c_int, [vp]),
        "gpg_mem_allocate": (C.c_int, [vp, P, C.c_int] + [C.POINTER(vp)] * 4),
        "gpg_mem_free": (C.c_int, [vp] + [C.POINTER(vp)] * 4),
        "gpg_asyn_poisson_gravity_solver": (C.c_int, [vp, vp, vp, vp, vp, C.c_int, P, C.c_int]),
        "gpg_synchronize": (C.c_int, [vp]),
        "gpg_last_iterations": (C.c_int, [vp, vp, vp, C.c_int]),
        "gpg_solve_batch_device": (C.c_int, [P, C.c_int, C.POINTER(GpgBatchGroup), vp, vp]),
        "gpg_batch_plan_create": (C.c_int, [C.POINTER(vp), P, C.c_int, C.POINTER(GpgBatchGroup), C.c_int,
                                            C.c_int]),
        "gpg_batch_plan_launch": (C.c_int, [vp, vp]),
        "gpg_batch_plan_destroy": (C.c_int, [vp]),
        "gpg_sor_variant_count": (C.c_int, []),
        "gpg_sor_variant_info": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "gpg_sor_variant_layout": (C.c_int, [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "gpg_sor_variant_staged": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
        "gpg_sor_variant_for_launch": (C.c_int, [C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_int)]),
        "gpg_sor_layout": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
        "gpg_set_sor_variant": (C.c_int, [C.c_int, C.c_int, C.c_int]),
        "gpg_get_sor_variant": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != GPG_OK:
        msg = library().gpg_last_error()
        raise GpgError(rc, msg.decode() if msg else "")


def _tptr(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("device API needs contiguous CUDA tensors")
    return C.c_void_p(t.data_ptr())


def solve_device(p: GpgParams, rho=None, pot_in=None, pot_out=None, flu=None, guess=None, iters=None,
                 resid=None, stream=None, npatch: int | None = None):
    """Run the Poisson(+gravity) path on torch CUDA tensors (stream-ordered).

    Allocates pot_out / iters / resid when not given (iters and resid always
    returned).  `stream` is a torch.cuda.Stream or None (current stream)."""
    import torch
    dt = torch.float32 if p.real_size == 4 else torch.float64
    src = rho if rho is not None else pot_out
    n = src.shape[0] if npatch is None else npatch
    dev = src.device
    gn = 8 + 2 * p.gra_ghost
    if pot_out is None:
        pot_out = torch.empty((n, gn, gn, gn), dtype=dt, device=dev)
    if iters is None:
        iters = torch.empty(n, dtype=torch.int32, device=dev)
    if resid is None:
        resid = torch.empty(n, dtype=torch.float64, device=dev)
    for t in (rho, pot_in, pot_out, flu, guess):
        if t is not None and t.dtype != dt:
            raise TypeError(f"expected {dt}, got {t.dtype}")
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    rc = library().gpg_poisson_gravity_device(
        C.byref(p), int(n), _tptr(rho), _tptr(pot_in), _tptr(pot_out), _tptr(flu), _tptr(guess),
        _tptr(iters), _tptr(resid), C.c_void_p(s.cuda_stream))
    check(rc)
    return pot_out, flu, iters, resid


def set_diagnose_device(device_id: int = 0, npgroup: int | None = None, nstream: int | None = None):
    """CUAPI_Set_Diagnose_Device: returns (npgroup, nstream) with defaults filled in."""
    from .abi import NULL_INT
    a = C.c_int(NULL_INT if npgroup is None else npgroup)
    b = C.c_int(NULL_INT if nstream is None else nstream)
    check(library().gpg_set_diagnose_device(C.byref(a), C.byref(b), device_id))
    return a.value, b.value


class Context:
    """Reference-shaped host API: one context = the reference's module globals
    (device arrays, pinned host arrays, streams)."""

    def __init__(self, device_id: int = 0, nstream: int = 4):
        self._ctx = C.c_void_p()
        check(library().gpg_context_create(C.byref(self._ctx), device_id, nstream))
        self.nstream = nstream
        self._host = None
        self.shape = None

    def allocate(self, shape: GpgParams, npatch_group: int):
        """CUAPI_MemAllocate_PoissonGravity: returns numpy views (rho, pot_in,
        pot_out, flu) over the library's pinned host buffers."""
        ptrs = [C.c_void_p() for _ in range(4)]
        check(library().gpg_mem_allocate(self._ctx, C.byref(shape), npatch_group,
                                         *[C.byref(q) for q in ptrs]))
        self.shape = shape.copy()
        sz = patch_sizes(shape)
        n = 8 * npatch_group
        ct = C.c_float if shape.real_size == 4 else C.c_double
        m, pn, gn = sz["rho_nxt"], sz["pot_nxt"], sz["gra_nxt"]
        shapes = [(n, m, m, m), (n, pn, pn, pn), (n, gn, gn, gn), (n, 5, 8, 8, 8)]
        views = []
        for q, shp in zip(ptrs, shapes):
            cnt = int(np.prod(shp))
            if cnt == 0:
                views.append(np.zeros(shp, dtype=shape.dtype))
                continue
            buf = (ct * cnt).from_address(q.value)
            views.append(np.ctypeslib.as_array(buf).reshape(shp))
        self._host = ptrs
        self.npatch = n
        return tuple(views)

    def asyn_solve(self, p: GpgParams, npatch_group: int, nstream: int | None = None, host=None):
        """CUAPI_Asyn_PoissonGravitySolver on the allocated pinned buffers (or
        on `host` = (rho, pot_in, pot_out, flu) numpy arrays)."""
        if host is None:
            ptrs = self._host if self._host is not None else [None] * 4
        else:
            ptrs = [C.c_void_p(a.ctypes.data) if a is not None else None for a in host]
        check(library().gpg_asyn_poisson_gravity_solver(self._ctx, ptrs[0], ptrs[1], ptrs[2], ptrs[3],
                                                        npatch_group, C.byref(p),
                                                        nstream or self.nstream))

    def synchronize(self):
        check(library().gpg_synchronize(self._ctx))

    def iterations(self, npatch: int):
        it = np.zeros(npatch, dtype=np.int32)
        rs = np.zeros(npatch, dtype=np.float64)
        check(library().gpg_last_iterations(self._ctx, C.c_void_p(it.ctypes.data),
                                            C.c_void_p(rs.ctypes.data), npatch))
        return it, rs

    def free(self):
        if self._host is not None:
            check(library().gpg_mem_free(self._ctx, *[C.byref(q) for q in self._host]))
            self._host = None

    def close(self):
        if self._ctx:
            self.free()
            check(library().gpg_context_destroy(self._ctx))
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ---------------------------------------------------------------------------
# batched mixed-ghost-size SOR
# ---------------------------------------------------------------------------
def make_batch_groups(p: GpgParams, groups: list[dict]):
    """ctypes array of gpg_batch_group from dicts of torch CUDA tensors
    (keys: ghost, rho, pot_in, pot_out, flu, guess, iters, resid, omega)."""
    arr = (GpgBatchGroup * max(1, len(groups)))()
    for i, g in enumerate(groups):
        a = arr[i]
        a.ghost = g["ghost"]
        a.npatch = int(g["rho"].shape[0])
        for k, f in (("rho", "d_rho"), ("pot_in", "d_pot_in"), ("pot_out", "d_pot_out"), ("flu", "d_flu"),
                     ("guess", "d_guess"), ("iters", "d_iters"), ("resid", "d_resid")):
            t = g.get(k)
            setattr(a, f, None if t is None else _tptr(t).value)
        a.sor_omega = g.get("omega", 0.0)
    return arr


def solve_batch_device(p: GpgParams, groups: list[dict], counter, stream=None):
    """One persistent launch over groups of different ghost sizes.  `counter`:
    a 1-element int32 CUDA tensor used as the work-queue counter."""
    import torch
    arr = make_batch_groups(p, groups)
    s = stream if stream is not None else torch.cuda.current_stream(counter.device)
    check(library().gpg_solve_batch_device(C.byref(p), len(groups), arr, _tptr(counter),
                                           C.c_void_p(s.cuda_stream)))


PLAN_PERSISTENT, PLAN_CONCURRENT = 0, 1


class BatchPlan:
    """The batch captured once into a CUDA graph; launch() replays it.
    mode PLAN_PERSISTENT: the work-queue kernel; PLAN_CONCURRENT: the
    per-ghost-size kernels as parallel graph branches."""

    def __init__(self, p: GpgParams, groups: list[dict], device_id: int = 0, mode: int = PLAN_PERSISTENT):
        self._plan = C.c_void_p()
        self._keep = groups  # buffers must outlive the graph
        arr = make_batch_groups(p, groups)
        check(library().gpg_batch_plan_create(C.byref(self._plan), C.byref(p), len(groups), arr, device_id,
                                              mode))

    def launch(self, stream=None):
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        check(library().gpg_batch_plan_launch(self._plan, C.c_void_p(s.cuda_stream)))

    def close(self):
        if self._plan:
            check(library().gpg_batch_plan_destroy(self._plan))
            self._plan = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
