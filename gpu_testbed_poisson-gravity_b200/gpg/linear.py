"""ctypes binding of the learned linear correction (gpg_lin_* in include/gpg.h).

The correction maps the residual of the interpolated start of a ghost-size-1
patch to the change of its interior potential; it is equivariant under the
reflections of the cube (4 class matrices of 64 x 64 over the 8 parity
blocks).  The fused solve applies it on the tensor cores inside the SOR kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import GpgParams
from .lib import GpgError, library

NPARAMS = 4 * 64 * 64


def _lin_lib():
    lib = library()
    if not getattr(lib, "_lin_sigs", False):
        vp = C.c_void_p
        P = C.POINTER(GpgParams)
        sig = {
            "gpg_lin_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_int]),
            "gpg_lin_destroy": (C.c_int, [vp]),
            "gpg_lin_param_count": (C.c_int, [C.POINTER(C.c_int64)]),
            "gpg_lin_get_params": (C.c_int, [vp, vp]),
            "gpg_lin_set_params": (C.c_int, [vp, vp]),
            "gpg_lin_solve_device": (C.c_int, [vp, P, C.c_int] + [vp] * 7),
            "gpg_lin_features": (C.c_int, [vp, P, C.c_int] + [vp] * 6),
            "gpg_lin_gradients": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp]),
            "gpg_lin_train_step": (C.c_int, [vp, C.c_int, vp, vp, C.c_float, vp, vp]),
            "gpg_lin_apply_gradient": (C.c_int, [vp, vp, C.c_float, vp]),
            "gpg_lin_check": (C.c_int, [vp]),
            "gpg_lin_set_wait_probe": (C.c_int, [vp, C.c_int]),
            "gpg_lin_variant_count": (C.c_int, []),
            "gpg_lin_set_variant": (C.c_int, [vp, C.c_int]),
            "gpg_lin_last_error": (C.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        lib._lin_sigs = True
    return lib


def _check(rc):
    if rc != 0:
        msg = _lin_lib().gpg_lin_last_error()
        raise GpgError(rc, msg.decode() if msg else "")


def _p(t):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("the learned correction needs contiguous CUDA tensors")
    return C.c_void_p(t.data_ptr())


class LinearGuess:
    """Learned linear correction of the interpolated start (ghost size 1, FP32)."""

    def __init__(self, max_batch: int = 4096, device_id: int = 0):
        self._l = C.c_void_p()
        _check(_lin_lib().gpg_lin_create(C.byref(self._l), max_batch, device_id))
        cnt = C.c_int64()
        _check(_lin_lib().gpg_lin_param_count(C.byref(cnt)))
        self.nparams = cnt.value
        self.max_batch = max_batch

    @staticmethod
    def _s(stream):
        import torch
        return C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        _check(_lin_lib().gpg_lin_get_params(self._l, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, dtype=np.float32).reshape(-1)
        if flat.size != self.nparams:
            raise ValueError(f"{flat.size} parameters for a model of {self.nparams}")
        _check(_lin_lib().gpg_lin_set_params(self._l, flat.ctypes.data_as(C.c_void_p)))

    def solve(self, p: GpgParams, rho, pot_in, pot_out=None, flu=None, iters=None, resid=None, stream=None):
        """SOR from the learned start (stream-ordered); returns (pot_out, flu, iters, resid)."""
        import torch
        n = rho.shape[0]
        gn = 8 + 2 * p.gra_ghost
        if pot_out is None:
            pot_out = torch.empty((n, gn, gn, gn), dtype=torch.float32, device=rho.device)
        if iters is None:
            iters = torch.empty(n, dtype=torch.int32, device=rho.device)
        if resid is None:
            resid = torch.empty(n, dtype=torch.float64, device=rho.device)
        _check(_lin_lib().gpg_lin_solve_device(self._l, C.byref(p), int(n), _p(rho), _p(pot_in), _p(pot_out),
                                               _p(flu), _p(iters), _p(resid), self._s(stream)))
        return pot_out, flu, iters, resid

    def features(self, p: GpgParams, rho, pot_in, target=None, stream=None):
        """(u, t): folded residual and, with a converged `target` [P][8]^3, the
        folded block-space target; t is None without a target."""
        import torch
        n = rho.shape[0]
        u = torch.empty((n, 8, 64), dtype=torch.float32, device=rho.device)
        t = torch.empty((n, 8, 64), dtype=torch.float32, device=rho.device) if target is not None else None
        _check(_lin_lib().gpg_lin_features(self._l, C.byref(p), int(n), _p(rho), _p(pot_in), _p(target), _p(u),
                                           _p(t), self._s(stream)))
        return u, t

    def gradients(self, u, t, grad=None, loss=None, stream=None):
        _check(_lin_lib().gpg_lin_gradients(self._l, int(u.shape[0]), _p(u), _p(t), _p(grad), _p(loss),
                                            self._s(stream)))

    def train_step(self, u, t, lr: float, loss=None, stream=None):
        _check(_lin_lib().gpg_lin_train_step(self._l, int(u.shape[0]), _p(u), _p(t), lr, _p(loss),
                                             self._s(stream)))

    def apply_gradient(self, grad, lr: float, stream=None):
        if grad.numel() != self.nparams or grad.dtype.itemsize != 4:
            raise ValueError(f"grad must be a float32 CUDA tensor of {self.nparams} values")
        _check(_lin_lib().gpg_lin_apply_gradient(self._l, _p(grad), lr, self._s(stream)))

    def set_variant(self, variant: int):
        """Launch shape of the fused solve (gpg_lin_set_variant); same results."""
        _check(_lin_lib().gpg_lin_set_variant(self._l, int(variant)))

    @staticmethod
    def variant_count() -> int:
        return int(_lin_lib().gpg_lin_variant_count())

    def set_wait_probe(self, polls: int):
        _check(_lin_lib().gpg_lin_set_wait_probe(self._l, int(polls)))

    def check(self):
        _check(_lin_lib().gpg_lin_check(self._l))

    def close(self):
        if self._l:
            _check(_lin_lib().gpg_lin_destroy(self._l))
            self._l = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
