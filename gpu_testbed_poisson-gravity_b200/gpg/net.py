"""ctypes binding of the learned initial guess (gpg_net_* in include/gpg.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .lib import GpgError, library

LAYERS = ((8, 32), (32, 32), (32, 32), (32, 16))   # (cin, cout), padded


def _net_lib():
    lib = library()
    if not getattr(lib, "_net_sigs", False):
        vp = C.c_void_p
        sig = {
            "gpg_net_create": (C.c_int, [C.POINTER(vp), C.c_int, C.c_uint64, C.c_int]),
            "gpg_net_destroy": (C.c_int, [vp]),
            "gpg_net_param_count": (C.c_int, [C.POINTER(C.c_int64)]),
            "gpg_net_get_params": (C.c_int, [vp, vp]),
            "gpg_net_set_params": (C.c_int, [vp, vp]),
            "gpg_net_predict": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp]),
            "gpg_net_predict_layers": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp]),
            "gpg_net_gradients": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, vp, vp, vp]),
            "gpg_net_train_step": (C.c_int, [vp, C.c_int, vp, vp, vp, C.c_double, C.c_float, vp, vp]),
            "gpg_net_apply_gradient": (C.c_int, [vp, vp, C.c_float, vp]),
            "gpg_net_check": (C.c_int, [vp]),
            "gpg_net_set_wait_probe": (C.c_int, [vp, C.c_int]),
            "gpg_net_last_error": (C.c_char_p, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        lib._net_sigs = True
    return lib


def _check(rc):
    if rc != 0:
        msg = _net_lib().gpg_net_last_error()
        raise GpgError(rc, msg.decode() if msg else "")


def split_params(flat: np.ndarray):
    """Flat parameter vector -> ([W0..W3] as [27][cin][cout], [b0..b3])."""
    ws, bs, o = [], [], 0
    for cin, cout in LAYERS:
        n = 27 * cin * cout
        ws.append(flat[o:o + n].reshape(27, cin, cout))
        o += n
        bs.append(flat[o:o + cout])
        o += cout
    return ws, bs


def flatten_params(ws, bs) -> np.ndarray:
    return np.concatenate([np.concatenate([w.reshape(-1), b.reshape(-1)]) for w, b in zip(ws, bs)]).astype(np.float32)


class Net:
    """Learned initial-guess network on the GPU (ghost-size-1 patches)."""

    def __init__(self, max_batch: int = 1024, seed: int = 1, device_id: int = 0):
        self._n = C.c_void_p()
        _check(_net_lib().gpg_net_create(C.byref(self._n), max_batch, seed, device_id))
        cnt = C.c_int64()
        _check(_net_lib().gpg_net_param_count(C.byref(cnt)))
        self.nparams = cnt.value
        self.max_batch = max_batch

    def params(self) -> np.ndarray:
        out = np.empty(self.nparams, dtype=np.float32)
        _check(_net_lib().gpg_net_get_params(self._n, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_params(self, flat: np.ndarray):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        _check(_net_lib().gpg_net_set_params(self._n, flat.ctypes.data_as(C.c_void_p)))

    @staticmethod
    def _s(stream):
        import torch
        return C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)

    def predict(self, rho, pot_in, guess, cnst: float, stream=None, fused: bool = True):
        """Interior guess; `fused` False runs the per-layer kernels instead."""
        fn = _net_lib().gpg_net_predict if fused else _net_lib().gpg_net_predict_layers
        _check(fn(self._n, int(rho.shape[0]), rho.data_ptr(), pot_in.data_ptr(), guess.data_ptr(), cnst,
                  self._s(stream)))

    def gradients(self, rho, pot_in, target, cnst: float, grad=None, loss=None, stream=None):
        _check(_net_lib().gpg_net_gradients(self._n, int(rho.shape[0]), rho.data_ptr(), pot_in.data_ptr(),
                                            target.data_ptr(), cnst,
                                            None if grad is None else grad.data_ptr(),
                                            None if loss is None else loss.data_ptr(), self._s(stream)))

    def train_step(self, rho, pot_in, target, cnst: float, lr: float, loss=None, stream=None):
        _check(_net_lib().gpg_net_train_step(self._n, int(rho.shape[0]), rho.data_ptr(), pot_in.data_ptr(),
                                             target.data_ptr(), cnst, lr,
                                             None if loss is None else loss.data_ptr(), self._s(stream)))

    def apply_gradient(self, grad, lr: float, stream=None):
        """Adam step with `grad` (a CUDA float32 tensor of nparams values)."""
        if grad.numel() != self.nparams or not grad.is_cuda or grad.dtype.itemsize != 4 or not grad.is_contiguous():
            raise ValueError(f"grad must be a contiguous CUDA float32 tensor of {self.nparams} values")
        _check(_net_lib().gpg_net_apply_gradient(self._n, grad.data_ptr(), lr, self._s(stream)))

    def check(self):
        _check(_net_lib().gpg_net_check(self._n))

    def set_wait_probe(self, polls: int):
        """Test hook (gpg_net_set_wait_probe)."""
        _check(_net_lib().gpg_net_set_wait_probe(self._n, int(polls)))

    def close(self):
        if self._n:
            _check(_net_lib().gpg_net_destroy(self._n))
            self._n = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
