"""gpg -- B200 per-patch Poisson-gravity library (Python side).

The compute path is the CUDA library lib/libgpg.so behind the C-ABI in
include/gpg.h; this package holds its ctypes binding (lib), the parameter
struct (abi), and the seeded synthetic input generator (inputs).
"""
from .abi import (GPG_INIT_GUESS, GPG_INIT_INTERP, GPG_INIT_ZERO, GPG_INT_CQUAD, GPG_INT_QUAD, GPG_MG,
                  GPG_SOR, GPG_STOP_REFERENCE, GPG_STOP_TOLERANCE, GpgParams, default_params,
                  patch_sizes)

__all__ = ["GpgParams", "default_params", "patch_sizes", "GPG_SOR", "GPG_MG", "GPG_INT_CQUAD",
           "GPG_INT_QUAD", "GPG_INIT_INTERP", "GPG_INIT_ZERO", "GPG_INIT_GUESS", "GPG_STOP_REFERENCE",
           "GPG_STOP_TOLERANCE"]
