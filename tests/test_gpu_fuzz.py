"""Seeded random configurations across the parameter space, GPU vs the CPU
oracle (needs a B200).

Each case draws: scheme (SOR / MG), precision, ghost size 1-5, output ghost
width 1-2, interpolation (CQUAD / QUAD), 5-point gradient, gravity on or off,
and per scheme the start (interpolated / zero / caller guess), stopping rule
(reference growth rule / relative tolerance), omega and iteration limits and
the SOR kernel variant (launch shape and lane layout), or the V-cycle count
and smoothing sweeps; 1-39 patches.  The comparison is the
one of test_gpu_parity: bit-identical fields wherever the per-patch iteration
counts agree, counts agreeing for >= 99 % of patches, the rest within the
relative L-infinity tolerance.
"""
import numpy as np
import pytest

from gpg.abi import (GPG_INIT_GUESS, GPG_INIT_INTERP, GPG_INIT_ZERO, GPG_INT_CQUAD, GPG_INT_QUAD, GPG_MG,
                     GPG_SOR, GPG_STOP_REFERENCE, GPG_STOP_TOLERANCE, default_params)
from gpg.inputs import make_patches
from oracle.oracle import run_oracle
from test_gpu_parity import compare, gpu_run, torch_cuda  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu

CASES = 64


def draw(i):
    rng = np.random.default_rng(9000 + i)
    scheme = int(rng.choice([GPG_SOR, GPG_MG]))
    rs = int(rng.choice([4, 8]))
    g = int(rng.integers(1, 6))
    G = int(rng.choice([1, 2])) if g >= 2 else 1   # output ghost width <= ghost size
    kw = dict(gra_ghost=G, p5_gradient=int(G == 2 and rng.random() < 0.5), gra_acc=int(rng.random() < 0.6),
              int_scheme=int(rng.choice([GPG_INT_CQUAD, GPG_INT_QUAD])))
    if scheme == GPG_SOR:
        stop = int(rng.choice([GPG_STOP_REFERENCE, GPG_STOP_TOLERANCE]))
        kw.update(init_mode=int(rng.choice([GPG_INIT_INTERP, GPG_INIT_ZERO, GPG_INIT_GUESS])), stop_mode=stop,
                  sor_omega=float(rng.uniform(1.3, 1.8)), sor_min_iter=int(rng.integers(1, 12)),
                  sor_max_iter=int(rng.integers(20, 120)))
        if stop == GPG_STOP_TOLERANCE:
            kw["sor_tolerance"] = 0.02 if rs == 4 else 1e-9
    else:
        kw.update(mg_max_iter=int(rng.integers(1, 6)), mg_npre_smooth=int(rng.integers(1, 4)),
                  mg_npost_smooth=int(rng.integers(1, 4)))
    variant = int(rng.integers(0, 14))
    return scheme, rs, g, kw, int(rng.integers(1, 40)), 9100 + i, variant


@pytest.mark.parametrize("i", range(CASES))
def test_random_configuration_matches_oracle(torch_cuda, i):
    import ctypes as C
    from gpg.lib import GpgError, check, library
    scheme, rs, g, kw, npatch, seed, variant = draw(i)
    dt = np.float32 if rs == 4 else np.float64
    p = default_params(rs, g, scheme, **kw)
    d = make_patches(npatch, g, seed=seed, gra_ghost=kw["gra_ghost"], dtype=dt, fluid=bool(kw["gra_acc"]))
    guess = None
    if kw.get("init_mode") == GPG_INIT_GUESS:
        m = 6 + 2 * g
        guess = (0.01 * np.random.default_rng(seed).standard_normal((npatch, m, m, m))).astype(dt)
    flu = d["flu"].copy() if kw["gra_acc"] else None
    o = run_oracle(p, d["rho"], d["pot_in"], flu=flu, guess=guess, accum_f64=True)
    lib = library()
    cur = C.c_int()
    check(lib.gpg_get_sor_variant(rs, g, C.byref(cur)))
    check(lib.gpg_set_sor_variant(rs, g, variant))
    try:
        out = gpu_run(torch_cuda, p, d, guess=guess)
    except GpgError as e:
        assert e.status == 5  # this variant does not fit this configuration
        out = None
    finally:
        check(lib.gpg_set_sor_variant(rs, g, -1))
    if out is None:
        out = gpu_run(torch_cuda, p, d, guess=guess)
    compare(p, out, o)
