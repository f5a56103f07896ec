"""Time one configuration of the Poisson(-gravity) path on the device.

    python gpu_testbed_poisson-gravity_b200/run_config.py --scheme mg --ghost 3 --prec 4 \
        --gra-ghost 2 --p5 --npatch 16384 [--gravity] [--reps 5] [--warm 3] [--variant V]

Seeded inputs from gpg.inputs (power-law density, analytic coarse potential,
fluid when --gravity), reference parameters (gpg_default_params) unless
overridden, CUDA events on the launching stream.  Prints one JSON line:
milliseconds per call, patches/s, mean iterations.  Used for profiling
recipes (one configuration per process).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from gpg.abi import GPG_MG, GPG_SOR, default_params  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--scheme", choices=["sor", "mg"], default="sor")
    ap.add_argument("--ghost", type=int, default=3)
    ap.add_argument("--prec", type=int, choices=[4, 8], default=4, help="bytes per real")
    ap.add_argument("--gra-ghost", type=int, default=1)
    ap.add_argument("--p5", action="store_true", help="5-point gravity gradient")
    ap.add_argument("--gravity", action="store_true", help="fused gravity update")
    ap.add_argument("--npatch", type=int, default=16384)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warm", type=int, default=3)
    ap.add_argument("--seed", type=int, default=21)
    ap.add_argument("--variant", type=int, default=None, help="SOR kernel variant (gpg_set_sor_variant)")
    a = ap.parse_args(argv)

    import ctypes as C
    import torch
    from gpg.lib import check, library, solve_device
    dev = torch.device("cuda:0")
    if a.variant is not None:
        check(library().gpg_set_sor_variant(a.prec, a.ghost, a.variant))
        v = C.c_int()
        check(library().gpg_get_sor_variant(a.prec, a.ghost, C.byref(v)))
    dt = np.float32 if a.prec == 4 else np.float64
    d = make_patches(a.npatch, a.ghost, seed=a.seed, gra_ghost=a.gra_ghost, dtype=dt, fluid=a.gravity)
    p = default_params(a.prec, a.ghost, GPG_SOR if a.scheme == "sor" else GPG_MG, gra_ghost=a.gra_ghost,
                       p5_gradient=int(a.p5), gra_acc=int(a.gravity))
    t = {k: torch.from_numpy(v).to(dev) for k, v in d.items() if k != "geometry"}
    gn = 8 + 2 * a.gra_ghost
    pot = torch.empty((a.npatch, gn, gn, gn), dtype=t["rho"].dtype, device=dev)
    it = torch.empty(a.npatch, dtype=torch.int32, device=dev)
    rs = torch.empty(a.npatch, dtype=torch.float64, device=dev)
    flu = t["flu"].clone() if a.gravity else None

    def run():  # the fluid is updated in place call after call (timing only)
        solve_device(p, t["rho"], t["pot_in"], pot_out=pot, flu=flu, iters=it, resid=rs)

    for _ in range(a.warm):
        run()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(a.reps):
        run()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / max(1, a.reps)
    print(json.dumps({"scheme": a.scheme, "ghost": a.ghost, "prec": a.prec, "gra_ghost": a.gra_ghost, "p5": a.p5,
                      "gravity": a.gravity, "npatch": a.npatch, "ms": ms, "patches_per_s": a.npatch / ms * 1e3,
                      "iters_mean": float(it.float().mean()), "variant": a.variant}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
