"""Calibrate the fixed-residual tolerance of GPG_STOP_POT_TOLERANCE.  TEST
INFRASTRUCTURE (runs the CPU oracle).

The reference SOR stops at its round-off floor: after the first sweep whose
L1 residual grows, once Iter+1 >= Min_Iter (CPU_PoissonSolver_SOR.cpp:
275-281).  From a zero interior that floor is a fixed multiple of the
potential's rounding error: residual / sum|phi_i| over the updated cells
(phi_i the interpolated coarse potential) clusters within a factor 1.2 per
(precision, ghost size), while residual / sum|Const rho| spreads over four
decades.  The tolerance is therefore

    tol(precision, ghost) = 2 x p90 of residual / sum|phi_i|

at the reference stopping point of zero-start SOR (Max_Iter raised so that
every patch reaches it), on the seeded power-law inputs (gpg.inputs), two
significant digits.  Every patch then reaches it, and it sits at the round-off
floor the reference rule stops at.

    python oracle/calibrate_tol.py [--npatch 1024] [--seed 11]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gpu_testbed_poisson-gravity_b200"))

from gpg.abi import GPG_INIT_ZERO, GPG_SOR, default_params  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402
from oracle.oracle import interp_cube, run_oracle  # noqa: E402


def floor_ratios(real_size: int, ghost: int, npatch: int, seed: int) -> dict:
    dt = np.float32 if real_size == 4 else np.float64
    d = make_patches(npatch, ghost, seed=seed, dtype=dt, fluid=False)
    p = default_params(real_size, ghost, GPG_SOR, gra_acc=0, gra_ghost=0, init_mode=GPG_INIT_ZERO,
                       sor_min_iter=10, sor_max_iter=400)
    _, _, it, res = run_oracle(p, d["rho"], d["pot_in"])
    scale = np.array([np.abs(interp_cube(c, ghost, 4)[1:-1, 1:-1, 1:-1].astype(np.float64)).sum()
                      for c in d["pot_in"]])
    q = res / scale
    return {"p50": float(np.median(q)), "p90": float(np.percentile(q, 90)), "max": float(q.max()),
            "sweeps_max": int(it.max()), "tol": float(f"{2 * np.percentile(q, 90):.2g}")}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--npatch", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=11)
    a = ap.parse_args(argv)
    out = {f"{'f32' if rs == 4 else 'f64'}_g{g}": floor_ratios(rs, g, a.npatch, a.seed)
           for rs in (4, 8) for g in range(1, 6)}
    print(json.dumps(out, indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
