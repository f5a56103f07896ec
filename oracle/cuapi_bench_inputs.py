"""Inputs and arguments of the CUAPI timing driver (oracle/cuapi_bench.cpp).
TEST INFRASTRUCTURE ONLY (tests/test_gpu_reference_gpu.py and the profiling
recipe that times the reference's GPU build beside this library).

    python oracle/cuapi_bench_inputs.py sor 5 1 f64 /tmp/in.bin [--reps 3 --warm 1]

writes the case's input file (rho, pot_in, flu in the reference's layouts,
seeded power-law patches of gpg.inputs) and prints the driver's arguments.
Parameters are the reference's defaults (Main.cpp:1142-1223): SOR Min_Iter
10, Max_Iter 60 / 100, Omega per ghost size; MG 10 / 20 cycles, 3 + 3
smoothing sweeps, tolerance 1e-6 / 1e-15; CQUAD interpolation.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "gpu_testbed_poisson-gravity_b200"))
sys.path.insert(0, os.path.dirname(HERE))

from gpg.abi import SOR_OMEGA  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402

from oracle.build import REF_GPU_CONFIGS  # noqa: E402

# (scheme, ghost, GRA ghost, precision, patches, P5 gradient): SOR on the
# 4096-patch batches of the plain-SOR workload, MG on 16384 patches with the
# 5-point gradient, and the reference README's own GPU benchmark sizes
# (README.txt:114-150: 256 patches at ghost 1 and 3)
CASES = ([c + ((16384, 1) if c[0] == "mg" else (4096, 0)) for c in REF_GPU_CONFIGS]
         + [("sor", 1, 1, "f32", 256, 0), ("sor", 3, 1, "f32", 256, 0)])


def case_id(case) -> str:
    return "{}_g{}_G{}_{}_{}".format(*case[:5])


def write_inputs(case, path: str) -> None:
    scheme, g, G, prec, npatch, _ = case
    dt = np.float64 if prec == "f64" else np.float32
    d = make_patches(npatch, g, seed=61 + g, gra_ghost=G, dtype=dt, fluid=True)
    with open(path, "wb") as f:
        for k in ("rho", "pot_in", "flu"):
            f.write(np.ascontiguousarray(d[k], dtype=dt).tobytes())


def driver_args(case, fin: str, fout: str, reps: int = 10, warm: int = 2) -> list[str]:
    scheme, g, G, prec, npatch, p5 = case
    f64 = prec == "f64"
    return ["--in", fin, "--out", fout, "--npg", str(npatch // 8), "--nstream", "4", "--reps", str(reps),
            "--warm", str(warm), "--min-iter", "10", "--max-iter", "100" if f64 else "60",
            "--omega", repr(SOR_OMEGA[g]), "--mg-max-iter", "20" if f64 else "10", "--mg-npre", "3",
            "--mg-npost", "3", "--mg-tol", "1e-15" if f64 else "1e-6", "--int-scheme", "4", "--p5", str(p5)]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("scheme", choices=["sor", "mg"])
    ap.add_argument("ghost", type=int)
    ap.add_argument("gra_ghost", type=int)
    ap.add_argument("prec", choices=["f32", "f64"])
    ap.add_argument("input_file")
    ap.add_argument("--npatch", type=int, default=None, help="patches (default: the case's first size)")
    ap.add_argument("--out", default=os.devnull)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warm", type=int, default=2)
    a = ap.parse_args(argv)
    found = [c for c in CASES if c[:4] == (a.scheme, a.ghost, a.gra_ghost, a.prec)
             and (a.npatch is None or c[4] == a.npatch)]
    if not found:
        ap.error(f"no such case; cases: {[case_id(c) for c in CASES]}")
    case = found[0]
    write_inputs(case, a.input_file)
    print(" ".join(driver_args(case, a.input_file, a.out, a.reps, a.warm)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
