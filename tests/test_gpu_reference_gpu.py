"""The reference's own GPU path, recompiled for sm_100a, beside this library
on the same CUAPI calls and inputs (needs a B200).

oracle/build.py (build_ref_gpu) compiles the reference's GPU_API/ and
GPU_Solver/ sources unmodified for sm_100a, with one timing driver
(oracle/cuapi_bench.cpp) that also links on this library's CUAPI shim.  Both
executables run the reference's call sequence (CUAPI_MemAllocate,
CUAPI_Asyn_PoissonGravitySolver, CUAPI_Synchronize) on identical input bytes.
The check follows the reference's own accuracy test (Main.cpp:1007-1054:
error per element against the CPU solver, thresholds Makefile:56-70), with
this library's output, bit-identical to the reference CPU solver, in the
CPU's place.  Two departures: errors are taken relative to the largest
magnitude of the field (potential, or fluid component) in the patch, because
these inputs' potential and momenta pass through zero, where an error
relative to each element is unbounded (the reference's own inputs,
Main.cpp:524-580, keep the potential away from zero); and the potential
bound is twice the Makefile's, because the reference GPU solver tests its
residual every second sweep (SOR_MOD_REDUCTION 2, Header/CUPOT.h:119) and so
may stop one sweep away from the CPU solver.
Each run prints one ``REFGPU {json}`` line with both builds' per-call wall
times (host clock around the call and the synchronize: pinned H2D, kernels
and D2H, as Main.cpp:195-208 times it).
"""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import build as ob
from oracle.cuapi_bench_inputs import CASES, case_id, driver_args, write_inputs

pytestmark = pytest.mark.gpu


def _scaled(a, b):
    """|b - a| per element over the largest |a| of its patch and component
    (arrays [patch][component][cells])."""
    a, b = a.astype(np.float64), b.astype(np.float64)
    return np.abs(b - a) / np.abs(a).max(axis=2, keepdims=True)


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_reference_gpu_path_agrees_on_b200(case, tmp_path):
    scheme, g, G, prec, npatch, p5 = case
    exe_ref, exe_gpg = ob.cuapi_bench_exe("ref", *case[:4]), ob.cuapi_bench_exe("gpg", *case[:4])
    if not (os.path.exists(exe_ref) and os.path.exists(exe_gpg)):
        pytest.skip("reference GPU build absent (oracle/build.py build_ref_gpu needs the reference tree)")
    dt = np.float64 if prec == "f64" else np.float32
    fin = str(tmp_path / "in.bin")
    write_inputs(case, fin)
    res = {}
    outs = {}
    try:
        for kind, exe in (("reference_gpu_sm100a", exe_ref), ("this_library", exe_gpg)):
            fout = str(tmp_path / f"out_{kind}.bin")
            r = subprocess.run([exe] + driver_args(case, fin, fout), capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, (kind, r.stdout[-2000:], r.stderr[-2000:])
            res[kind] = json.loads(r.stdout.strip().splitlines()[-1])
            raw = np.fromfile(fout, dtype=dt)
            os.remove(fout)
            gn = 8 + 2 * G
            outs[kind] = (raw[:npatch * gn ** 3], raw[npatch * gn ** 3:])
    finally:
        os.remove(fin)  # up to 275 MB per case
    poi, gra = (float(x) for x in ob.MAXERR[(scheme, prec)])
    mine, ref = outs["this_library"], outs["reference_gpu_sm100a"]
    pot_err = _scaled(mine[0].reshape(npatch, 1, -1), ref[0].reshape(npatch, 1, -1))
    flu_err = _scaled(mine[1].reshape(npatch, 5, -1), ref[1].reshape(npatch, 5, -1))
    line = {"case": case_id(case), "npatch": npatch, "p5": p5,
            "pot_err_max": float(pot_err.max()), "pot_err_p999": float(np.percentile(pot_err, 99.9)),
            "pot_patches_differing": int((pot_err.reshape(npatch, -1).max(1) > 0).sum()),
            "flu_err_max": float(flu_err.max()), **res}
    print("REFGPU " + json.dumps(line))
    assert np.isfinite(outs["reference_gpu_sm100a"][0]).all()
    assert (pot_err <= 2 * poi).all(), line
    assert (flu_err <= gra).all(), line
