"""Build recipes for the oracle (test infrastructure only).

* ``build_oracle()``  compiles the C restatement ``oracle/gpg_oracle.c`` into
  ``oracle/liboracle.so`` (gcc -O3 -fopenmp, baseline x86-64, no FMA
  contraction, so that float results are bit-identical to the reference's
  own CPU code built the same way).
* ``build_ref()``     compiles the reference's unmodified CPU solver sources
  (CPU_Solver/*.cpp and Auxiliary/*.cpp, read in place from the reference
  tree) plus ``oracle/ref_driver.cpp`` into one shared object per
  compile-time configuration, ``oracle/_ref/libref_<scheme>_g<g>_G<G>_<prec>.so``.
  The reference fixes every array size with macros (Makefile:13-85), hence one
  object per (POT_GHOST_SIZE, GRA_GHOST_SIZE, precision, scheme).  The flags
  follow the GNU branch of the reference Makefile (Makefile:171: -O3 -fopenmp)
  with the macro set of Makefile:13-85; GPU_ARCH only has to name a known
  architecture for Header/Macro.h:27-31 and has no effect on CPU code.

Run ``python oracle/build.py [--ref /path/to/reference]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
REF_OUT = os.path.join(HERE, "_ref")
DEFAULT_REF = "/root/reference"

REF_SOURCES = [
    "CPU_Solver/CPU_PoissonGravitySolver.cpp",
    "CPU_Solver/CPU_PoissonSolver_SOR.cpp",
    "CPU_Solver/CPU_PoissonSolver_MG.cpp",
    "CPU_Solver/CPU_GravitySolver.cpp",
    "Auxiliary/Aux_Message.cpp",
    "Auxiliary/Aux_Error.cpp",
]


def ref_configs():
    for scheme in ("sor", "mg"):
        for g in range(1, 6):
            for G in (1, 2):
                if G > g:
                    continue
                for prec in ("f32", "f64"):
                    yield scheme, g, G, prec


def ref_lib_name(scheme: str, g: int, G: int, prec: str) -> str:
    return f"libref_{scheme}_g{g}_G{G}_{prec}.so"


def ref_lib_path(scheme: str, g: int, G: int, prec: str) -> str:
    return os.path.join(REF_OUT, ref_lib_name(scheme, g, G, prec))


def reference_macros(scheme: str, g: int, G: int, prec: str) -> list[str]:
    d = ["-DGRAVITY", "-DGPU", "-DOPENMP", f"-DPOT_SCHEME={scheme.upper()}",
         "-DGPU_ARCH=PASCAL", "-DPATCH_SIZE=8", "-DNEWTON_G=1.e-5",
         f"-DPOT_GHOST_SIZE={g}", f"-DGRA_GHOST_SIZE={G}", "-DDH=1.0", "-DDT=1.e-2"]
    if prec == "f64":
        d.append("-DFLOAT8")
    return d


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stderr[-4000:])


def build_oracle(verbose: bool = False) -> str:
    out = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "gpg_oracle.c")
    deps = [src, os.path.join(HERE, "gpg_oracle_body.h"), os.path.join(REPO, "include", "gpg.h")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = ["gcc", "-O3", "-std=c99", "-fopenmp", "-fPIC", "-shared", "-Wall", "-Wno-unknown-pragmas",
           "-o", out, src, "-lm"]
    if verbose:
        print(" ".join(cmd))
    _run(cmd)
    return out


def _build_one(ref_root: str, scheme: str, g: int, G: int, prec: str) -> str:
    out = ref_lib_path(scheme, g, G, prec)
    srcs = [os.path.join(ref_root, s) for s in REF_SOURCES] + [os.path.join(HERE, "ref_driver.cpp")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(s) for s in srcs):
        return out
    cmd = (["g++", "-O3", "-fopenmp", "-fPIC", "-shared", "-fvisibility=hidden", "-w",
            "-Wl,-Bsymbolic", "-I" + os.path.join(ref_root, "Header")]
           + reference_macros(scheme, g, G, prec) + ["-o", out] + srcs)
    _run(cmd)
    return out


def build_ref(ref_root: str = DEFAULT_REF, jobs: int | None = None) -> list[str]:
    """Compile every reference configuration; returns the built paths.
    Does nothing (returns []) when the reference tree is absent."""
    if not os.path.isdir(os.path.join(ref_root, "CPU_Solver")):
        return []
    os.makedirs(REF_OUT, exist_ok=True)
    jobs = jobs or os.cpu_count() or 4
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_build_one, ref_root, *c) for c in ref_configs()]
        return [f.result() for f in futs]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--ref", default=DEFAULT_REF)
    ap.add_argument("--no-ref", action="store_true")
    a = ap.parse_args(argv)
    print(build_oracle(verbose=True))
    if not a.no_ref:
        libs = build_ref(a.ref)
        print(f"{len(libs)} reference configurations in {REF_OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
