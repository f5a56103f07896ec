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

* ``build_ref_gpu()`` compiles the reference's GPU_API/ and GPU_Solver/
  sources (the CUDA_FILE list of Makefile:164-167, read in place) for sm_100a
  with nvcc, plus ``oracle/cuapi_bench.cpp``, into one timing executable per
  configuration, ``oracle/_ref/cuapi_bench_ref_<cfg>``; ``build_cuapi_bench()``
  links the same driver on this library's CUAPI shim and libgpg
  (``oracle/_ref/cuapi_bench_gpg_<cfg>``), so both run the same calls on the
  same inputs.  The nvcc flags follow Makefile:195-206 (-O3, -Xptxas -dlcm=ca
  for the CUPOT files) with the reference's macro set; ``ref_gpu_compat.h`` is
  force-included for the one pre-Volta intrinsic.

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
# the reference tree: $GPG_REFERENCE_ROOT, else a checkout named "reference"
# beside this repository; absent trees are skipped by build_ref/build_integration
DEFAULT_REF = os.environ.get("GPG_REFERENCE_ROOT") or os.path.join(os.path.dirname(REPO), "reference")

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


# ---------------------------------------------------------------------------
# integration: the reference's own driver (Main.cpp) relinked on libgpg
# ---------------------------------------------------------------------------
PKG = os.path.join(REPO, "gpu_testbed_poisson-gravity_b200")
SHIM = os.path.join(PKG, "csrc", "cuapi", "cuapi_compat.cpp")
LIBGPG_DIR = os.path.join(PKG, "lib")
# (scheme, POT_GHOST_SIZE, GRA_GHOST_SIZE, precision)
INTEGRATION_CONFIGS = [("sor", 1, 1, "f32"), ("sor", 5, 1, "f32"), ("sor", 3, 2, "f64"),
                       ("mg", 3, 2, "f32"), ("mg", 2, 1, "f64")]
# DataCompare thresholds of the reference Makefile (Makefile:56-70)
MAXERR = {("sor", "f32"): ("5.e-6", "8.e-6"), ("sor", "f64"): ("3.e-15", "1.e-14"),
          ("mg", "f32"): ("4.e-5", "4.e-5"), ("mg", "f64"): ("3.e-14", "3.e-14")}


def integration_exe(scheme, g, G, prec):
    return os.path.join(REF_OUT, f"main_{scheme}_g{g}_G{G}_{prec}")


def _build_integration_one(ref_root, scheme, g, G, prec):
    out = integration_exe(scheme, g, G, prec)
    srcs = [os.path.join(ref_root, "Main.cpp")] + [os.path.join(ref_root, s) for s in REF_SOURCES]
    deps = srcs + [SHIM, os.path.join(REPO, "include", "gpg_cuapi.h"), os.path.join(LIBGPG_DIR, "libgpg.so")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    poi, gra = MAXERR[(scheme, prec)]
    macros = reference_macros(scheme, g, G, prec) + [
        "-DCPULOAD=420000", "-DINIT_WIDTH=410.0", "-DINIT_INDEX=2.1", "-DINIT_OFFSET=0.09",
        f"-DPOI_MAXERR={poi}", f"-DGRA_MAXERR={gra}"]
    shim_macros = [m for m in macros if not m.startswith("-DPOT_SCHEME")] + [
        f"-DPOT_SCHEME={1 if scheme == 'sor' else 2}"]
    shim_obj = out + "_shim.o"
    _run(["g++", "-O2", "-fPIC", "-c", "-o", shim_obj, SHIM] + shim_macros)
    _run(["g++", "-O3", "-fopenmp", "-w", "-I" + os.path.join(ref_root, "Header")] + macros
         + ["-o", out] + srcs + [shim_obj, "-L" + LIBGPG_DIR, "-lgpg",
                                 "-Wl,-rpath,$ORIGIN/../../gpu_testbed_poisson-gravity_b200/lib"])
    return out


def build_integration(ref_root: str = DEFAULT_REF) -> list[str]:
    """Link the reference's unmodified Main.cpp + CPU solvers against the CUAPI
    shim and libgpg (one executable per configuration, in oracle/_ref/)."""
    if not os.path.isdir(os.path.join(ref_root, "CPU_Solver")):
        return []
    if not os.path.exists(os.path.join(LIBGPG_DIR, "libgpg.so")):
        raise RuntimeError("build libgpg.so first")
    os.makedirs(REF_OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = [ex.submit(_build_integration_one, ref_root, *c) for c in INTEGRATION_CONFIGS]
        return [f.result() for f in futs]


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


# ---------------------------------------------------------------------------
# the reference's own GPU path recompiled for sm_100a, and the same timing
# driver on this library (test infrastructure: tests/test_gpu_reference_gpu.py)
# ---------------------------------------------------------------------------
REF_GPU_API = ["CUAPI_Set_Diagnose_Device.cu", "CUAPI_Synchronize.cu", "CUAPI_Asyn_PoissonGravitySolver.cu",
               "CUAPI_MemAllocate_PoissonGravity.cu", "CUAPI_MemFree_PoissonGravity.cu"]
REF_GPU_SOLVER = ["CUPOT_PoissonSolver_SOR_10to14cube.cu", "CUPOT_PoissonSolver_SOR_16to18cube.cu",
                  "CUPOT_GravitySolver.cu", "CUPOT_PoissonSolver_MG.cu"]
BENCH_DRIVER = os.path.join(HERE, "cuapi_bench.cpp")
GPU_COMPAT = os.path.join(HERE, "ref_gpu_compat.h")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_LIB = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")
# (scheme, POT_GHOST_SIZE, GRA_GHOST_SIZE, precision): SOR at every ghost size
# and precision, MG in FP32 up to ghost 4 (its FP64 and 18^3 forms take
# per-block device malloc, CUPOT_PoissonSolver_MG.cu:136-145,186-187, which
# these comparisons leave out)
REF_GPU_CONFIGS = ([("sor", g, 1, p) for g in range(1, 6) for p in ("f32", "f64")]
                   + [("sor", 3, 2, "f32"), ("mg", 3, 2, "f32")])


def cuapi_bench_exe(kind: str, scheme: str, g: int, G: int, prec: str) -> str:
    return os.path.join(REF_OUT, f"cuapi_bench_{kind}_{scheme}_g{g}_G{G}_{prec}")


def _bench_macros(scheme, g, G, prec):
    poi, gra = MAXERR[(scheme, prec)]
    return reference_macros(scheme, g, G, prec) + [
        "-DCPULOAD=420000", "-DINIT_WIDTH=410.0", "-DINIT_INDEX=2.1", "-DINIT_OFFSET=0.09",
        f"-DPOI_MAXERR={poi}", f"-DGRA_MAXERR={gra}"]


def _build_ref_gpu_one(ref_root, scheme, g, G, prec):
    out = cuapi_bench_exe("ref", scheme, g, G, prec)
    cus = ([os.path.join(ref_root, "GPU_API", f) for f in REF_GPU_API]
           + [os.path.join(ref_root, "GPU_Solver", f) for f in REF_GPU_SOLVER])
    hdrs = [os.path.join(ref_root, "Header", h) for h in os.listdir(os.path.join(ref_root, "Header"))]
    incl = [os.path.join(ref_root, "GPU_Solver", f) for f in os.listdir(os.path.join(ref_root, "GPU_Solver"))]
    aux = [os.path.join(ref_root, s) for s in REF_SOURCES if s.startswith("Auxiliary/")]
    deps = cus + hdrs + incl + aux + [BENCH_DRIVER, GPU_COMPAT]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    macros = _bench_macros(scheme, g, G, prec)
    inc = ["-I" + os.path.join(ref_root, "Header"), "-I" + os.path.join(ref_root, "GPU_Solver")]
    objs = []
    for src in cus:
        obj = out + "_" + os.path.basename(src).replace(".cu", ".o")
        extra = ["-Xptxas", "-dlcm=ca"] if os.path.basename(src).startswith("CUPOT_") else []
        _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-w", "-include", GPU_COMPAT]
             + extra + inc + macros + ["-c", "-o", obj, src])
        objs.append(obj)
    _run(["g++", "-O3", "-w", "-DREF_GPU", "-I" + os.path.join(CUDA_LIB, "..", "include")] + inc + macros
         + ["-o", out, BENCH_DRIVER] + aux + objs + ["-L" + CUDA_LIB, "-lcudart", "-Wl,-rpath," + CUDA_LIB])
    for o in objs:
        os.remove(o)
    return out


def _build_cuapi_bench_one(ref_root, scheme, g, G, prec):
    out = cuapi_bench_exe("gpg", scheme, g, G, prec)
    aux = [os.path.join(ref_root, s) for s in REF_SOURCES if s.startswith("Auxiliary/")]
    deps = aux + [BENCH_DRIVER, SHIM, os.path.join(REPO, "include", "gpg_cuapi.h"),
                  os.path.join(LIBGPG_DIR, "libgpg.so")]
    if os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    macros = _bench_macros(scheme, g, G, prec)
    shim_macros = [m for m in macros if not m.startswith("-DPOT_SCHEME")] + [
        f"-DPOT_SCHEME={1 if scheme == 'sor' else 2}"]
    shim_obj = out + "_shim.o"
    _run(["g++", "-O2", "-fPIC", "-c", "-o", shim_obj, SHIM] + shim_macros)
    _run(["g++", "-O3", "-w", "-I" + os.path.join(ref_root, "Header")] + macros
         + ["-o", out, BENCH_DRIVER] + aux + [shim_obj, "-L" + LIBGPG_DIR, "-lgpg",
                                              "-Wl,-rpath,$ORIGIN/../../gpu_testbed_poisson-gravity_b200/lib"])
    os.remove(shim_obj)
    return out


def build_ref_gpu(ref_root: str = DEFAULT_REF) -> list[str]:
    """Both timing executables of every REF_GPU_CONFIGS entry (reference GPU
    path for sm_100a; this library through its CUAPI shim)."""
    if not os.path.isdir(os.path.join(ref_root, "GPU_Solver")):
        return []
    if not os.path.exists(os.path.join(LIBGPG_DIR, "libgpg.so")):
        raise RuntimeError("build libgpg.so first")
    os.makedirs(REF_OUT, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        futs = [ex.submit(_build_ref_gpu_one, ref_root, *c) for c in REF_GPU_CONFIGS]
        futs += [ex.submit(_build_cuapi_bench_one, ref_root, *c) for c in REF_GPU_CONFIGS]
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
        exes = build_integration(a.ref)
        print(f"{len(exes)} integration executables in {REF_OUT}")
        exes = build_ref_gpu(a.ref)
        print(f"{len(exes)} CUAPI timing executables in {REF_OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
