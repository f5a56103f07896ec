"""Build libgpg.so (the CUDA library behind include/gpg.h) for sm_100a, in-tree.

    python gpu_testbed_poisson-gravity_b200/build.py [--force]

Output: gpu_testbed_poisson-gravity_b200/lib/libgpg.so; the ptxas resource
report (registers, spills, shared memory per kernel) goes to
_build/ptxas_libgpg.log at the repository root.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgpg.so")
BUILD_LOG_DIR = os.path.join(REPO, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden", "-Xptxas", "-v"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
            + [os.path.join(REPO, "include", "gpg.h")])


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def _compile(src: str, obj: str):
    cmd = [nvcc()] + ARCH + NVCC_FLAGS + ["-c", "-o", obj, src]
    return cmd, subprocess.run(cmd, capture_output=True, text=True)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every csrc/*.cu to an object (in parallel), then link libgpg.so."""
    if not force and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD_LOG_DIR, exist_ok=True)
    objs = [os.path.join(BUILD_LOG_DIR, os.path.basename(s)[:-3] + ".o") for s in sources()]
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(objs)) as ex:
        results = list(ex.map(_compile, sources(), objs))
    log = ""
    for cmd, r in results:
        if verbose:
            print(" ".join(cmd))
        log += r.stdout + r.stderr
    with open(os.path.join(BUILD_LOG_DIR, "ptxas_libgpg.log"), "w") as f:
        f.write(log)
    for cmd, r in results:
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    link = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr[-6000:])
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
