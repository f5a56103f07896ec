"""Generate the golden vectors in tests/golden/ from the reference's own CPU code.

Each fixture runs CPU_PoissonGravitySolver of the reference (compiled from its
unmodified sources by oracle/build.py into oracle/_ref/) on one patch group of
8 seeded patches (gpg.inputs.make_patches) and stores:

* ``iters``     [8]      per-patch SOR iteration counts the reference printed
* ``pot_out``   [2,...]  potential of patches 0 and 5
* ``flu``       [1,...]  fluid of patch 0 after the gravity update
* ``input_sha`` sha256 of the generated input bytes (detects generator drift)

Usage:  python tests/golden/make_golden.py   (needs oracle/_ref/, i.e. the
reference sources present when oracle/build.py ran).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gpu_testbed_poisson-gravity_b200"))

from gpg.abi import GPG_MG, GPG_SOR, default_params  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402

NPATCH = 8
KEEP_POT = (0, 5)


def cases():
    """(name, scheme, real_size, ghost, gra_ghost, int_scheme, p5)."""
    for scheme, sname in ((GPG_SOR, "sor"), (GPG_MG, "mg")):
        for rs in (4, 8):
            for g in range(1, 6):
                yield f"{sname}_g{g}_G1_cquad_{rs * 8}", scheme, rs, g, 1, 4, 0
            yield f"{sname}_g3_G2_cquad_p5_{rs * 8}", scheme, rs, 3, 2, 4, 1
    for rs in (4, 8):
        for g in (1, 4):
            yield f"sor_g{g}_G1_quad_{rs * 8}", GPG_SOR, rs, g, 1, 5, 0
        yield f"mg_g2_G1_quad_{rs * 8}", GPG_MG, rs, 2, 1, 5, 0


def case_inputs(name, rs, g, G):
    seed = int.from_bytes(hashlib.sha256(name.encode()).digest()[:4], "little")
    dt = np.float32 if rs == 4 else np.float64
    return make_patches(NPATCH, g, seed=seed, gra_ghost=G, dtype=dt), seed


def input_sha(d) -> str:
    h = hashlib.sha256()
    for k in ("rho", "pot_in", "flu"):
        h.update(np.ascontiguousarray(d[k]).tobytes())
    return h.hexdigest()


def main() -> int:
    from oracle.oracle import run_reference
    index = {}
    for name, scheme, rs, g, G, isch, p5 in cases():
        d, seed = case_inputs(name, rs, g, G)
        p = default_params(rs, g, scheme, gra_ghost=G, int_scheme=isch, p5_gradient=p5)
        pot, flu, iters = run_reference(p, d["rho"], d["pot_in"].copy(), flu=d["flu"].copy(),
                                        nthreads=1)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), iters=iters,
                            pot_out=pot[list(KEEP_POT)], flu=flu[:1],
                            input_sha=np.array(input_sha(d)))
        index[name] = {"scheme": scheme, "real_size": rs, "ghost": g, "gra_ghost": G,
                       "int_scheme": isch, "p5_gradient": p5, "seed": seed,
                       "iters": iters.tolist()}
        print(name, iters.tolist())
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump({"npatch": NPATCH, "keep_pot": list(KEEP_POT), "cases": index}, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
