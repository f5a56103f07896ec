"""Autotuner for the SOR kernel variants (patches per CTA x pass order).

For every (precision, ghost size) it times each variant of libgpg's SOR
kernel on a seeded batch with the reference parameters (CUDA events on the
launching stream, warm-up first), checks that all variants return the same
bits, and writes the fastest choice to lib/sor_tune.txt beside libgpg.so,
which the library reads on first use (include/gpg.h, gpg_set_sor_variant).

    python gpu_testbed_poisson-gravity_b200/autotune.py [--npatch 4096] [--json out.json]

With --sizes (a comma-separated list of patch counts) it only reports: every
variant's time at each size, for choosing the small-launch table (kSorSmall
in csrc/gpg_api.cu); --gravity adds the fused gravity update to each launch.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from gpg.abi import GPG_SOR, default_params  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402
from gpg.lib import GpgError, check, library, solve_device  # noqa: E402


def variants():
    """(variant, patches per CTA, phased pass, lanes per pair column, rows per lane)."""
    lib = library()
    out = []
    for v in range(lib.gpg_sor_variant_count()):
        ppc, ph, z, y = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib.gpg_sor_variant_info(v, C.byref(ppc), C.byref(ph)))
        check(lib.gpg_sor_variant_layout(v, C.byref(z), C.byref(y)))
        out.append((v, ppc.value, bool(ph.value), z.value, y.value))
    return out


def time_variant(torch, p, t, reps=5, warm=2):
    flu = t.get("flu")
    for _ in range(warm):
        solve_device(p, t["rho"], t["pot_in"], pot_out=t["pot_out"], flu=flu, iters=t["iters"], resid=t["resid"])
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        solve_device(p, t["rho"], t["pot_in"], pot_out=t["pot_out"], flu=flu, iters=t["iters"], resid=t["resid"])
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def tune(npatch=4096, precisions=(4, 8), ghosts=(1, 2, 3, 4, 5)):
    import torch
    lib = library()
    dev = torch.device("cuda:0")
    report = {}
    for rs in precisions:
        for g in ghosts:
            p = default_params(rs, g, GPG_SOR, gra_acc=0)
            dt = np.float32 if rs == 4 else np.float64
            d = make_patches(npatch, g, seed=4242 + g, dtype=dt, fluid=False)
            tdt = torch.float32 if rs == 4 else torch.float64
            gn = 8 + 2 * p.gra_ghost
            t = dict(rho=torch.from_numpy(d["rho"]).to(dev), pot_in=torch.from_numpy(d["pot_in"]).to(dev),
                     pot_out=torch.empty((npatch, gn, gn, gn), dtype=tdt, device=dev),
                     iters=torch.empty(npatch, dtype=torch.int32, device=dev),
                     resid=torch.empty(npatch, dtype=torch.float64, device=dev))
            cur = C.c_int()
            check(lib.gpg_get_sor_variant(rs, g, C.byref(cur)))
            times, ref = {}, None
            for v, ppc, ph, z, y in variants():
                check(lib.gpg_set_sor_variant(rs, g, v))
                try:
                    ms = time_variant(torch, p, t)
                except GpgError as e:
                    times[v] = None
                    continue
                out = t["pot_out"].cpu().numpy()
                if ref is None:
                    ref = out
                elif not np.array_equal(out, ref):
                    raise RuntimeError(f"variant {v} changed the result (f{8 * rs} g{g})")
                times[v] = ms
            ok = {v: ms for v, ms in times.items() if ms is not None}
            best = min(ok, key=ok.get)
            check(lib.gpg_set_sor_variant(rs, g, best))
            report[f"f{8 * rs}_g{g}"] = {"best": best, "default": cur.value, "ms": times,
                                         "shape": {v: {"patches_per_cta": ppc, "phased": ph, "lanes_per_column": z,
                                                       "rows_per_lane": y} for v, ppc, ph, z, y in variants()}}
            print(f"f{8 * rs} g{g}: " + "  ".join(f"v{v}={'-' if ms is None else f'{ms:.3f}'}"
                                                 for v, ms in times.items()) + f"  -> v{best}", flush=True)
    return report


def sizes_report(sizes, gravity: bool, precisions=(4, 8), ghosts=(1, 2, 3, 4, 5), reps=50):
    """Every variant's launch time (microseconds, CUDA events, mean of reps
    after 5 warm-up launches) at each patch count; the library's own choice
    is restored afterwards (gpg_set_sor_variant -1)."""
    import torch
    lib = library()
    dev = torch.device("cuda:0")
    out = []
    for rs in precisions:
        for g in ghosts:
            for n in sizes:
                dt = np.float32 if rs == 4 else np.float64
                d = make_patches(n, g, seed=21, dtype=dt, fluid=gravity)
                tdt = torch.float32 if rs == 4 else torch.float64
                t = dict(rho=torch.from_numpy(d["rho"]).to(dev), pot_in=torch.from_numpy(d["pot_in"]).to(dev),
                         pot_out=torch.empty((n, 10, 10, 10), dtype=tdt, device=dev),
                         iters=torch.empty(n, dtype=torch.int32, device=dev),
                         resid=torch.empty(n, dtype=torch.float64, device=dev))
                if gravity:
                    t["flu"] = torch.from_numpy(d["flu"]).to(dev)
                p = default_params(rs, g, GPG_SOR, gra_acc=int(gravity))
                row = {}
                for v, *_ in variants():
                    check(lib.gpg_set_sor_variant(rs, g, v))
                    try:
                        row[v] = round(1e3 * time_variant(torch, p, t, reps=reps, warm=5), 2)
                    except GpgError:
                        row[v] = None
                check(lib.gpg_set_sor_variant(rs, g, -1))
                rec = {"precision": f"f{8 * rs}", "ghost": g, "npatch": n, "us": row}
                out.append(rec)
                print(json.dumps(rec), flush=True)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--npatch", type=int, default=4096)
    ap.add_argument("--json", default=None)
    ap.add_argument("--no-write", action="store_true")
    ap.add_argument("--sizes", default=None, help="report only: variant times at these patch counts")
    ap.add_argument("--gravity", action="store_true", help="with --sizes: fused gravity update in each launch")
    a = ap.parse_args(argv)
    if a.sizes:
        rep = sizes_report([int(x) for x in a.sizes.split(",")], a.gravity)
        if a.json:
            with open(a.json, "w") as f:
                json.dump(rep, f, indent=1)
        return 0
    rep = tune(a.npatch)
    if not a.no_write:
        path = os.path.join(HERE, "lib", "sor_tune.txt")
        with open(path, "w") as f:
            for k, r in rep.items():
                prec, g = k.split("_g")
                f.write(f"{prec} {g} {r['best']}\n")
        print("wrote", path)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rep, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
