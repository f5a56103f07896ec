#!/usr/bin/env python
"""Benchmark of the per-patch Poisson(-gravity) hot path on B200.

Workload (one "step"): plain red-black SOR with the reference's parameters and
convergence rule (interpolated start, stop when the L1 residual grows after
Min_Iter = 10, Max_Iter 60 / 100) over ghost sizes 2, 3, 4, 5 with 4096
patches each, in FP32 and in FP64 -- 8 batches, 32768 patches per step per GPU.
Inputs: seeded power-law density rho = (r/8)^-2 (1 + 0.05 N(0,1)) in a 16^3-
patch box and the matching analytic coarse potential (gpg.inputs).

Reported (one JSON line from rank 0):
  value      patches/s over the whole job, inputs resident in HBM (device timing,
             CUDA events on the timing stream, max over ranks); the 8 batches
             run on their own streams, forked from and joined to the timing
             stream; value_one_stream times the same steps one launch at a time,
             and that pass gives the per-kernel times (per_batch_ms, roofline)
  e2e        the same through the reference-shaped host API (pinned host
             buffers, H2D + solve + D2H per step; host clock around a full sync;
             batches pipelined across steps, lockstep_value with a full sync
             after every step)
  roofline   dominant kernel: compulsory HBM bytes per launch / mean launch time;
             roofline.onchip: its shared-memory wavefronts per launch (measured
             sweeps x cell updates x the shared accesses per update of the
             kernel's layout) / launch time, against one wavefront per cycle
             per SM at the sampled clock
  cpu_baseline  the reference's own CPU code (oracle/_ref, all host threads) on
             a bounded sample of the same workload
`--impl reference` runs only the reference CPU path (rank 0) and prints its line.
Multi-GPU (torchrun): every rank solves its own 32768 patches (weak scaling, no
collective in the solve); only the timing max goes through the process group.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "gpu_testbed_poisson-gravity_b200"))

from gpg.abi import GPG_SOR, default_params, patch_sizes  # noqa: E402
from gpg.inputs import make_patches  # noqa: E402

METRIC = "patches/s to fixed residual on 1 B200: learned-init+SOR vs plain SOR"
WORKLOAD = ("plain SOR, reference rule (interpolated start, stop on residual growth, Min 10 / Max 60|100), "
            "ghost 2-5 x 4096 patches, FP32+FP64, Poisson only")


def bench_config() -> dict:
    """The workload of one step on one GPU; identical in both arms."""
    return {"workload": WORKLOAD, "patches_per_gpu_per_step": NPATCH * len(GHOSTS) * len(PRECS)}
GHOSTS = (2, 3, 4, 5)
PRECS = (4, 8)
NPATCH = 4096
L2_BYTES = 126 * 2 ** 20


def workload(rank: int, only=None):
    """[(params, inputs)] for the 8 batches of one step on this rank
    (`only`: keep the batches named like f64_g5)."""
    out = []
    for rs in PRECS:
        for g in GHOSTS:
            if only and f"f{8 * rs}_g{g}" not in only:
                continue
            p = default_params(rs, g, GPG_SOR, gra_acc=0)
            dt = np.float32 if rs == 4 else np.float64
            d = make_patches(NPATCH, g, seed=1000 * (rank + 1) + g, dtype=dt, fluid=False)
            out.append((p, d))
    return out


def compulsory_bytes(p) -> int:
    s = patch_sizes(p)
    return (s["rho"] + s["pot_in"] + s["pot_out"]) * p.real_size


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"gpg_bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once samples flow (nvidia-smi takes a
            # fraction of a second to start), so that it is covered
            t0 = time.time()
            while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
                time.sleep(0.02)
            time.sleep(0.1)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return None
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                except ValueError:
                    continue
        if not rows:
            return None
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for _, _, flags in rows for n, fl in zip(names, flags) if fl.lower() == "active"})
        sm = sorted(r[0] for r in rows)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(r[1] for r in rows), "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference CPU path
# ---------------------------------------------------------------------------
_HOST_THREADS = 0


def host_threads() -> int:
    """All OpenMP threads of the host, read once before any run narrows them
    (the reference's CPU objects share one OpenMP runtime: a one-core run
    would otherwise leave every later call on one thread)."""
    global _HOST_THREADS
    if not _HOST_THREADS:
        from oracle.oracle import oracle_lib
        _HOST_THREADS = max(1, oracle_lib().oracle_max_threads())
    return _HOST_THREADS


def reference_cpu(batches, budget_s: float = 20.0, nthreads: int = 0, keep: dict | None = None):
    """Time the reference's CPU_PoissonGravitySolver (oracle/_ref; the C port
    of oracle/ when the reference objects are absent) on a bounded sample of
    every batch.  Returns (patches/s, cores, kind, sample description); `keep`
    receives {batch index: (patch indices, potential)} of the timed runs."""
    from oracle.oracle import ref_available, run_oracle, run_reference
    kind = "reference" if all(ref_available("sor", p.ghost, 1, "f32" if p.real_size == 4 else "f64")
                              for p, _ in batches) else "port"
    cores = nthreads or host_threads()
    nthreads = cores
    # per batch sample: n patches spread over the batch, sized from a probe run
    total_t, total_p, desc = 0.0, 0, []
    per_batch = budget_s / len(batches)
    for p, d in batches:
        n = 64
        while True:
            t0 = time.perf_counter()
            _run_cpu(kind, p, d, n, nthreads)
            dt = time.perf_counter() - t0
            if dt > per_batch / 4 or n >= len(d["rho"]):
                break
            n = min(len(d["rho"]), n * 4)
        t0 = time.perf_counter()
        res = _run_cpu(kind, p, d, n, nthreads)
        dt = time.perf_counter() - t0
        if keep is not None:
            keep[len(desc)] = res
        total_t += dt
        total_p += n
        desc.append(f"g{p.ghost}/f{8 * p.real_size}:{n}")
    return total_p / total_t, cores, kind, "patches per batch " + ",".join(desc)


def _run_cpu(kind, p, d, n, nthreads):
    from oracle.oracle import run_oracle, run_reference
    # n patches spread evenly over the batch (patch positions cover the box in
    # order, so a prefix would be one corner of it)
    idx = np.linspace(0, len(d["rho"]) - 1, n).round().astype(np.int64)
    rho = np.ascontiguousarray(d["rho"][idx])
    pin = np.ascontiguousarray(d["pot_in"][idx])
    if kind == "reference":
        q = p.copy(gra_acc=0)
        pot = run_reference(q, rho, pin.copy(), nthreads=nthreads)[0]
    else:
        pot = run_oracle(p, rho, pin, accum_f64=False, nthreads=nthreads)[0]
    return idx, pot


def rel_linf(a, b) -> float:
    """max over patches of ||a - b||_inf / ||b||_inf"""
    a = np.asarray(a, dtype=np.float64).reshape(len(a), -1)
    b = np.asarray(b, dtype=np.float64).reshape(len(b), -1)
    return float((np.abs(a - b).max(1) / np.maximum(np.abs(b).max(1), 1e-300)).max())


def headline_errors(torch, batches, dev_in, keep: dict) -> dict:
    """Relative L-infinity error of every batch's potential against the
    reference CPU solver (on the patches its timed sample solved) and, for the
    FP32 batches, against the FP64 solution of the same inputs (the library's
    FP64 path, which equals the FP64 CPU restatement bit for bit)."""
    from gpg.lib import solve_device
    out = {}
    for k, ((p, _), t) in enumerate(zip(batches, dev_in)):
        gpu = t["pot_out"].cpu().numpy()
        rec = {}
        if k in keep:
            idx, ref = keep[k]
            rec["vs_reference_cpu"] = rel_linf(gpu[idx], ref)
            rec["patches_vs_reference_cpu"] = int(len(idx))
        if p.real_size == 4:
            p64 = default_params(8, p.ghost, GPG_SOR, gra_acc=0)
            pot64 = solve_device(p64, t["rho"].double(), t["pot_in"].double())[0]
            rec["vs_fp64"] = rel_linf(gpu, pot64.cpu().numpy())
        out[f"f{8 * p.real_size}_g{p.ghost}"] = rec
    return out


# ---------------------------------------------------------------------------
# the other configurations of the path, measured beside the headline (not the bench value)
# ---------------------------------------------------------------------------
def _event_ms(torch, fn, reps=5, warm=3):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def extra_configs(torch, dev, cpu: bool):
    """MG + 5-point gravity (16384 patches, ghost 3, FP32); the mixed batch
    (65536 patches, ghost 1-5 in 30/30/20/10/10 %, rho0 log-uniform over 4
    decades, zero start, absolute L1 tolerance, one persistent launch replayed
    from a CUDA graph); plain SOR from zero start to a fixed relative
    tolerance (the plain-SOR arm of the metric)."""
    from gpg.abi import GPG_INIT_ZERO, GPG_STOP_ABS_TOLERANCE
    from gpg.inputs import log_uniform, mixed_ghost_assignment
    from gpg.lib import BatchPlan, solve_device
    out = {}
    # --- MG + P5 gravity -----------------------------------------------------
    n = 16384
    d = make_patches(n, 3, seed=21, gra_ghost=2, dtype=np.float32)
    p = default_params(4, 3, 2, gra_ghost=2, p5_gradient=1)
    t = {k: torch.from_numpy(v).to(dev) for k, v in d.items() if k != "geometry"}
    pot = torch.empty((n, 12, 12, 12), device=dev)
    it = torch.empty(n, dtype=torch.int32, device=dev)
    rs = torch.empty(n, dtype=torch.float64, device=dev)
    flu = t["flu"].clone()
    ms = _event_ms(torch, lambda: solve_device(p, t["rho"], t["pot_in"], pot_out=pot, flu=flu, iters=it, resid=rs))
    rec = {"workload": "MG V-cycle, ghost 3, FP32 (FP64 error norm), 5-point gravity, 16384 patches",
           "patches_per_s": n / ms * 1e3, "ms": ms, "cycles_mean": float(it.float().mean())}
    # errors of one fresh solve (the timed calls updated the fluid repeatedly)
    flu1 = t["flu"].clone()
    solve_device(p, t["rho"], t["pot_in"], pot_out=pot, flu=flu1, iters=it, resid=rs)
    gpot, gflu = pot.cpu().numpy(), flu1.cpu().numpy()
    p64 = default_params(8, 3, 2, gra_ghost=2, p5_gradient=1)
    pot64, flu64, _, _ = solve_device(p64, t["rho"].double(), t["pot_in"].double(), flu=t["flu"].double())
    rec["errors"] = {"pot_vs_fp64": rel_linf(gpot, pot64.cpu().numpy()),
                     "flu_vs_fp64": rel_linf(gflu, flu64.cpu().numpy())}
    if cpu:
        from oracle.oracle import ref_available, run_reference
        if ref_available("mg", 3, 2, "f32"):
            # 4096 patches spread over the batch, all host threads, a warm-up
            # call and the best of 3 timed calls
            m = 4096
            idx = np.linspace(0, n - 1, m).round().astype(np.int64)
            sub = {k: np.ascontiguousarray(d[k][idx]) for k in ("rho", "pot_in", "flu")}
            best = None
            for r in range(4):
                pin_c, flu_c = sub["pot_in"].copy(), sub["flu"].copy()
                t0 = time.perf_counter()
                rpot, rflu, _ = run_reference(p, sub["rho"], pin_c, flu=flu_c, nthreads=host_threads())
                dt = time.perf_counter() - t0
                if r > 0:
                    best = dt if best is None else min(best, dt)
            rec["cpu_reference"] = {"patches_per_s": m / best, "cores": host_threads(),
                                    "sample": f"{m} patches spread over the batch, warm-up + best of 3"}
            rec["errors"]["pot_vs_reference_cpu"] = rel_linf(gpot[idx], rpot)
            rec["errors"]["flu_vs_reference_cpu"] = rel_linf(gflu[idx], rflu)
    out["mg_gravity_g3_f32_16384"] = rec
    # --- the reference's CPU-runnable default: 256 patches, ghost 1, FP32 ----
    out["sor_g1_f32_256"] = default_case(torch, dev, cpu)
    # --- mixed batch ---------------------------------------------------------
    N = 65536
    gh = mixed_ghost_assignment(N, 7)
    rho0 = log_uniform(N, 8)
    groups, crsum = [], 0.0
    for g in range(1, 6):
        idx = np.flatnonzero(gh == g)
        dd = make_patches(len(idx), g, seed=100 + g, rho0=rho0[idx], dtype=np.float32, fluid=False)
        cr = np.abs(dd["rho"].astype(np.float64)).reshape(len(idx), -1).sum(1).max() * 4 * np.pi * 1e-5
        crsum = max(crsum, cr)
        m = len(idx)
        groups.append({"ghost": g, "rho": torch.from_numpy(dd["rho"]).to(dev),
                       "pot_in": torch.from_numpy(dd["pot_in"]).to(dev),
                       "pot_out": torch.empty((m, 10, 10, 10), device=dev),
                       "iters": torch.empty(m, dtype=torch.int32, device=dev),
                       "resid": torch.empty(m, dtype=torch.float64, device=dev)})
    # three stopping rules on the same mix (SOR, FP32, one CUDA-graph launch,
    # the faster of the persistent work-queue kernel and the concurrent
    # per-ghost-size kernels):
    #  reference:      the reference's own rule (interpolated start, stop when
    #                  the L1 residual grows, Min_Iter 10, Max_Iter 60) -- the
    #                  accuracy every reference caller gets; the headline row
    #  fixed_residual: zero start to the calibrated fixed residual (the largest
    #                  per-ghost value, 1.4e-6 x sum|interpolated phi|)
    #  absolute:       zero start to one absolute L1 tolerance, 3 % of the
    #                  largest source norm: stops light patches after a sweep or
    #                  two (the spread of iteration counts the configuration
    #                  asks for exists only under an absolute tolerance, since
    #                  the problem is linear in rho0); its per-patch error is
    #                  large by construction
    from gpg.abi import GPG_STOP_POT_TOLERANCE, POT_TOL
    rules = {
        "reference": default_params(4, 1, GPG_SOR, gra_acc=0),
        "fixed_residual": default_params(4, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_POT_TOLERANCE,
                                         sor_tolerance=max(POT_TOL[(4, g)] for g in range(1, 6)), sor_min_iter=1,
                                         sor_max_iter=300, gra_acc=0),
        "absolute": default_params(4, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_ABS_TOLERANCE,
                                   sor_tolerance=0.03 * crsum, sor_min_iter=1, sor_max_iter=200, gra_acc=0)}
    pot64s = []
    for g in groups:
        p64 = default_params(8, g["ghost"], GPG_SOR, gra_acc=0)
        pot64s.append(solve_device(p64, g["rho"].double(), g["pot_in"].double())[0].cpu().numpy())
    mixed = {"workload": "65536 patches, ghost 1-5 (30/30/20/10/10 %), rho0 log-uniform 1..1e4, FP32 SOR, one "
                         "CUDA-graph launch (faster of the persistent work-queue kernel and the concurrent "
                         "per-ghost-size kernels); rows: stopping rules"}
    for name, pb in rules.items():
        plan = BatchPlan(pb, groups, dev.index, mode=0)
        ms = _event_ms(torch, lambda: plan.launch())
        plan.close()
        plan = BatchPlan(pb, groups, dev.index, mode=1)
        ms_conc = _event_ms(torch, lambda: plan.launch())
        plan.close()
        its = np.concatenate([g["iters"].cpu().numpy() for g in groups])

        def separate():
            for g in groups:
                q = pb.copy(ghost=g["ghost"], sor_omega={1: 1.49, 2: 1.57, 3: 1.62, 4: 1.65, 5: 1.69}[g["ghost"]])
                solve_device(q, g["rho"], g["pot_in"], pot_out=g["pot_out"], iters=g["iters"], resid=g["resid"])
        ms_sep = _event_ms(torch, separate)
        per_patch, abs_err, scale = [], 0.0, 0.0
        for g, pot64 in zip(groups, pot64s):
            a_ = g["pot_out"].cpu().numpy().astype(np.float64).reshape(len(pot64), -1)
            b_ = pot64.reshape(len(pot64), -1)
            e = np.abs(a_ - b_).max(1)
            per_patch.append(e / np.abs(b_).max(1))
            abs_err, scale = max(abs_err, float(e.max())), max(scale, float(np.abs(b_).max()))
        per_patch = np.concatenate(per_patch)
        mixed[name] = {
            "rule": {"reference": "interpolated start, stop at the first growth of the L1 residual, Min_Iter 10, "
                                  "Max_Iter 60 (CPU_PoissonSolver_SOR.cpp:275-281)",
                     "fixed_residual": f"zero start, L1 residual <= {pb.sor_tolerance:.2g} x sum|interpolated phi|",
                     "absolute": f"zero start, L1 residual <= {pb.sor_tolerance:.4g} (3 % of the largest source "
                                 "norm)"}[name],
            "patches_per_s": N / min(ms, ms_conc) * 1e3, "ms_graph_persistent_work_queue": ms,
            "ms_graph_concurrent_per_ghost_kernels": ms_conc, "ms_one_launch_per_ghost_size": ms_sep,
            "iters_min": int(its.min()), "iters_p50": float(np.median(its)), "iters_max": int(its.max()),
            "frac_max_iter": float((its >= pb.sor_max_iter).mean()),
            "vs_fp64": {"rel_linf_max_over_patches": float(per_patch.max()),
                        "rel_linf_median_over_patches": float(np.median(per_patch)),
                        "linf_over_batch_max_potential": abs_err / scale}}
    mixed["patches_per_s"] = mixed["reference"]["patches_per_s"]
    mixed["headline_rule"] = "reference"
    out["batch_mixed_65536_f32"] = mixed
    # --- plain SOR, zero start, calibrated fixed residual ---------------------
    from gpg.abi import fixed_residual_params
    tot_ms, tot_n = 0.0, 0
    per = {}
    for rs_ in (4, 8):
        for g in GHOSTS:
            dd = make_patches(NPATCH, g, seed=1000 + g, dtype=np.float32 if rs_ == 4 else np.float64, fluid=False)
            pp = fixed_residual_params(rs_, g, init_mode=GPG_INIT_ZERO, max_iter=300, gra_ghost=1)
            tt = {k: torch.from_numpy(v).to(dev) for k, v in dd.items() if k != "geometry"}
            po = torch.empty((NPATCH, 10, 10, 10), device=dev, dtype=torch.float32 if rs_ == 4 else torch.float64)
            ms = _event_ms(torch, lambda: solve_device(pp, tt["rho"], tt["pot_in"], pot_out=po, iters=it[:NPATCH],
                                                       resid=rs[:NPATCH]))
            p64 = default_params(8, g, GPG_SOR, gra_acc=0)
            pot64 = solve_device(p64, tt["rho"].double(), tt["pot_in"].double())[0]
            itn = it[:NPATCH].cpu().numpy()
            per[f"f{8 * rs_}_g{g}"] = {"ms": ms, "iters_mean": float(itn.mean()), "iters_max": int(itn.max()),
                                       "rel_linf_vs_fp64": rel_linf(po.cpu().numpy(), pot64.cpu().numpy())}
            tot_ms += ms
            tot_n += NPATCH
    out["plain_sor_zero_start_fixed_residual"] = {
        "workload": "ghost 2-5 x 4096 patches x FP32/FP64, zero interior start, stop at the calibrated fixed "
                    "residual (L1 residual <= POT_TOL(precision, ghost) x sum|interpolated phi|), Max_Iter 300",
        "patches_per_s": tot_n / tot_ms * 1e3, "per_batch": per}
    return out


def default_case(torch, dev, cpu: bool) -> dict:
    """The reference's default run (Main.cpp:1142-1157 parameters): 256
    patches, ghost 1, FP32, SOR with the reference rule and the gravity update
    (GRA_GHOST 1).  Launch-latency bound on a B200: the line gives the
    latency of one device-resident solve and the reference CPU beside it."""
    from gpg.lib import solve_device
    n = 256
    d = make_patches(n, 1, seed=5, dtype=np.float32)
    p = default_params(4, 1, GPG_SOR)
    t = {k: torch.from_numpy(v).to(dev) for k, v in d.items() if k != "geometry"}
    pot = torch.empty((n, 10, 10, 10), device=dev)
    it = torch.empty(n, dtype=torch.int32, device=dev)
    rs = torch.empty(n, dtype=torch.float64, device=dev)
    flu = t["flu"].clone()
    ms = _event_ms(torch, lambda: solve_device(p, t["rho"], t["pot_in"], pot_out=pot, flu=flu, iters=it, resid=rs),
                   reps=50, warm=5)
    rec = {"workload": "256 patches, ghost 1, FP32, SOR reference rule + gravity (the reference's default run)",
           "ms": ms, "patches_per_s": n / ms * 1e3, "timing": "device-resident, CUDA events, mean of 50 calls"}
    if cpu:
        from oracle.oracle import ref_available, run_reference
        if ref_available("sor", 1, 1, "f32"):
            best = None
            for r in range(4):
                t0 = time.perf_counter()
                rpot, rflu, _ = run_reference(p, d["rho"], d["pot_in"].copy(), flu=d["flu"].copy(),
                                              nthreads=host_threads())
                dt = time.perf_counter() - t0
                if r > 0:
                    best = dt if best is None else min(best, dt)
            flu1 = t["flu"].clone()
            solve_device(p, t["rho"], t["pot_in"], pot_out=pot, flu=flu1)
            rec["cpu_reference"] = {"ms": best * 1e3, "patches_per_s": n / best,
                                    "cores": host_threads(), "sample": "all 256, warm-up + best of 3"}
            rec["errors"] = {"pot_vs_reference_cpu": rel_linf(pot.cpu().numpy(), rpot),
                             "flu_vs_reference_cpu": rel_linf(flu1.cpu().numpy(), rflu)}
    return rec


def learned_config(torch):
    """The learned-guess workload on 65536 held-out ghost-1 FP32 patches
    (rho0 log-uniform over 4 decades, power index uniform in [1.5, 2.5]), every
    start solved to the calibrated fixed residual: zero-start plain SOR (the
    metric's comparison), the interpolated start (the reference's), the
    learned linear correction fused into the SOR kernel, and the 4 x 32
    conv net's guess; errors against the FP64 solution; the fused kernel's
    HBM roofline and the conv net's tensor roofline."""
    import learned
    from gpg.linear import LinearGuess
    from gpg.net import Net
    if not os.path.exists(learned.DEFAULT_LIN + ".bin"):
        return {"unavailable": "no trained linear correction (run learned.py train --model lin)"}
    lin = LinearGuess(max_batch=1)
    learned.load_lin(lin)
    net = None
    if os.path.exists(learned.DEFAULT_WEIGHTS + ".bin"):
        net = Net(max_batch=1024)
        learned.load(net, learned.DEFAULT_WEIGHTS)
    rec = learned.evaluate(net=net, lin=lin, npatch=65536, seed=99, reps=10)
    lin.close()
    if net is not None:
        net.close()
    peaks = _measured_peaks() or {}
    n = 65536
    ms = rec["learned_linear"]["ms"]
    # compulsory HBM bytes of the fused solve per patch: rho 8^3 + coarse 8^3
    # in, interior 8^3 out (FP32); weights are read once per CTA
    byts = (512 + 512 + 512) * 4
    hbm = peaks.get("hbm_gbs")
    rec["learned_linear"]["roofline"] = {
        "bound": "hbm", "unit": "GB/s", "kernel": "lin_sor_kernel (fold + tcgen05 MMA + unfold + SOR)",
        "achieved": byts * n / (ms / 1e3) / 1e9, "peak": hbm, "frac": (byts * n / (ms / 1e3) / 1e9 / hbm) if hbm else None,
        "bytes_per_patch": byts, "tensor_flop_per_patch": learned.LIN_FLOP_EXECUTED,
        "tensor_tflops": learned.LIN_FLOP_EXECUTED * n / ms * 1e-9}
    if "learned_conv" in rec:
        peak = peaks.get("bf16_tflops")
        c = rec["learned_conv"]
        ms_net = c["ms_network"]
        c["network_roofline"] = {
            "bound": "tensor", "unit": "TFLOP/s", "achieved": c["network_tflops"],
            "achieved_executed": learned.NET_FLOP_EXECUTED * n / ms_net * 1e-9, "peak": peak,
            "peak_kind": "measured bf16 burst" if peak else None,
            "frac": c["network_tflops"] / peak if peak else None}
    rec["weights"] = {"linear": os.path.relpath(learned.DEFAULT_LIN, REPO) + ".bin",
                      "conv": os.path.relpath(learned.DEFAULT_WEIGHTS, REPO) + ".bin"}
    rec["e2e"] = learned_e2e(torch, steps=5)
    return rec


def learned_e2e(torch, steps: int) -> dict:
    """The learned-init solve and the zero-start plain solve end to end
    through the public entry points (gpg_lin_solve_device,
    gpg_poisson_gravity_device): every step copies the 65536 patches' inputs
    from pinned host memory, solves to the fixed residual and copies the
    interior potential and sweep counts back; host clock around a full sync."""
    import learned
    from gpg.abi import GPG_INIT_INTERP, GPG_INIT_ZERO
    from gpg.lib import solve_device
    from gpg.linear import LinearGuess
    dev = torch.device("cuda", torch.cuda.current_device())
    n = 65536
    rho_h, pin_h = learned.dataset(n, 99)
    h_rho, h_pin = torch.from_numpy(rho_h).pin_memory(), torch.from_numpy(pin_h).pin_memory()
    h_pot = torch.empty((n, 8, 8, 8), dtype=torch.float32).pin_memory()
    h_it = torch.empty(n, dtype=torch.int32).pin_memory()
    d_rho, d_pin = torch.empty_like(h_rho, device=dev), torch.empty_like(h_pin, device=dev)
    d_pot = torch.empty((n, 8, 8, 8), device=dev)
    d_it = torch.empty(n, dtype=torch.int32, device=dev)
    d_rs = torch.empty(n, dtype=torch.float64, device=dev)
    lin = LinearGuess(max_batch=1)
    learned.load_lin(lin)
    arms = {"learned": (learned.sor_params(4, GPG_INIT_INTERP),
                        lambda p: lin.solve(p, d_rho, d_pin, pot_out=d_pot, iters=d_it, resid=d_rs)),
            "plain_zero_start": (learned.sor_params(4, GPG_INIT_ZERO),
                                 lambda p: solve_device(p, d_rho, d_pin, pot_out=d_pot, iters=d_it, resid=d_rs))}
    out = {"h2d_bytes_per_step": int(h_rho.numel() * 4 + h_pin.numel() * 4),
           "d2h_bytes_per_step": int(h_pot.numel() * 4 + h_it.numel() * 4), "unit": "patches/s",
           "timing": "host clock around a full device sync, copies and solve on the current stream"}
    for name, (p, solve_fn) in arms.items():
        def step():
            d_rho.copy_(h_rho, non_blocking=True)
            d_pin.copy_(h_pin, non_blocking=True)
            solve_fn(p)
            h_pot.copy_(d_pot, non_blocking=True)
            h_it.copy_(d_it, non_blocking=True)
        step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        torch.cuda.synchronize()
        out[name] = n * steps / (time.perf_counter() - t0)
    lin.check()
    lin.close()
    out["ratio"] = out["learned"] / out["plain_zero_start"]
    return out


def learned_vs_plain(rec: dict) -> dict:
    """The headline comparison (learned-init + SOR vs plain zero-start SOR to
    the fixed residual), from learned_config()."""
    if "learned_linear" not in rec:
        return {"unavailable": rec.get("unavailable", "no learned arm")}
    z, i, l = rec["plain_zero_start"], rec["plain_interpolated_start"], rec["learned_linear"]
    out = {"ratio": l["patches_per_s"] / z["patches_per_s"],
           "learned_init_patches_per_s": l["patches_per_s"],
           "plain_zero_start_patches_per_s": z["patches_per_s"],
           "ratio_vs_interpolated_start": l["patches_per_s"] / i["patches_per_s"],
           "plain_interpolated_start_patches_per_s": i["patches_per_s"],
           "sweeps_mean": {"learned": l["sweeps"]["mean"], "zero_start": z["sweeps"]["mean"],
                           "interpolated_start": i["sweeps"]["mean"]},
           "rel_linf_vs_fp64_max": {"learned": l["rel_linf_vs_fp64"]["max"],
                                    "zero_start": z["rel_linf_vs_fp64"]["max"],
                                    "interpolated_start": i["rel_linf_vs_fp64"]["max"]},
           "workload": rec["workload"] + "; learned init = interpolated start + learned linear correction "
                                         "(fused, tcgen05), plain = zero-start SOR",
           "tolerance": rec["tolerance"], "timing": "device-resident, CUDA events, mean of 10 launches"}
    if "learned_conv" in rec:
        out["conv_net_ratio"] = rec["learned_conv"]["patches_per_s"] / z["patches_per_s"]
    if "e2e" in rec:
        out["e2e"] = rec["e2e"]
    return out


def _measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return None


def launch_command(argv: list[str], gpus: int, port: int) -> list[str]:
    """The torchrun command that runs this script on `gpus` local ranks."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(gpus),
            "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + list(argv)


def ensure_ranks(argv: list[str], gpus: int) -> int | None:
    """--gpus N without a process group: start N ranks (torchrun) and return
    its exit status; inside a process group, --gpus must equal WORLD_SIZE
    (exit status 2 otherwise); None = carry on in this process."""
    world = os.environ.get("WORLD_SIZE")
    if world is None:
        if gpus <= 1:
            return None
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        return subprocess.call(launch_command(argv, gpus, port))
    if int(world) != gpus:
        print(json.dumps({"error": f"--gpus {gpus} but WORLD_SIZE {world}"}), file=sys.stderr, flush=True)
        return 2
    return None


def launch_check() -> int:
    """CPU check of the rank set-up (gloo): every rank joins, the max over
    ranks reaches rank 0, which prints n_gpus = the world size."""
    import datetime
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    t = torch.tensor([float(rank + 1)])
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        print(json.dumps({"n_gpus": world, "max_over_ranks": float(t.item())}), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else list(argv)
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--launch-check", action="store_true",
                    help="CPU check of the --gpus rank set-up (gloo); no GPU work")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpg", choices=["gpg", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--one-stream", action="store_true",
                    help="time the step with its batches one after another on one stream")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the other configurations (MG, mixed batch, learned guess)")
    ap.add_argument("--only", default=None,
                    help="comma list of batches to run (e.g. f64_g5); profiling cases, not a bench line")
    a = ap.parse_args(argv)
    rc = ensure_ranks(argv, a.gpus)
    if rc is not None:
        return rc
    if a.launch_check:
        return launch_check()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return 0
        batches = workload(0)
        t_all = []
        for _ in range(a.warmup):
            reference_cpu(batches, budget_s=min(2.0, 10.0 / max(1, a.warmup)))
        vals = []
        for _ in range(a.steps):
            # bounded CPU sample per step; the whole run stays near a minute
            v, cores, kind, sample = reference_cpu(batches, budget_s=max(0.8, min(8.0, 48.0 / max(1, a.steps))))
            vals.append(v)
        v = float(np.median(vals))
        line = {"metric": METRIC, "value": v, "unit": "patches/s", "n_gpus": a.gpus, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": NPATCH * len(batches) / v * 1e3, "scaling": "weak",
                "higher_is_better": True, "impl": "reference",
                "dtype": "f32+f64", "data": "synthetic",
                "config": bench_config(),
                "cpu_baseline": {"value": v, "unit": "patches/s", "cores": cores, "kind": kind,
                                 "sample": sample},
                "e2e": {"value": v, "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "vs_baseline": None}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)
    from gpg.lib import Context, library, solve_device
    library()

    batches = workload(rank, a.only.split(",") if a.only else None)
    dev_in = []
    for p, d in batches:
        n = len(d["rho"])
        gn = 8 + 2 * p.gra_ghost
        tdt = torch.float32 if p.real_size == 4 else torch.float64
        dev_in.append(dict(rho=torch.from_numpy(d["rho"]).to(dev), pot_in=torch.from_numpy(d["pot_in"]).to(dev),
                           pot_out=torch.empty((n, gn, gn, gn), dtype=tdt, device=dev),
                           iters=torch.empty(n, dtype=torch.int32, device=dev),
                           resid=torch.empty(n, dtype=torch.float64, device=dev)))
    stream = torch.cuda.current_stream(dev)
    step_inputs = sum((d["rho"].nbytes + d["pot_in"].nbytes) for _, d in batches)
    # one stream per batch: the batches are independent, so a batch's first
    # patches run while the previous one's last patches finish
    side = [torch.cuda.Stream(dev) for _ in batches]

    def step_concurrent():
        fork = torch.cuda.Event()
        fork.record(stream)
        for (p, _), t, st in zip(batches, dev_in, side):
            st.wait_event(fork)
            solve_device(p, t["rho"], t["pot_in"], pot_out=t["pot_out"], iters=t["iters"], resid=t["resid"],
                         stream=st)
        for st in side:
            join = torch.cuda.Event()
            join.record(st)
            stream.wait_event(join)

    def step_sequential(events=None):
        for k, ((p, _), t) in enumerate(zip(batches, dev_in)):
            if events is not None:
                events[k][0].record(stream)
            solve_device(p, t["rho"], t["pot_in"], pot_out=t["pot_out"], iters=t["iters"], resid=t["resid"])
            if events is not None:
                events[k][1].record(stream)

    step = step_sequential if a.one_stream else step_concurrent
    for _ in range(max(a.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in batches]
          for _ in range(a.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_start, s_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        barrier()
        start.record(stream)
        for s in range(a.steps):
            step()
        stop.record(stream)
        barrier()
        # the same steps one launch at a time on one stream: per-kernel times
        # (roofline, per-batch fractions) without overlap between kernels
        s_start.record(stream)
        for s in range(a.steps):
            step_sequential(ev[s])
        s_stop.record(stream)
        barrier()
    ms = start.elapsed_time(stop)
    ms_seq = s_start.elapsed_time(s_stop)
    per_kernel = np.array([[e[0].elapsed_time(e[1]) for e in row] for row in ev])  # [steps, batches]
    if world > 1:
        t = torch.tensor([ms, ms_seq], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms, ms_seq = float(t[0].item()), float(t[1].item())
    patches_step = NPATCH * len(batches)
    value = world * patches_step * a.steps / (ms / 1e3)
    value_one_stream = world * patches_step * a.steps / (ms_seq / 1e3)
    iters = [t["iters"].cpu().numpy() for t in dev_in]

    # ---- end to end through the reference-shaped host API ----------------
    e2e = None
    if not a.no_e2e:
        ctxs = []
        for (p, d) in batches:
            c = Context(dev.index, nstream=4)
            rho, pin, pout, _ = c.allocate(p, NPATCH // 8)
            rho[...] = d["rho"]
            pin[...] = d["pot_in"]
            ctxs.append(c)
        def e2e_run(steps, pipelined):
            # pipelined: a batch waits only for its own previous results (on the
            # host) before its next inputs go out, so the copy engines never
            # drain between steps; lockstep: every step ends with a full sync
            barrier()
            t0 = time.perf_counter()
            for _ in range(steps):
                for (p, _), c in zip(batches, ctxs):
                    if pipelined:
                        c.synchronize()
                    c.asyn_solve(p, NPATCH // 8)
                if not pipelined:
                    for c in ctxs:
                        c.synchronize()
            for c in ctxs:
                c.synchronize()
            barrier()
            el = time.perf_counter() - t0
            if world > 1:
                t = torch.tensor([el], device=dev)
                torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
                el = float(t.item())
            return el

        e2e_run(2, False)
        e2e_s = e2e_run(a.steps, True)
        lock_s = e2e_run(a.steps, False)
        h2d = step_inputs
        d2h = sum(NPATCH * (patch_sizes(p)["pot_out"] * p.real_size + 4 + 8) for p, _ in batches)
        # host link: pinned -> device copy bandwidth, the bound of this leg
        hb = torch.empty(256 * 2 ** 20, dtype=torch.uint8).pin_memory()
        db = torch.empty_like(hb, device=dev)
        # the link's capability: the fastest of 8 timed copies (the host is
        # shared, so single copies vary by 20 %)
        link_ms = min(_event_ms(torch, lambda: db.copy_(hb, non_blocking=True), reps=1, warm=1 if r == 0 else 0)
                      for r in range(8))
        link_gbs = hb.numel() / (link_ms / 1e3) / 1e9
        del hb, db
        e2e = {"value": world * patches_step * a.steps / e2e_s, "unit": "patches/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "timing": "host clock around full device sync",
               "pipelining": "each batch's previous results are on the host before its next inputs are "
                             "issued; no global sync between steps",
               "lockstep_value": world * patches_step * a.steps / lock_s,
               "h2d_link_gbs": link_gbs,
               "h2d_bound_patches_per_s": world * patches_step / (h2d / (link_gbs * 1e9))}
        for c in ctxs:
            c.close()

    # ---- roofline of the dominant kernel ---------------------------------
    tot = per_kernel.sum(0)
    k = int(np.argmax(tot))
    pk, _ = batches[k]
    launch_ms = float(per_kernel[:, k].mean())
    algo_bytes = compulsory_bytes(pk) * NPATCH
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = algo_bytes / (launch_ms / 1e3) / 1e9
    traffic = None
    try:
        with open(os.path.join(REPO, "profiles", "ncu_traffic.json")) as f:
            tr = json.load(f)
        traffic = tr.get(f"sor_f{8 * pk.real_size}_g{pk.ghost}_{NPATCH}")
    except OSError:
        pass

    # on-chip bound of the same kernel: the shared-memory accesses one cell
    # update needs in the layout the kernel runs (one row per lane: 3 loads +
    # 1 store; two rows per lane: 2 loads + 1 store; a column split between
    # two lanes adds one load per lane, row and pass); a warp-wide access of
    # 4-byte (8-byte) values is 1 (2) wavefronts; the pipe serves one wavefront
    # per cycle per SM
    clocks = clk.summary()
    sm_mhz = float(clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0))
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    onchip_peak = nsm * sm_mhz * 1e6

    def layout(p):
        import ctypes as C
        from gpg.lib import check
        lib = library()
        v, z, y = C.c_int(), C.c_int(), C.c_int()
        check(lib.gpg_sor_variant_for_launch(p.real_size, p.ghost, NPATCH, C.byref(v)))
        check(lib.gpg_sor_variant_layout(v.value, C.byref(z), C.byref(y)))
        m = 6 + 2 * p.ghost
        acc = (4.0 if y.value == 1 else 3.0) + (1.0 / (m // z.value) if z.value == 2 else 0.0)
        return v.value, z.value, y.value, acc

    def wavefronts_of(p, it):
        acc = layout(p)[3]
        return float(it.astype(np.float64).sum()) * (6 + 2 * p.ghost) ** 3 * acc * (p.real_size * 32 // 128) / 32

    wavefronts = wavefronts_of(pk, iters[k])
    vk, zk, yk, acck = layout(pk)
    import ctypes as C
    from gpg.lib import check
    stg = C.c_int()
    check(library().gpg_sor_variant_staged(vk, C.byref(stg)))
    kname = "staged_sor_kernel" if stg.value else "sor_kernel"
    onchip = {"resource": "shared-memory pipe", "unit": "wavefronts/s",
              "achieved": wavefronts / (launch_ms / 1e3), "peak": onchip_peak,
              "frac": wavefronts / (launch_ms / 1e3) / onchip_peak,
              "algorithmic_wavefronts_per_launch": wavefronts,
              "achieved_gbs": wavefronts * 128 / (launch_ms / 1e3) / 1e9, "peak_gbs": onchip_peak * 128 / 1e9,
              "variant": {"id": vk, "lanes_per_column": zk, "rows_per_lane": yk},
              "model": f"measured sweeps x RHO_NXT^3 cell updates x {acck:.3f} shared accesses per update "
                       "(this variant's layout); 1 wavefront (128 B)/cycle/SM "
                       f"at the sampled {sm_mhz:.0f} MHz x {nsm} SMs"}

    line = {
        "metric": METRIC, "value": value, "unit": "patches/s", "n_gpus": world, "steps": a.steps,
        "warmup": max(a.warmup, 3), "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": bench_config(),
        "global_batch": world * patches_step,
        "l2": f"step inputs {step_inputs / 1e9:.2f} GB > 126 MB L2 (no flush needed)",
        "parallelism": f"patch shards x{world}",
        "gpu_launches": len(batches) * a.steps,
        "batches": ("one stream" if a.one_stream
                    else "one stream per batch, forked from and joined to the timing stream"),
        "value_one_stream": value_one_stream,
        "per_batch_ms": {f"f{8 * p.real_size}_g{p.ghost}": float(per_kernel[:, i].mean())
                         for i, (p, _) in enumerate(batches)},
        "mean_iters": {f"f{8 * p.real_size}_g{p.ghost}": float(it.mean()) for (p, _), it in zip(batches, iters)},
        "onchip_frac_per_batch": {
            f"f{8 * p.real_size}_g{p.ghost}":
                wavefronts_of(p, it) / (float(per_kernel[:, i].mean()) / 1e3) / onchip_peak
            for i, ((p, _), it) in enumerate(zip(batches, iters))},
        "roofline": {"bound": "hbm", "kernel": f"{kname} f{8 * pk.real_size} g{pk.ghost}",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes_per_launch": algo_bytes,
                     "launch_ms": launch_ms, "peak_source": "measured" if peaks else "fallback",
                     "launch_timing": "CUDA events around each launch in the one-stream pass of the same steps",
                     "onchip": onchip},
        "e2e": e2e,
        "clocks": clocks,
    }
    if rank == 0 and not a.no_cpu_baseline and world == 1:
        keep = {}
        v, cores, kind, sample = reference_cpu(batches, budget_s=20.0, keep=keep)
        line["cpu_baseline"] = {"value": v, "unit": "patches/s", "cores": cores, "kind": kind, "sample": sample}
        # the same code on one core (smaller sample): the per-core cost of the reference
        v1, _, _, sample1 = reference_cpu(batches, budget_s=6.0, nthreads=1)
        line["cpu_baseline"]["one_core"] = {"value": v1, "unit": "patches/s", "cores": 1, "sample": sample1}
        line["errors"] = headline_errors(torch, batches, dev_in, keep)
    if rank == 0 and not a.only and world == 1:
        rec = learned_config(torch)
        line["learned_vs_plain"] = learned_vs_plain(rec)
    if rank == 0 and not a.no_extra and not a.only and world == 1:
        line["extra"] = extra_configs(torch, dev, cpu=not a.no_cpu_baseline)
        line["extra"]["learned_init_sor_g1"] = rec
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
