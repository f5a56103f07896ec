"""Train and evaluate the learned initial guess for ghost-size-1 SOR.

    python gpu_testbed_poisson-gravity_b200/learned.py train --npatch 1048576 --epochs 2 \
        --out gpu_testbed_poisson-gravity_b200/weights/learned_init
    python gpu_testbed_poisson-gravity_b200/learned.py eval  --npatch 65536 \
        --weights gpu_testbed_poisson-gravity_b200/weights/learned_init

Data: seeded ghost-1 patches (gpg.inputs) with rho0 log-uniform over 4
decades and power index uniform in [1.5, 2.5].  Targets are the plain SOR's own
solutions (reference rule from the interpolated start, i.e. converged to the
FP32 round-off floor) computed by libgpg.  Training and inference run on the
library's tensor-core kernels (gpg_net_*).  Evaluation solves held-out patches
(other seeds) from a zero start and from the learned guess to the same
relative tolerance and reports sweeps, patches/s (the network's inference
included) and the error against an FP64 solution of the same patches.
Weights are saved as <out>.bin (float32) with a <out>.json header;
weights/learned_init.* is the checkpoint of the command above (2^20 patches,
seed 1, 2 epochs of batch 1024, Adam with a cosine learning-rate schedule).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402

from gpg.abi import (GPG_INIT_GUESS, GPG_INIT_INTERP, GPG_INIT_ZERO, GPG_SOR,  # noqa: E402
                     GPG_STOP_TOLERANCE, default_params)
from gpg.inputs import log_uniform, make_patches  # noqa: E402

CNST = float(np.float32(np.float32(4 * np.pi * 1e-5) * np.float32(1.0) * np.float32(1.0)))
CHUNK = 65536
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "learned_init")
# algorithmic FLOPs of one patch's forward pass: 3^3 convolutions 3 -> 32 -> 32
# -> 32 on the 10^3 cube, 32 -> 1 on the 8^3 interior
NET_FLOP = 2 * 27 * (1000 * (3 * 32 + 32 * 32 + 32 * 32) + 512 * 32)
# FLOPs the fused kernel's MMAs execute per patch (M=128 x K=16 tiles): 10 row
# tiles x 14 tap pairs (N=32) for layer 1, 10 x 27 x 2 K halves (N=32) for
# layers 2 and 3, 8 x 27 x 2 (N=16) for layer 4
NET_FLOP_EXECUTED = 2 * 128 * 16 * (32 * (10 * 14 + 2 * 10 * 27 * 2) + 16 * 8 * 27 * 2)


def dataset(n: int, seed: int, dtype=np.float32, first: int = 0, stop: int | None = None):
    """(rho, pot_in) [..][8]^3 of ghost-1 patches first..stop of an n-patch set,
    generated in chunks of CHUNK patches, each from its own seeds; a range
    that starts on a chunk boundary (a data-parallel shard) gets exactly the
    patches the whole set has there."""
    stop = n if stop is None else stop
    if first % CHUNK or not 0 <= first <= stop <= n:
        raise ValueError("shard must start on a chunk boundary and lie inside the set")
    rho = np.empty((stop - first, 8, 8, 8), dtype=dtype)
    pin = np.empty((stop - first, 8, 8, 8), dtype=dtype)
    for c0 in range(first, stop, CHUNK):
        m = min(CHUNK, n - c0)
        s = seed * 1000 + c0 // CHUNK
        rng = np.random.Generator(np.random.PCG64(s + 7))
        d = make_patches(m, 1, seed=s, rho0=log_uniform(m, s + 3), index=rng.uniform(1.5, 2.5, m),
                         dtype=dtype, fluid=False)
        k = min(m, stop - c0)
        rho[c0 - first:c0 - first + k] = d["rho"][:k]
        pin[c0 - first:c0 - first + k] = d["pot_in"][:k]
    return rho, pin


def shard(n: int, rank: int, world: int) -> tuple[int, int]:
    """Rank's [first, stop) of an n-patch training set, whole chunks per rank."""
    from gpg.shard import shard_bounds
    nchunk = (n + CHUNK - 1) // CHUNK
    if world > nchunk:
        raise ValueError(f"{world} ranks for {nchunk} chunks of {CHUNK} patches")
    lo, hi = shard_bounds(nchunk, world)[rank]
    return lo * CHUNK, min(hi * CHUNK, n)


def sor_params(real_size: int, init_mode: int, stop_mode: int = GPG_STOP_TOLERANCE, tol: float = 0.02,
               max_iter: int = 300):
    return default_params(real_size, 1, GPG_SOR, gra_acc=0, gra_ghost=0, init_mode=init_mode, stop_mode=stop_mode,
                          sor_tolerance=tol, sor_min_iter=1, sor_max_iter=max_iter)


def solve(torch, p, rho, pin, guess=None):
    from gpg.lib import solve_device
    pot, _, it, rs = solve_device(p, rho, pin, guess=guess)
    return pot, it, rs


def targets(torch, rho, pin):
    """The plain SOR's own converged solutions: reference rule, interpolated start."""
    p = default_params(4, 1, GPG_SOR, gra_acc=0, gra_ghost=0)
    pot, _, _ = solve(torch, p, rho, pin)
    return pot


def save(net, path: str, meta: dict):
    flat = net.params()
    flat.tofile(path + ".bin")
    with open(path + ".json", "w") as f:
        json.dump(dict(meta, nparams=int(flat.size), dtype="float32",
                       layers=[[8, 32], [32, 32], [32, 32], [32, 16]],
                       layout="per layer W[27][cin][cout] then b[cout]"), f, indent=1)


def load(net, path: str):
    flat = np.fromfile(path + ".bin", dtype=np.float32)
    if flat.size != net.nparams:
        raise ValueError(f"{path}.bin has {flat.size} parameters, the network {net.nparams}")
    net.set_params(flat)


def train(npatch: int, epochs: int, batch: int, lr: float, seed: int, out: str | None, log=print):
    """Train on npatch patches with global batch `batch`.  Under torchrun
    (RANK / WORLD_SIZE set) this is data-parallel over NCCL: every rank builds
    its own chunk shard and the same initial network, computes the gradient of
    its batch / world patches, the gradients are averaged with an all-reduce
    and every rank applies the same Adam step; rank 0 saves the checkpoint.
    One process without a process group runs gpg_net_train_step directly."""
    import torch
    import torch.distributed as dist
    from gpg.net import Net
    from gpg.shard import allreduce_mean_
    distributed = "RANK" in os.environ and "WORLD_SIZE" in os.environ
    rank, world = (int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])) if distributed else (0, 1)
    if distributed and not dist.is_initialized():
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", torch.cuda.current_device())
    if batch % world:
        raise ValueError(f"global batch {batch} is not a multiple of {world} ranks")
    lb = batch // world
    t0 = time.time()
    first, stop = shard(npatch, rank, world)
    rho_h, pin_h = dataset(npatch, seed, first=first, stop=stop)
    rho, pin = torch.from_numpy(rho_h).to(dev), torch.from_numpy(pin_h).to(dev)
    del rho_h, pin_h
    tgt = targets(torch, rho, pin)
    torch.cuda.synchronize()
    t_data = time.time() - t0
    nb = (stop - first) // lb
    if distributed:  # every rank takes the same number of steps
        t = torch.tensor([nb], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        nb = int(t.item())
    net = Net(max_batch=lb, seed=seed)
    loss = torch.empty(1, device=dev)
    grad = torch.empty(net.nparams, device=dev) if distributed else None
    nstep = epochs * nb
    g = torch.Generator(device="cpu").manual_seed(seed + 7919 * rank)
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hist = []
    s_ev.record()
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(nb, generator=g)
        for bi in perm.tolist():
            sl = slice(bi * lb, (bi + 1) * lb)
            cur_lr = float(lr * 0.5 * (1 + np.cos(np.pi * step / max(1, nstep))))   # cosine schedule
            if distributed:
                net.gradients(rho[sl], pin[sl], tgt[sl], CNST, grad=grad, loss=loss)
                allreduce_mean_(grad)
                net.apply_gradient(grad, cur_lr)
            else:
                net.train_step(rho[sl], pin[sl], tgt[sl], CNST, cur_lr, loss=loss)
            step += 1
            if step % 200 == 0 or step == nstep:
                if distributed:
                    allreduce_mean_(loss)
                hist.append((step, float(loss.item())))
                if rank == 0:
                    log(f"step {step}/{nstep} loss {hist[-1][1]:.4e}")
    e_ev.record()
    torch.cuda.synchronize()
    net.check()
    ms = s_ev.elapsed_time(e_ev)
    meta = {"npatch": npatch, "epochs": epochs, "batch": batch, "lr": lr, "seed": seed, "steps": nstep,
            "ranks": world, "train_ms": ms, "ms_per_step": ms / max(1, nstep), "data_s": t_data,
            "loss_history": hist}
    if out and rank == 0:
        save(net, out, meta)
    return net, meta


def _event_ms(torch, fn, reps=3):
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def evaluate(net, npatch: int, seed: int, tol: float = 0.02):
    """Zero-start plain SOR vs learned-guess SOR to the same relative tolerance
    (and the reference's interpolated start beside them), then all three
    starts under the reference's own stopping rule."""
    import torch
    dev = torch.device("cuda:0")
    rho_h, pin_h = dataset(npatch, seed)
    rho, pin = torch.from_numpy(rho_h).to(dev), torch.from_numpy(pin_h).to(dev)
    p0 = sor_params(4, GPG_INIT_ZERO, tol=tol)
    pg = sor_params(4, GPG_INIT_GUESS, tol=tol)
    guess = torch.empty((npatch, 8, 8, 8), device=dev)
    out = {}
    ms_plain = _event_ms(torch, lambda: solve(torch, p0, rho, pin))
    pot0, it0, _ = solve(torch, p0, rho, pin)
    ms_net = _event_ms(torch, lambda: net.predict(rho, pin, guess, CNST))
    ms_net_layers = _event_ms(torch, lambda: net.predict(rho, pin, guess, CNST, fused=False))
    net.predict(rho, pin, guess, CNST)
    ms_sor_g = _event_ms(torch, lambda: solve(torch, pg, rho, pin, guess=guess))
    potg, itg, _ = solve(torch, pg, rho, pin, guess=guess)
    net.check()
    # FP64 solution of the same patches: reference rule from the interpolated start
    p64 = default_params(8, 1, GPG_SOR, gra_acc=0, gra_ghost=0)
    pot64, _, _ = solve(torch, p64, rho.double(), pin.double())
    ref = pot64.cpu().numpy().reshape(npatch, -1)

    def err(pot):
        a = pot.double().cpu().numpy().reshape(npatch, -1)
        return float((np.abs(a - ref).max(1) / np.abs(ref).max(1)).max())

    def stats(it):
        a = it.cpu().numpy()
        return {"mean": float(a.mean()), "p50": float(np.median(a)), "p90": float(np.percentile(a, 90)),
                "max": int(a.max())}

    out["tolerance"] = f"L1 residual <= {tol} x L1 source norm, Min_Iter 1, Max_Iter 300, FP32"
    out["plain_zero_start"] = {"sweeps": stats(it0), "ms": ms_plain, "patches_per_s": npatch / ms_plain * 1e3,
                               "rel_linf_vs_fp64": err(pot0)}
    out["learned_init"] = {"sweeps": stats(itg), "ms_network": ms_net, "ms_network_per_layer_kernels": ms_net_layers,
                           "network_tflops": NET_FLOP * npatch / ms_net * 1e-9, "ms_sor": ms_sor_g,
                           "ms": ms_net + ms_sor_g, "patches_per_s": npatch / (ms_net + ms_sor_g) * 1e3,
                           "rel_linf_vs_fp64": err(potg)}
    pi = sor_params(4, GPG_INIT_INTERP, tol=tol)
    ms_interp = _event_ms(torch, lambda: solve(torch, pi, rho, pin))
    poti, iti, _ = solve(torch, pi, rho, pin)
    out["plain_interpolated_start"] = {"sweeps": stats(iti), "ms": ms_interp,
                                       "patches_per_s": npatch / ms_interp * 1e3, "rel_linf_vs_fp64": err(poti)}
    g = guess.double().cpu().numpy().reshape(npatch, -1)
    out["learned_init"]["guess_rel_linf_vs_fp64"] = float((np.abs(g - ref).max(1) / np.abs(ref).max(1)).mean())
    out["speedup_vs_plain"] = ms_plain / (ms_net + ms_sor_g)
    out["sweep_ratio"] = out["plain_zero_start"]["sweeps"]["mean"] / max(1e-9, out["learned_init"]["sweeps"]["mean"])
    # the reference's own criterion (Min_Iter 10, stop when the L1 residual
    # grows, Max_Iter 60) from its interpolated start, a zero start and the guess
    rr = {"criterion": "reference rule: Min_Iter 10, stop at the first growth of the L1 residual, Max_Iter 60, FP32"}
    for name, mode in (("interpolated_start", GPG_INIT_INTERP), ("zero_start", GPG_INIT_ZERO),
                       ("learned_start", GPG_INIT_GUESS)):
        pr = default_params(4, 1, GPG_SOR, gra_acc=0, gra_ghost=0, init_mode=mode)
        gg = guess if mode == GPG_INIT_GUESS else None
        ms = _event_ms(torch, lambda: solve(torch, pr, rho, pin, guess=gg))
        pot, it, _ = solve(torch, pr, rho, pin, guess=gg)
        tot = ms + (ms_net if mode == GPG_INIT_GUESS else 0.0)
        rr[name] = {"sweeps": stats(it), "ms": tot, "patches_per_s": npatch / tot * 1e3,
                    "rel_linf_vs_fp64": err(pot)}
    out["reference_rule"] = rr
    return out


def time_predict(npatch: int, reps: int, weights: str | None = DEFAULT_WEIGHTS, per_layer: bool = True):
    """Device time of the network's forward pass over npatch held-out patches:
    the one-kernel path and (per_layer) the per-layer kernels, CUDA events."""
    import torch
    from gpg.net import Net
    rho_h, pin_h = dataset(npatch, 99)
    rho, pin = torch.from_numpy(rho_h).cuda(), torch.from_numpy(pin_h).cuda()
    net = Net(max_batch=min(npatch, 4096))
    if weights and os.path.exists(weights + ".bin"):
        load(net, weights)
    guess = torch.empty((npatch, 8, 8, 8), device="cuda")
    out = {"npatch": npatch}
    for fused in (True, False) if per_layer else (True,):
        ms = _event_ms(torch, lambda: net.predict(rho, pin, guess, CNST, fused=fused), reps)
        key = "fused" if fused else "per_layer"
        out[key] = {"ms": ms, "tflops": NET_FLOP * npatch / ms * 1e-9,
                    "tflops_executed": NET_FLOP_EXECUTED * npatch / ms * 1e-9}
    net.check()
    net.close()
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--npatch", type=int, default=1 << 20)
    t.add_argument("--epochs", type=int, default=2)
    t.add_argument("--batch", type=int, default=1024)
    t.add_argument("--lr", type=float, default=2e-3)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--eval", type=int, default=65536, help="held-out patches evaluated after training (0: none)")
    e = sub.add_parser("eval")
    e.add_argument("--npatch", type=int, default=65536)
    e.add_argument("--weights", default=DEFAULT_WEIGHTS)
    e.add_argument("--seed", type=int, default=99)
    tm = sub.add_parser("time", help="time the network's forward pass")
    tm.add_argument("--npatch", type=int, default=65536)
    tm.add_argument("--reps", type=int, default=5)
    tm.add_argument("--fused-only", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "time":
        print(json.dumps(time_predict(a.npatch, a.reps, per_layer=not a.fused_only)))
    elif a.cmd == "train":
        net, meta = train(a.npatch, a.epochs, a.batch, a.lr, a.seed, a.out)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}))
            if a.eval:
                print(json.dumps(evaluate(net, a.eval, 99), indent=1))
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()
    else:
        from gpg.net import Net
        net = Net(max_batch=4096)
        load(net, a.weights)
        print(json.dumps(evaluate(net, a.npatch, a.seed), indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
