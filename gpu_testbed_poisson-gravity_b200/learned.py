"""Train and evaluate the learned initial guesses for ghost-size-1 SOR.

    python gpu_testbed_poisson-gravity_b200/learned.py train --model lin --npatch 1048576 \
        --epochs 64 --batch 2048 --lr 2e-3 --out gpu_testbed_poisson-gravity_b200/weights/lin_correction
    python gpu_testbed_poisson-gravity_b200/learned.py train --model conv --npatch 1048576 --epochs 2 \
        --out gpu_testbed_poisson-gravity_b200/weights/learned_init
    python gpu_testbed_poisson-gravity_b200/learned.py eval --npatch 65536

Two models, both trained on the GPU by the library's own kernels:

* ``lin`` (gpg_lin_*): a learned linear correction of the interpolated start,
  equivariant under the cube's reflections (4 class matrices of 64 x 64 over
  the parity blocks of the residual of that start), fused into the SOR kernel
  and applied on the tensor cores (65,536 FLOP per patch);
* ``conv`` (gpg_net_*): the 4-layer 3^3 convolution network (8 -> 32 -> 32 ->
  32 -> 16 channels) that maps density and boundary shell to the interior
  (116.7 MFLOP per patch).

Data: seeded ghost-1 patches (gpg.inputs) with rho0 log-uniform over 4
decades and power index uniform in [1.5, 2.5].  Targets are the plain SOR's own
solutions (reference rule from the interpolated start, i.e. converged to the
round-off floor) computed by libgpg: FP32 for the conv net, FP64 rounded to
FP32 for the linear correction.  Evaluation solves held-out patches
(other seeds) to the calibrated fixed residual (GPG_STOP_POT_TOLERANCE,
gpg.abi.POT_TOL) from a zero start, from the interpolated start and from each
learned start, and reports sweeps, patches/s (the model's cost included) and
the error against an FP64 solution of the same patches.  Weights are saved as
<out>.bin (float32) with a <out>.json header; weights/lin_correction.* and
weights/learned_init.* are the checkpoints of the commands above.
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
                     POT_TOL, default_params, fixed_residual_params)
from gpg.inputs import log_uniform, make_patches  # noqa: E402

CNST = float(np.float32(np.float32(4 * np.pi * 1e-5) * np.float32(1.0) * np.float32(1.0)))
CHUNK = 65536
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "learned_init")
DEFAULT_LIN = os.path.join(HERE, "weights", "lin_correction")
# learned linear correction per patch: 8 blocks x 64 x 64 multiply-adds
# (algorithmic) and 16 MMAs of 128 x 16 x 16 per 8 patches (executed: the two
# blocks of an MMA also meet each other's matrix)
LIN_FLOP = 8 * 2 * 64 * 64
LIN_FLOP_EXECUTED = 16 * 2 * 128 * 16 * 16 // 8
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


def sor_params(real_size: int, init_mode: int, max_iter: int = 300):
    """SOR to the calibrated fixed residual (Min_Iter 1, Poisson only)."""
    return fixed_residual_params(real_size, 1, init_mode=init_mode, max_iter=max_iter)


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


def _stats(it):
    a = it.cpu().numpy()
    return {"mean": float(a.mean()), "p50": float(np.median(a)), "p90": float(np.percentile(a, 90)),
            "max": int(a.max())}


def evaluate(net=None, lin=None, npatch: int = 65536, seed: int = 99, reps: int = 5, rule: bool = True):
    """Every start solved to the same calibrated fixed residual (FP32,
    GPG_STOP_POT_TOLERANCE, Min_Iter 1, Max_Iter 300): zero interior (the
    plain SOR the metric compares against), the reference's interpolated
    start, the learned linear correction (`lin`, fused into the SOR kernel)
    and the convolution network's guess (`net`, a separate inference kernel
    ahead of the SOR).  Times are CUDA-event means over `reps` launches after a
    warm-up, the model's own cost included.  With `rule`, the same starts
    under the reference's own stopping rule as well."""
    import torch
    dev = torch.device("cuda:0")
    rho_h, pin_h = dataset(npatch, seed)
    rho, pin = torch.from_numpy(rho_h).to(dev), torch.from_numpy(pin_h).to(dev)
    # FP64 solution of the same patches: reference rule, interpolated start
    p64 = default_params(8, 1, GPG_SOR, gra_acc=0, gra_ghost=0)
    pot64, _, _ = solve(torch, p64, rho.double(), pin.double())
    ref = pot64.cpu().numpy().reshape(npatch, -1)
    scale = np.abs(ref).max(1)

    def err(pot):
        a = pot.double().cpu().numpy().reshape(npatch, -1)
        e = np.abs(a - ref).max(1) / scale
        return {"max": float(e.max()), "p50": float(np.median(e))}

    out = {"workload": f"{npatch} held-out ghost-1 patches (seed {seed}), FP32",
           "tolerance": (f"L1 residual <= {POT_TOL[(4, 1)]} x sum|interpolated phi| over the updated cells "
                         "(calibrated fixed residual, GPG_STOP_POT_TOLERANCE), Min_Iter 1, Max_Iter 300")}
    guess = torch.empty((npatch, 8, 8, 8), device=dev) if net is not None else None

    def arm(p, start: str, **kw):
        if start == "lin":
            fn = lambda: lin.solve(p, rho, pin)  # noqa: E731
        elif start == "conv":
            def fn():
                net.predict(rho, pin, guess, CNST)
                return solve(torch, p, rho, pin, guess=guess)
        else:
            fn = lambda: solve(torch, p, rho, pin)  # noqa: E731
        ms = _event_ms(torch, fn, reps)
        res = fn()
        pot, it = res[0], res[2] if start == "lin" else res[1]
        rec = {"sweeps": _stats(it), "ms": ms, "patches_per_s": npatch / ms * 1e3, "rel_linf_vs_fp64": err(pot)}
        rec.update(kw)
        return rec

    out["plain_zero_start"] = arm(sor_params(4, GPG_INIT_ZERO), "plain")
    out["plain_interpolated_start"] = arm(sor_params(4, GPG_INIT_INTERP), "plain")
    if lin is not None:
        out["learned_linear"] = arm(sor_params(4, GPG_INIT_INTERP), "lin", model="linear correction",
                                    flop_per_patch=LIN_FLOP, flop_per_patch_executed=LIN_FLOP_EXECUTED)
        lin.check()
    if net is not None:
        ms_net = _event_ms(torch, lambda: net.predict(rho, pin, guess, CNST), reps)
        out["learned_conv"] = arm(sor_params(4, GPG_INIT_GUESS), "conv", model="conv net", ms_network=ms_net,
                                  network_tflops=NET_FLOP * npatch / ms_net * 1e-9, flop_per_patch=NET_FLOP,
                                  flop_per_patch_executed=NET_FLOP_EXECUTED)
        net.check()
    z = out["plain_zero_start"]["ms"]
    for k in ("plain_interpolated_start", "learned_linear", "learned_conv"):
        if k in out:
            out[k]["speedup_vs_zero_start"] = z / out[k]["ms"]
    if lin is not None:
        out["learned_linear"]["speedup_vs_interpolated_start"] = (out["plain_interpolated_start"]["ms"] /
                                                                  out["learned_linear"]["ms"])
    if rule:
        rr = {"criterion": "reference rule: Min_Iter 10, stop at the first growth of the L1 residual, Max_Iter 60"}
        pr = lambda mode: default_params(4, 1, GPG_SOR, gra_acc=0, gra_ghost=0, init_mode=mode)  # noqa: E731
        rr["zero_start"] = arm(pr(GPG_INIT_ZERO), "plain")
        rr["interpolated_start"] = arm(pr(GPG_INIT_INTERP), "plain")
        if lin is not None:
            rr["learned_linear"] = arm(pr(GPG_INIT_INTERP), "lin")
        if net is not None:
            rr["learned_conv"] = arm(pr(GPG_INIT_GUESS), "conv")
        out["reference_rule"] = rr
    return out


def targets64(torch, rho, pin):
    """The plain SOR's own FP64 solutions of the same (FP32) inputs: reference
    rule from the interpolated start (converged to the FP64 round-off floor),
    rounded once to FP32."""
    p = default_params(8, 1, GPG_SOR, gra_acc=0, gra_ghost=0)
    pot, _, _ = solve(torch, p, rho.double(), pin.double())
    return pot.float()


def lin_data(lin, rho, pin, chunk: int = CHUNK):
    """Training features (u, t) of ghost-1 patches: the folded residual of the
    interpolated start and the folded correction to the plain SOR's FP64
    solution (whose rounding error is far below that of an FP32 solve at its
    floor, which would otherwise set the loss floor)."""
    import torch
    n = rho.shape[0]
    u = torch.empty((n, 8, 64), device=rho.device)
    t = torch.empty((n, 8, 64), device=rho.device)
    p = sor_params(4, GPG_INIT_INTERP)
    for c0 in range(0, n, chunk):
        sl = slice(c0, min(n, c0 + chunk))
        tg = targets64(torch, rho[sl], pin[sl])
        uu, tt = lin.features(p, rho[sl], pin[sl], target=tg)
        u[sl], t[sl] = uu, tt
    return u, t


def train_lin(npatch: int, epochs: int, batch: int, lr: float, seed: int, out: str | None, log=print):
    """Train the linear correction on npatch patches with global batch `batch`
    (Adam, cosine learning rate, parameters from zero).  Under torchrun the
    step is data-parallel as in train(): per-rank gradients of batch / world
    patches, averaged with an all-reduce, the same Adam step everywhere."""
    import torch
    import torch.distributed as dist
    from gpg.linear import LinearGuess
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
    lin = LinearGuess(max_batch=lb)
    u, t = lin_data(lin, torch.from_numpy(rho_h).to(dev), torch.from_numpy(pin_h).to(dev))
    del rho_h, pin_h
    torch.cuda.synchronize()
    t_data = time.time() - t0
    nb = (stop - first) // lb
    if distributed:
        tn = torch.tensor([nb], device=dev)
        dist.all_reduce(tn, op=dist.ReduceOp.MIN)
        nb = int(tn.item())
    loss = torch.empty(1, device=dev)
    grad = torch.empty(lin.nparams, device=dev) if distributed else None
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
            cur_lr = float(lr * 0.5 * (1 + np.cos(np.pi * step / max(1, nstep))))
            if distributed:
                lin.gradients(u[sl], t[sl], grad=grad, loss=loss)
                allreduce_mean_(grad)
                lin.apply_gradient(grad, cur_lr)
            else:
                lin.train_step(u[sl], t[sl], cur_lr, loss=loss)
            step += 1
            if step % 256 == 0 or step == nstep:
                if distributed:
                    allreduce_mean_(loss)
                hist.append((step, float(loss.item())))
                if rank == 0:
                    log(f"step {step}/{nstep} loss {hist[-1][1]:.4e}")
    e_ev.record()
    torch.cuda.synchronize()
    ms = s_ev.elapsed_time(e_ev)
    meta = {"model": "linear correction", "npatch": npatch, "epochs": epochs, "batch": batch, "lr": lr,
            "seed": seed, "steps": nstep, "ranks": world, "train_ms": ms, "ms_per_step": ms / max(1, nstep),
            "data_s": t_data, "loss_history": hist}
    if out and rank == 0:
        flat = lin.params()
        flat.tofile(out + ".bin")
        with open(out + ".json", "w") as f:
            json.dump(dict(meta, nparams=int(flat.size), dtype="float32",
                           layout="W[class 0..3][row: output orbit][column: input orbit], orbit = z*16 + y*4 + x "
                                  "in the class representative's axes"), f, indent=1)
    return lin, meta


def load_lin(lin, path: str = DEFAULT_LIN):
    flat = np.fromfile(path + ".bin", dtype=np.float32)
    lin.set_params(flat)


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
    t.add_argument("--model", choices=("conv", "lin"), default="conv")
    t.add_argument("--npatch", type=int, default=1 << 20)
    t.add_argument("--epochs", type=int, default=None, help="default: conv 2, lin 64")
    t.add_argument("--batch", type=int, default=None, help="default: conv 1024, lin 2048")
    t.add_argument("--lr", type=float, default=None, help="default: conv 2e-3, lin 2e-3")
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", default=None, help="default: weights/learned_init (conv), weights/lin_correction (lin)")
    t.add_argument("--eval", type=int, default=65536, help="held-out patches evaluated after training (0: none)")
    e = sub.add_parser("eval")
    e.add_argument("--npatch", type=int, default=65536)
    e.add_argument("--weights", default=DEFAULT_WEIGHTS, help="conv net checkpoint ('' to skip)")
    e.add_argument("--lin", default=DEFAULT_LIN, help="linear correction checkpoint ('' to skip)")
    e.add_argument("--seed", type=int, default=99)
    tm = sub.add_parser("time", help="time the network's forward pass")
    tm.add_argument("--npatch", type=int, default=65536)
    tm.add_argument("--reps", type=int, default=5)
    tm.add_argument("--fused-only", action="store_true")
    a = ap.parse_args(argv)
    if a.cmd == "time":
        print(json.dumps(time_predict(a.npatch, a.reps, per_layer=not a.fused_only)))
    elif a.cmd == "train":
        conv = a.model == "conv"
        epochs = a.epochs if a.epochs is not None else (2 if conv else 64)
        lr = a.lr if a.lr is not None else 2e-3
        batch = a.batch if a.batch is not None else (1024 if conv else 2048)
        out = a.out if a.out is not None else (DEFAULT_WEIGHTS if conv else DEFAULT_LIN)
        fn = train if conv else train_lin
        model, meta = fn(a.npatch, epochs, batch, lr, a.seed, out)
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}))
            if a.eval:
                kw = {"net": model} if conv else {"lin": model}
                print(json.dumps(evaluate(npatch=a.eval, seed=99, **kw), indent=1))
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.barrier()
            dist.destroy_process_group()
    else:
        net = lin = None
        if a.weights:
            from gpg.net import Net
            net = Net(max_batch=4096)
            load(net, a.weights)
        if a.lin:
            from gpg.linear import LinearGuess
            lin = LinearGuess(max_batch=1)
            load_lin(lin, a.lin)
        print(json.dumps(evaluate(net, lin, a.npatch, a.seed), indent=1))
    return 0


if __name__ == "__main__":
    sys.exit(main())
