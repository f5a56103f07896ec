"""Patch sharding over ranks (one process per GPU).

Patches are independent (each reads only its own density, coarse potential
and fluid; ghost zones come from the coarse level through the inputs), so a
multi-GPU solve is a partition of the patch list with no exchange inside the
solve: rank r solves a contiguous range, the host scatters inputs and gathers
outputs.  Ranges are balanced by an estimated per-patch cost (cells x
expected sweeps) when one is given, else by count.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(npatch: int, world: int, cost=None) -> list[tuple[int, int]]:
    """Contiguous [start, stop) per rank covering 0..npatch exactly once."""
    if world < 1 or npatch < 0:
        raise ValueError("world >= 1 and npatch >= 0 required")
    if cost is None:
        base, extra = divmod(npatch, world)
        out, s = [], 0
        for r in range(world):
            n = base + (1 if r < extra else 0)
            out.append((s, s + n))
            s += n
        return out
    cost = np.asarray(cost, dtype=np.float64)
    if cost.shape != (npatch,) or (cost < 0).any():
        raise ValueError("cost must be a non-negative [npatch] array")
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")))
    cuts.append(npatch)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, npatch))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def patch_cost(ghost, expected_sweeps=None) -> np.ndarray:
    """Estimated cost per patch: interior cells x expected sweeps."""
    ghost = np.asarray(ghost)
    cells = (6 + 2 * ghost) ** 3
    sweeps = 1.0 if expected_sweeps is None else np.asarray(expected_sweeps, dtype=np.float64)
    return cells * sweeps


def scatter_solve_gather(arrays: dict, solve, group=None, src: int = 0, cost=None) -> dict | None:
    """Rank `src` holds full host arrays ({name: ndarray [P, ...]}); every rank
    receives its contiguous slice, runs `solve(slices) -> {name: ndarray}`
    locally, and `src` gathers the outputs in patch order.  Point-to-point
    transfers only; nothing is exchanged while ranks solve.  `cost` (on `src`:
    an estimated cost per patch, e.g. patch_cost of a mixed-ghost batch)
    balances the slices by cost instead of by count; `src` sends the bounds
    to every rank.  Returns the gathered outputs on `src`, None elsewhere."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    meta = [None]
    if rank == src:
        n = len(next(iter(arrays.values())))
        meta = [{k: (v.shape, str(v.dtype)) for k, v in arrays.items()} |
                {"__n": n, "__bounds": shard_bounds(n, world, cost)}]
    dist.broadcast_object_list(meta, src=src, group=group)
    meta = meta[0]
    n = meta.pop("__n")
    bounds = meta.pop("__bounds")
    lo, hi = bounds[rank]
    local = {}
    for k, (shape, dt) in meta.items():
        if rank == src:
            for r in range(world):
                if r == src:
                    continue
                a, b = bounds[r]
                dist.send(torch.from_numpy(np.ascontiguousarray(arrays[k][a:b])), dst=r, group=group)
            local[k] = np.ascontiguousarray(arrays[k][lo:hi])
        else:
            buf = torch.empty((hi - lo,) + tuple(shape[1:]), dtype=getattr(torch, dt))
            dist.recv(buf, src=src, group=group)
            local[k] = buf.numpy()
    out = solve(local)
    names = sorted(out)
    if rank == src:
        full = {}
        for k in names:
            v = out[k]
            full[k] = np.empty((n,) + v.shape[1:], dtype=v.dtype)
            full[k][lo:hi] = v
            for r in range(world):
                if r == src:
                    continue
                a, b = bounds[r]
                buf = torch.empty((b - a,) + v.shape[1:], dtype=torch.from_numpy(v[:0]).dtype)
                dist.recv(buf, src=r, group=group)
                full[k][a:b] = buf.numpy()
        return full
    for k in names:
        dist.send(torch.from_numpy(np.ascontiguousarray(out[k])), dst=src, group=group)
    return None


def allreduce_mean_(t, group=None):
    """In-place mean of tensor `t` over the ranks of `group` (the gradient
    exchange of data-parallel training: every rank ends with the same
    average).  A no-op without an initialised process group."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return t
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    w = dist.get_world_size(group)
    if w > 1:
        t.div_(w)
    return t
