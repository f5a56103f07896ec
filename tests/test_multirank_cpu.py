"""Multi-rank patch sharding on CPU (gloo, world size 2): partition logic and
the scatter -> local solve -> gather path.  The local solve here is the CPU
oracle (test infrastructure); on GPUs each rank calls libgpg instead."""
import os
import socket

import numpy as np
import pytest

from gpg.shard import patch_cost, shard_bounds


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 64, 1001):
        for w in (1, 2, 3, 8):
            b = shard_bounds(n, w)
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
            sizes = [hi - lo for lo, hi in b]
            assert max(sizes) - min(sizes) <= 1


def test_cost_balanced_bounds():
    rng = np.random.default_rng(0)
    g = rng.integers(1, 6, size=1000)
    cost = patch_cost(g, expected_sweeps=rng.uniform(10, 100, size=1000))
    b = shard_bounds(1000, 4, cost)
    per = [cost[lo:hi].sum() for lo, hi in b]
    assert b[0][0] == 0 and b[-1][1] == 1000
    assert max(per) / min(per) < 1.1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "gpu_testbed_poisson-gravity_b200"))
    import torch.distributed as dist
    from gpg.abi import GPG_SOR, default_params
    from gpg.inputs import make_patches
    from gpg.shard import scatter_solve_gather
    from oracle.oracle import run_oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p = default_params(4, 2, GPG_SOR)
    arrays = None
    if rank == 0:
        d = make_patches(21, 2, seed=3)
        arrays = {"rho": d["rho"], "pot_in": d["pot_in"], "flu": d["flu"]}

    def solve(local):
        pot, flu, it, _ = run_oracle(p, local["rho"], local["pot_in"], flu=local["flu"].copy())
        return {"pot_out": pot, "flu": flu, "iters": it}

    out = scatter_solve_gather(arrays, solve)
    if rank == 0:
        pot, flu, it, _ = run_oracle(p, arrays["rho"], arrays["pot_in"], flu=arrays["flu"].copy())
        q.put(bool(np.array_equal(out["pot_out"], pot) and np.array_equal(out["flu"], flu)
                   and np.array_equal(out["iters"], it)))
    dist.barrier()
    dist.destroy_process_group()


def test_scatter_solve_gather_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=120)
    assert all(pr.exitcode == 0 for pr in procs)
    assert q.get(timeout=5) is True
