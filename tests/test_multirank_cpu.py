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


def _mixed_worker(rank, world, port, q):
    """A mixed-ghost batch (each patch's arrays padded to the largest shape)
    split by cost: ranks get unequal patch counts and the gathered result is
    the single-process one."""
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "gpu_testbed_poisson-gravity_b200"))
    import torch.distributed as dist
    from gpg.abi import GPG_SOR, default_params
    from gpg.inputs import make_patches
    from gpg.shard import patch_cost, scatter_solve_gather
    from oracle.oracle import run_oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ghosts = np.array([1] * 12 + [5] * 4 + [3] * 8, dtype=np.int32)
    arrays, cost = None, None
    if rank == 0:
        rho = np.zeros((len(ghosts), 16 ** 3), np.float32)
        pin = np.zeros((len(ghosts), 12 ** 3), np.float32)
        for i, g in enumerate(ghosts):
            d = make_patches(1, int(g), seed=40 + i, fluid=False)
            rho[i, :d["rho"].size] = d["rho"].reshape(-1)
            pin[i, :d["pot_in"].size] = d["pot_in"].reshape(-1)
        arrays = {"ghost": ghosts, "rho": rho, "pot_in": pin}
        cost = patch_cost(ghosts)

    def solve_one(g, rho, pin):
        m, pn = 6 + 2 * g, 4 + 2 * ((g + 3) // 2)
        p = default_params(4, g, GPG_SOR, gra_acc=0, gra_ghost=0)
        pot, _, it, _ = run_oracle(p, np.ascontiguousarray(rho[:, :m ** 3].reshape(-1, m, m, m)),
                                   np.ascontiguousarray(pin[:, :pn ** 3].reshape(-1, pn, pn, pn)))
        return pot.reshape(len(rho), -1)[:, :512], it

    def solve(local):
        pots = np.zeros((len(local["ghost"]), 512), np.float32)
        its = np.zeros(len(local["ghost"]), np.int32)
        for g in np.unique(local["ghost"]):
            sel = local["ghost"] == g
            pots[sel], its[sel] = solve_one(int(g), local["rho"][sel], local["pot_in"][sel])
        return {"pot": pots, "iters": its, "count": np.full(len(its), len(its), np.int32)}

    out = scatter_solve_gather(arrays, solve, cost=cost)
    if rank == 0:
        want = solve({"ghost": ghosts, "rho": arrays["rho"], "pot_in": arrays["pot_in"]})
        counts = sorted(set(out["count"].tolist()))
        q.put(bool(np.array_equal(out["pot"], want["pot"]) and np.array_equal(out["iters"], want["iters"])
                   and len(counts) == 2))
    dist.barrier()
    dist.destroy_process_group()


def test_cost_balanced_scatter_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mixed_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=120)
    assert all(pr.exitcode == 0 for pr in procs)
    assert q.get(timeout=5) is True


def _mean_worker(rank, world, port, q):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "gpu_testbed_poisson-gravity_b200"))
    import torch
    import torch.distributed as dist
    from gpg.shard import allreduce_mean_
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g = torch.arange(5, dtype=torch.float32) * (rank + 1)      # rank-dependent "gradient"
    allreduce_mean_(g)
    q.put((rank, g.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_gradient_mean_gloo_world2():
    """The gradient exchange of data-parallel training: every rank ends with
    the same mean of the ranks' gradients."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mean_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    want = [1.5 * i for i in range(5)]
    assert got[0] == want and got[1] == want


def test_training_shards_cover_the_set():
    """Rank shards of the learned guess's training set are whole chunks that
    cover it once, and a shard's patches are the whole set's patches there."""
    import learned
    C = learned.CHUNK
    for n in (C, 3 * C + 5, 16 * C):
        for w in (1, 2, 3):
            if w > (n + C - 1) // C:
                continue
            b = [learned.shard(n, r, w) for r in range(w)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
            assert all(lo % C == 0 for lo, _ in b)
    with pytest.raises(ValueError):
        learned.shard(C, 0, 2)
    n = C + 40
    full_rho, full_pin = learned.dataset(n, 5)
    part_rho, part_pin = learned.dataset(n, 5, first=C, stop=n)
    assert np.array_equal(part_rho, full_rho[C:]) and np.array_equal(part_pin, full_pin[C:])
    with pytest.raises(ValueError):
        learned.dataset(n, 5, first=7, stop=n)
