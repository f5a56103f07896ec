"""Batched mixed-ghost-size SOR in one persistent launch (needs a B200).

Each patch of a mixed batch must come out bit-identical to solving its group
alone with the per-ghost-size kernel, and match the oracle; the CUDA-graph
plan must replay the same result."""
import numpy as np
import pytest

from gpg.abi import GPG_INIT_ZERO, GPG_SOR, GPG_STOP_ABS_TOLERANCE, default_params
from gpg.inputs import log_uniform, make_patches, mixed_ghost_assignment
from oracle.oracle import run_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def build_groups(torch, rs, npatch, seed, gra_acc, dev):
    gh = mixed_ghost_assignment(npatch, seed)
    rho0 = log_uniform(npatch, seed + 1)
    dt = np.float32 if rs == 4 else np.float64
    tdt = torch.float32 if rs == 4 else torch.float64
    groups, host = [], []
    for g in range(1, 6):
        idx = np.flatnonzero(gh == g)
        d = make_patches(len(idx), g, seed=seed + 10 * g, rho0=rho0[idx], dtype=dt)
        n = len(idx)
        t = {"ghost": g, "rho": torch.from_numpy(d["rho"]).to(dev), "pot_in": torch.from_numpy(d["pot_in"]).to(dev),
             "pot_out": torch.zeros((n, 10, 10, 10), dtype=tdt, device=dev),
             "iters": torch.zeros(n, dtype=torch.int32, device=dev),
             "resid": torch.zeros(n, dtype=torch.float64, device=dev)}
        if gra_acc:
            t["flu"] = torch.from_numpy(d["flu"].copy()).to(dev)
        groups.append(t)
        host.append(d)
    return groups, host


@pytest.mark.parametrize("rs", [4, 8])
def test_batch_bit_identical_to_single_kernels(torch, rs):
    from gpg.lib import solve_batch_device, solve_device
    dev = torch.device("cuda:0")
    tol = 1e-4 if rs == 4 else 1e-10
    p = default_params(rs, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_ABS_TOLERANCE,
                       sor_tolerance=tol, sor_min_iter=1, sor_max_iter=200)
    groups, host = build_groups(torch, rs, 203, seed=31, gra_acc=True, dev=dev)
    flu0 = [g["flu"].clone() for g in groups]
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    solve_batch_device(p, groups, counter)
    torch.cuda.synchronize()
    for g, f0 in zip(groups, flu0):
        q = p.copy(ghost=g["ghost"], sor_omega={1: 1.49, 2: 1.57, 3: 1.62, 4: 1.65, 5: 1.69}[g["ghost"]])
        pot, flu, it, rsd = solve_device(q, g["rho"], g["pot_in"], flu=f0)
        torch.cuda.synchronize()
        assert torch.equal(pot, g["pot_out"]), g["ghost"]
        assert torch.equal(flu, g["flu"]), g["ghost"]
        assert torch.equal(it, g["iters"]) and torch.equal(rsd, g["resid"])
    its = np.concatenate([g["iters"].cpu().numpy() for g in groups])
    assert its.max() >= 2 * max(1, its.min())  # rho0 over 4 decades: counts spread widely


def test_batch_matches_oracle(torch):
    from gpg.lib import solve_batch_device
    dev = torch.device("cuda:0")
    p = default_params(4, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_ABS_TOLERANCE,
                       sor_tolerance=1e-4, sor_min_iter=1, sor_max_iter=200, gra_acc=0)
    groups, host = build_groups(torch, 4, 97, seed=77, gra_acc=False, dev=dev)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    solve_batch_device(p, groups, counter)
    torch.cuda.synchronize()
    for g, d in zip(groups, host):
        q = p.copy(ghost=g["ghost"], sor_omega={1: 1.49, 2: 1.57, 3: 1.62, 4: 1.65, 5: 1.69}[g["ghost"]])
        op, _, oi, _ = run_oracle(q, d["rho"], d["pot_in"], accum_f64=True)
        gi = g["iters"].cpu().numpy()
        same = gi == oi
        assert same.mean() >= 0.99
        assert np.array_equal(g["pot_out"].cpu().numpy()[same], op[same])


@pytest.mark.parametrize("mode", [0, 1])
def test_batch_plan_graph_replay(torch, mode):
    from gpg.lib import BatchPlan, solve_batch_device
    dev = torch.device("cuda:0")
    p = default_params(4, 1, GPG_SOR, gra_acc=0)
    groups, _ = build_groups(torch, 4, 150, seed=5, gra_acc=False, dev=dev)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    solve_batch_device(p, groups, counter)
    torch.cuda.synchronize()
    want = [g["pot_out"].clone() for g in groups]
    plan = BatchPlan(p, groups, mode=mode)
    for g in groups:
        g["pot_out"].zero_()
    plan.launch()
    torch.cuda.synchronize()
    assert all(torch.equal(a, g["pot_out"]) for a, g in zip(want, groups))
    for g in groups:
        g["pot_out"].zero_()
    plan.launch()
    plan.launch()
    torch.cuda.synchronize()
    assert all(torch.equal(a, g["pot_out"]) for a, g in zip(want, groups))
    plan.close()


def test_batch_rejects_bad_input(torch):
    from gpg.lib import GpgError, solve_batch_device
    dev = torch.device("cuda:0")
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    groups, _ = build_groups(torch, 4, 40, seed=9, gra_acc=False, dev=dev)
    with pytest.raises(GpgError):  # gravity requested but no fluid arrays
        solve_batch_device(default_params(4, 1, GPG_SOR), groups, counter)
    from gpg.abi import GPG_MG
    with pytest.raises(GpgError):  # multigrid is not batched
        solve_batch_device(default_params(4, 1, GPG_MG, gra_acc=0), groups, counter)
    solve_batch_device(default_params(4, 1, GPG_SOR, gra_acc=0), [], counter)  # empty batch
