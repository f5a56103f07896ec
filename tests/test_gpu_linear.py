"""Learned linear correction fused into ghost-1 FP32 SOR (gpg_lin_*), against
the CPU restatement oracle/lin_oracle.py and the library's own plain SOR.

* features (folded residual and target) are FP32 with the kernel's operand
  order: bit-identical to the oracle;
* with zero weights the correction vanishes and the fused solve must equal
  the plain interpolated-start solve bit for bit (same lane layout);
* with weights, the tensor cores sum the BF16 products in FP32 in their own
  order: the start differs from the oracle's FP64 sums by rounding only
  (tolerance stated per test), and the solve to the calibrated fixed residual
  agrees with the oracle's SOR from the oracle's start within the FP32
  tolerance of the path (relative L-inf 1e-5)."""
import numpy as np
import pytest

from gpg.abi import (GPG_ERR_CUDA, GPG_ERR_INVALID, GPG_INIT_INTERP, GPG_SOR, GPG_STOP_ABS_TOLERANCE,
                     GPG_STOP_POT_TOLERANCE, GPG_STOP_REFERENCE, GPG_STOP_TOLERANCE, default_params,
                     fixed_residual_params)
from gpg.inputs import log_uniform, make_patches

pytestmark = pytest.mark.gpu
CNST = float(np.float32(np.float32(4 * np.pi * 1e-5) * np.float32(1.0) * np.float32(1.0)))


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


@pytest.fixture(scope="module")
def lin(torch):
    from gpg.linear import LinearGuess
    m = LinearGuess(max_batch=256)
    yield m
    m.close()


def _patches(n, seed, fluid=False):
    rng = np.random.default_rng(seed + 5)
    return make_patches(n, 1, seed=seed, rho0=log_uniform(n, seed + 3), index=rng.uniform(1.5, 2.5, n),
                        fluid=fluid)


def _cubes(pin):
    from oracle.oracle import interp_cube
    return np.stack([interp_cube(c, 1, 4) for c in pin])


def _green():
    from oracle.lin_oracle import green_params
    return green_params().astype(np.float32).reshape(-1)


def test_features_bit_identical_to_oracle(torch, lin):
    from oracle import lin_oracle as lo
    d = _patches(37, 3)
    rng = np.random.default_rng(1)
    target = (d["pot_in"][:, 2:6, 2:6, 2:6].mean() * (1 + 1e-3 * rng.standard_normal((37, 8, 8, 8)))).astype(np.float32)
    p = fixed_residual_params(4, 1)
    u, t = lin.features(p, torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda(),
                        target=torch.from_numpy(target).cuda())
    torch.cuda.synchronize()
    cubes = _cubes(d["pot_in"])
    want_u = lo.features(cubes, d["rho"], CNST)
    want_t = lo.targets(cubes, target)
    assert np.array_equal(u.cpu().numpy(), want_u)
    assert np.array_equal(t.cpu().numpy(), want_t)


@pytest.mark.parametrize("stop", [GPG_STOP_REFERENCE, GPG_STOP_POT_TOLERANCE, GPG_STOP_TOLERANCE,
                                  GPG_STOP_ABS_TOLERANCE])
@pytest.mark.parametrize("gra", [0, 1])
def test_zero_weights_equal_interpolated_start(torch, lin, stop, gra):
    """W = 0: the start is the interpolated potential (+0), so every field,
    sweep count and residual equals the plain solve's."""
    from gpg.lib import solve_device
    lin.set_params(np.zeros(lin.nparams, dtype=np.float32))
    n = 45  # a partial last batch of the fused kernel
    d = _patches(n, 7, fluid=bool(gra))
    tol = {GPG_STOP_REFERENCE: 0.0, GPG_STOP_POT_TOLERANCE: 9.8e-7, GPG_STOP_TOLERANCE: 1e-4,
           GPG_STOP_ABS_TOLERANCE: 1e-9}[stop]
    p = default_params(4, 1, GPG_SOR, gra_acc=gra, gra_ghost=gra, init_mode=GPG_INIT_INTERP, stop_mode=stop,
                       sor_tolerance=tol, sor_min_iter=1 if stop else 10, sor_max_iter=200)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    flu_a = torch.from_numpy(d["flu"].copy()).cuda() if gra else None
    flu_b = torch.from_numpy(d["flu"].copy()).cuda() if gra else None
    pa, fa, ia, ra = solve_device(p, rho, pin, flu=flu_a)
    pb, fb, ib, rb = lin.solve(p, rho, pin, flu=flu_b)
    torch.cuda.synchronize()
    lin.check()
    assert torch.equal(ia, ib) and torch.equal(ra, rb)
    assert torch.equal(pa, pb)
    if gra:
        assert torch.equal(fa, fb)


def test_start_matches_oracle(torch, lin):
    """Max_Iter 0 returns the start itself: interpolation + unfold(W fold(r0))."""
    from oracle import lin_oracle as lo
    lin.set_params(_green())
    d = _patches(29, 11)
    p = fixed_residual_params(4, 1, sor_max_iter=0)
    pot, _, it, _ = lin.solve(p, torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda())
    torch.cuda.synchronize()
    lin.check()
    got = pot.cpu().numpy().astype(np.float64)
    cubes = _cubes(d["pot_in"])
    want = lo.learned_start(_green(), cubes, d["rho"], CNST).astype(np.float64)
    interp = cubes[:, 1:-1, 1:-1, 1:-1].astype(np.float64)
    # the correction (want - interp) agrees to FP32 accumulation rounding
    corr = np.abs(want - interp).reshape(29, -1).max(1)
    diff = np.abs(got - want).reshape(29, -1).max(1)
    assert (it.cpu().numpy() == 0).all()
    assert (diff <= 1e-4 * corr + 2 * np.spacing(np.abs(want).reshape(29, -1).max(1).astype(np.float32))).all(), \
        (diff / np.maximum(corr, 1e-30)).max()


def test_solve_matches_oracle_sor_from_oracle_start(torch, lin):
    from oracle import lin_oracle as lo
    from oracle.oracle import run_oracle
    lin.set_params(_green())
    n = 64
    d = _patches(n, 13)
    p = fixed_residual_params(4, 1)
    pot, _, it, _ = lin.solve(p, torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda())
    torch.cuda.synchronize()
    lin.check()
    start = lo.learned_start(_green(), _cubes(d["pot_in"]), d["rho"], CNST).astype(np.float32)
    from gpg.abi import GPG_INIT_GUESS
    q = fixed_residual_params(4, 1, init_mode=GPG_INIT_GUESS)
    opot, _, oit, _ = run_oracle(q, d["rho"], d["pot_in"], guess=np.ascontiguousarray(start))
    got = pot.cpu().numpy().reshape(n, -1).astype(np.float64)
    want = opot.reshape(n, -1).astype(np.float64)
    rel = np.abs(got - want).max(1) / np.abs(want).max(1)
    assert rel.max() < 1e-5, rel.max()
    gi = it.cpu().numpy()
    assert np.mean(np.abs(gi - oit) <= 1) == 1.0 and np.mean(gi == oit) >= 0.9, (gi, oit)


def test_gradients_match_oracle(torch, lin):
    from oracle import lin_oracle as lo
    rng = np.random.default_rng(5)
    w = (0.02 * rng.standard_normal(lin.nparams)).astype(np.float32)
    lin.set_params(w)
    n = 96
    u = rng.standard_normal((n, 8, 64)).astype(np.float32) * np.float32(10.0) ** rng.uniform(-6, 0, (n, 1, 1)).astype(np.float32)
    t = rng.standard_normal((n, 8, 64)).astype(np.float32) * np.abs(u).max((1, 2), keepdims=True) * np.float32(0.05)
    grad = torch.empty(lin.nparams, device="cuda")
    loss = torch.empty(1, device="cuda")
    lin.gradients(torch.from_numpy(u).cuda(), torch.from_numpy(t).cuda(), grad=grad, loss=loss)
    torch.cuda.synchronize()
    want_loss, want_grad = lo.gradients(w, u, t)
    assert abs(loss.item() - want_loss) <= 1e-5 * want_loss
    g = grad.cpu().numpy().astype(np.float64).reshape(-1)
    assert np.linalg.norm(g - want_grad.reshape(-1)) <= 1e-5 * np.linalg.norm(want_grad)


def test_training_recovers_the_correction(torch, lin):
    """A short training run on the plain SOR's own FP64 solutions drives the
    loss down, W towards the exact correction (minus the inverse Laplacian of
    the interior, block form; the full 64-epoch run lands within 0.04 % of
    it) and the held-out start far below the interpolated start's error."""
    import learned
    from gpg.linear import LinearGuess
    from oracle.lin_oracle import green_params
    m = LinearGuess(max_batch=1024)
    rho, pin = learned.dataset(16384, 21)
    u, t = learned.lin_data(m, torch.from_numpy(rho).cuda(), torch.from_numpy(pin).cuda())
    loss = torch.empty(1, device="cuda")
    first = None
    nstep = 6000
    for step in range(nstep):
        sl = slice((step % 16) * 1024, (step % 16 + 1) * 1024)
        m.train_step(u[sl], t[sl], 2e-3 * 0.5 * (1 + np.cos(np.pi * step / nstep)), loss=loss)
        if step == 0:
            first = loss.item()
    m.gradients(u[:1024], t[:1024], loss=loss)
    last = loss.item()
    assert last < 0.1 * first, (first, last)
    w = m.params().reshape(4, 64, 64).astype(np.float64)
    g = green_params()
    assert np.linalg.norm(w - g) < 0.6 * np.linalg.norm(g), np.linalg.norm(w - g) / np.linalg.norm(g)
    # held-out patches: the learned start is far closer to the FP64 solution
    # than the interpolated start it corrects
    from gpg.lib import solve_device
    rho, pin = learned.dataset(2048, 23)
    rho, pin = torch.from_numpy(rho).cuda(), torch.from_numpy(pin).cuda()
    sol = solve_device(default_params(8, 1, GPG_SOR, gra_acc=0, gra_ghost=0), rho.double(), pin.double())[0]
    p0 = fixed_residual_params(4, 1, sor_max_iter=0)
    learned_start = m.solve(p0, rho, pin)[0].double()
    interp_start = solve_device(p0, rho, pin)[0].double()
    e_l = (learned_start - sol).abs().amax(dim=(1, 2, 3)) / sol.abs().amax(dim=(1, 2, 3))
    e_i = (interp_start - sol).abs().amax(dim=(1, 2, 3)) / sol.abs().amax(dim=(1, 2, 3))
    assert e_l.median().item() < 0.2 * e_i.median().item(), (e_l.median().item(), e_i.median().item())
    m.close()


def test_bounded_wait_reports_timeout_and_recovers(torch, lin):
    """The kernel's bounded tensor-core wait: a wait on a barrier nothing
    signals gives up after a few polls, the solve still completes through the
    normal path, gpg_lin_check reports GPG_ERR_CUDA once, and the next solve
    is clean."""
    from gpg.lib import GpgError
    lin.set_params(np.zeros(lin.nparams, dtype=np.float32))
    d = _patches(16, 17)
    p = fixed_residual_params(4, 1, init_mode=GPG_INIT_INTERP)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    ref = lin.solve(p, rho, pin)[0].clone()
    lin.set_wait_probe(4)
    pot = lin.solve(p, rho, pin)[0]
    torch.cuda.synchronize()
    with pytest.raises(GpgError) as ei:
        lin.check()
    assert ei.value.status == GPG_ERR_CUDA
    assert torch.equal(pot, ref)
    lin.set_wait_probe(0)
    pot = lin.solve(p, rho, pin)[0]
    torch.cuda.synchronize()
    lin.check()
    assert torch.equal(pot, ref)


def test_rejects_other_shapes(torch, lin):
    from gpg.lib import GpgError
    d = _patches(8, 1)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    for kw in ({"ghost": 2}, {"real_size": 8}):
        p = default_params(kw.get("real_size", 4), kw.get("ghost", 1), GPG_SOR)
        with pytest.raises(GpgError):
            lin.solve(p, rho, pin)


def test_launch_shapes_give_the_same_bits(torch, lin):
    """Every launch shape of the fused solve (staged or not, 2 or 3 groups of
    teams per SM) computes each patch the same way: identical results."""
    lin.set_params(_green())
    d = _patches(203, 31)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    p = fixed_residual_params(4, 1)
    outs = []
    try:
        for v in range(lin.variant_count()):
            lin.set_variant(v)
            pot, _, it, rs = lin.solve(p, rho, pin)
            torch.cuda.synchronize()
            lin.check()
            outs.append((pot.clone(), it.clone(), rs.clone()))
    finally:
        lin.set_variant(0)
    assert len(outs) >= 2
    for o in outs[1:]:
        assert all(torch.equal(a, b) for a, b in zip(o, outs[0]))


def test_trained_correction_doubles_throughput(torch):
    """The committed checkpoint on held-out patches, every start to the same
    calibrated fixed residual: the learned start reaches it with at least twice
    the patches/s of the zero-start plain SOR, in fewer sweeps than the
    interpolated start, with the FP64 error of the zero start or better (median;
    the maximum within 25 % of it and inside the 1e-5 FP32 bound)."""
    import learned
    from gpg.linear import LinearGuess
    lin = LinearGuess(max_batch=1)
    learned.load_lin(lin)
    r = learned.evaluate(lin=lin, npatch=32768, seed=77, reps=10, rule=False)
    lin.close()
    z, i, l = r["plain_zero_start"], r["plain_interpolated_start"], r["learned_linear"]
    assert l["patches_per_s"] >= 2.0 * z["patches_per_s"], r
    assert l["sweeps"]["mean"] < 0.5 * i["sweeps"]["mean"] and i["sweeps"]["mean"] < z["sweeps"]["mean"], r
    assert l["rel_linf_vs_fp64"]["p50"] <= z["rel_linf_vs_fp64"]["p50"], r
    assert l["rel_linf_vs_fp64"]["max"] <= 1.25 * z["rel_linf_vs_fp64"]["max"] and l["rel_linf_vs_fp64"]["max"] < 1e-5, r


def test_non_finite_input_stays_in_its_patch(torch, lin):
    """A NaN density cell poisons only its own patch: the fold and the unfold
    stay inside the patch and each patch is its own MMA column, so every
    other patch of the batch gives the same bits as without it."""
    lin.set_params(_green())
    d = _patches(24, 41)
    p = fixed_residual_params(4, 1, sor_max_iter=60)
    rho = torch.from_numpy(d["rho"]).cuda()
    pin = torch.from_numpy(d["pot_in"]).cuda()
    ref, _, ref_it, _ = lin.solve(p, rho, pin)
    ref, ref_it = ref.clone(), ref_it.clone()
    bad = rho.clone()
    bad[5, 3, 4, 2] = float("nan")
    pot, _, it, _ = lin.solve(p, bad, pin)
    torch.cuda.synchronize()
    lin.check()
    keep = [i for i in range(24) if i != 5]
    assert torch.equal(pot[keep], ref[keep]) and torch.equal(it[keep], ref_it[keep])
    assert torch.isnan(pot[5]).any() and int(it[5]) == 60


def test_misaligned_inputs_are_rejected(torch, lin):
    """The fused kernel stages whole patches with bulk copies (16-byte
    aligned): a misaligned input pointer is an argument error, not a fault."""
    import ctypes as C
    from gpg.linear import _lin_lib
    d = _patches(8, 43)
    rho = torch.from_numpy(np.concatenate([np.zeros(1, np.float32), d["rho"].reshape(-1)])).cuda()
    pin = torch.from_numpy(d["pot_in"]).cuda()
    out = torch.empty((8, 8, 8, 8), device="cuda")
    p = fixed_residual_params(4, 1)
    lib = _lin_lib()
    rc = lib.gpg_lin_solve_device(lin._l, C.byref(p), 8, C.c_void_p(rho.data_ptr() + 4), C.c_void_p(pin.data_ptr()),
                                  C.c_void_p(out.data_ptr()), None, None, None,
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == GPG_ERR_INVALID and b"aligned" in lib.gpg_lin_last_error()


def test_data_parallel_training_under_torchrun(torch, tmp_path):
    """learned.py train --model lin under torchrun (NCCL process group, one
    rank here: per-rank gradients, the all-reduce, the shared Adam step) saves
    the same weights as the single-process run of the same configuration."""
    import os
    import socket
    import subprocess
    import sys
    import learned
    script = os.path.join(os.path.dirname(learned.__file__), "learned.py")
    args = ["train", "--model", "lin", "--npatch", "65536", "--epochs", "1", "--batch", "2048", "--eval", "0"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r1 = subprocess.run([sys.executable, script] + args + ["--out", str(tmp_path / "single")], env=env,
                        capture_output=True, text=True, timeout=600)
    assert r1.returncode == 0, r1.stderr[-2000:]
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    r2 = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "1",
                         "--master-addr", "127.0.0.1", "--master-port", str(port), script] + args +
                        ["--out", str(tmp_path / "dp")], env=env, capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr[-2000:]
    w1 = np.fromfile(str(tmp_path / "single.bin"), dtype=np.float32)
    w2 = np.fromfile(str(tmp_path / "dp.bin"), dtype=np.float32)
    assert w1.size == w2.size == 16384 and np.array_equal(w1, w2)
