"""Learned initial guess: tensor-core network vs its FP64 oracle (needs a B200).

The oracle (oracle/convnet_oracle.py) rounds to bfloat16 where the kernels
store bfloat16; what remains are FP32-vs-FP64 accumulation differences (which
now and then flip one bfloat16 rounding of an activation), so the checks are
relative L2 errors.  Measured on B200 over four seeds: forward <= 6.3e-4,
weight and bias gradients <= 2.3e-4, loss <= 1.6e-6; the tolerances below
are 3-10x those."""
import numpy as np
import pytest

from gpg.inputs import make_patches

pytestmark = pytest.mark.gpu
CNST = np.float32(4 * np.pi * 1e-5)  # Poi_Coeff * dh^2 in float


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def _data(n, seed):
    d = make_patches(n, 1, seed=seed, fluid=False)
    rng = np.random.default_rng(seed)
    target = (d["pot_in"][:, :, :, :].mean() * (1 + 0.1 * rng.standard_normal((n, 8, 8, 8)))).astype(np.float32)
    return d["rho"], d["pot_in"], target


def _oracle_inputs(rho, pot_in):
    from oracle.oracle import interp_cube
    from oracle.convnet_oracle import make_input
    cubes = np.stack([interp_cube(p, 1, 4) for p in pot_in])
    return make_input(rho, cubes, CNST)


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.mark.parametrize("seed", [11, 33])
def test_forward_matches_oracle(torch, seed):
    from gpg.net import Net, split_params
    from oracle.convnet_oracle import forward
    rho, pin, _ = _data(3, seed)
    net = Net(max_batch=4, seed=seed % 7 + 1)
    ws, bs = split_params(net.params().astype(np.float64))
    guess = torch.empty((3, 8, 8, 8), device="cuda")
    net.predict(torch.from_numpy(rho).cuda(), torch.from_numpy(pin).cuda(), guess, float(CNST))
    torch.cuda.synchronize()
    net.check()
    x0, s = _oracle_inputs(rho, pin)
    _, y4 = forward(x0, ws, bs)
    want = y4[:, 1:-1, 1:-1, 1:-1, 0] * s[:, None, None, None]
    assert rel(guess.cpu().numpy(), want) < 2e-3
    net.close()


@pytest.mark.parametrize("seed", [21, 33])
def test_gradients_match_oracle(torch, seed):
    from gpg.net import Net, split_params
    from oracle.convnet_oracle import loss_and_grads
    rho, pin, tgt = _data(3, seed)
    net = Net(max_batch=4, seed=seed % 7 + 1)
    p = net.params()
    ws, bs = split_params(p.astype(np.float64))
    grad = torch.empty(net.nparams, device="cuda")
    loss = torch.empty(1, device="cuda")
    net.gradients(torch.from_numpy(rho).cuda(), torch.from_numpy(pin).cuda(), torch.from_numpy(tgt).cuda(),
                  float(CNST), grad=grad, loss=loss)
    torch.cuda.synchronize()
    net.check()
    x0, s = _oracle_inputs(rho, pin)
    ol, odw, odb = loss_and_grads(x0, ws, bs, tgt, s)
    assert abs(loss.item() - ol) <= 2e-5 * abs(ol)
    gws, gbs = split_params(grad.cpu().numpy().astype(np.float64))
    for l in range(4):
        assert rel(gws[l], odw[l]) < 1e-3, (l, rel(gws[l], odw[l]))
        assert rel(gbs[l], odb[l]) < 1e-3, (l, rel(gbs[l], odb[l]))
    net.close()


def test_training_reduces_loss(torch):
    from gpg.net import Net
    d = make_patches(64, 1, seed=31, fluid=False)
    from gpg.abi import GPG_INIT_ZERO, GPG_SOR, GPG_STOP_TOLERANCE, default_params
    from gpg.lib import solve_device
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    p = default_params(4, 1, GPG_SOR, gra_acc=0, gra_ghost=0, init_mode=GPG_INIT_ZERO,
                       stop_mode=GPG_STOP_TOLERANCE, sor_tolerance=0.02, sor_min_iter=1, sor_max_iter=200)
    pot, _, _, _ = solve_device(p, rho, pin)          # GRA window = the 8^3 interior
    target = pot.contiguous()
    net = Net(max_batch=64, seed=7)
    loss = torch.empty(1, device="cuda")
    first = None
    for it in range(60):
        net.train_step(rho, pin, target, float(CNST), 1e-3, loss=loss)
        if first is None:
            torch.cuda.synchronize()
            first = loss.item()
    torch.cuda.synchronize()
    net.check()
    assert loss.item() < 0.5 * first
    net.close()


@pytest.mark.parametrize("npatch", [1, 150, 1000])
def test_fused_predict_matches_layers(torch, npatch):
    """The one-kernel forward pass equals the per-layer kernels bit for bit
    (1 patch; fewer patches than SMs; several patches per CTA, so the weight
    ring wraps across layers and patches)."""
    from gpg.inputs import log_uniform
    from gpg.net import Net
    rng = np.random.default_rng(npatch)
    d = make_patches(npatch, 1, seed=40 + npatch, rho0=log_uniform(npatch, 5), index=rng.uniform(1.5, 2.5, npatch),
                     fluid=False)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    net = Net(max_batch=256, seed=9)
    p = net.params()
    p += 0.05 * rng.standard_normal(p.size).astype(np.float32)   # every bias and weight non-trivial
    net.set_params(p)
    fused = torch.full((npatch, 8, 8, 8), float("nan"), device="cuda")
    layers = torch.full((npatch, 8, 8, 8), float("nan"), device="cuda")
    net.predict(rho, pin, fused, float(CNST))
    net.predict(rho, pin, layers, float(CNST), fused=False)
    torch.cuda.synchronize()
    net.check()
    assert not torch.isnan(fused).any()
    assert torch.equal(fused, layers)
    net.close()


def test_learned_guess_reduces_sweeps(torch):
    """A network trained briefly on the plain SOR's own solutions (ghost 1,
    rho0 log-uniform, power index in [1.5, 2.5]) starts the SOR closer to the
    solution: fewer sweeps to the calibrated fixed residual on held-out
    patches, at the same error against the FP64 solution.  (Its inference
    costs far more than the sweeps it saves: the throughput comparison is
    recorded by learned.evaluate and asserted for the linear correction.)"""
    import learned
    net, meta = learned.train(npatch=65536, epochs=2, batch=512, lr=2e-3, seed=3, out=None, log=lambda *a: None)
    assert meta["loss_history"][-1][1] < 0.1 * meta["loss_history"][0][1] or meta["loss_history"][-1][1] < 1e-3
    r = learned.evaluate(net=net, npatch=4096, seed=77, reps=1, rule=False)
    plain, guess = r["plain_zero_start"], r["learned_conv"]
    assert guess["sweeps"]["mean"] < 0.85 * plain["sweeps"]["mean"], r
    assert guess["sweeps"]["p50"] < plain["sweeps"]["p50"], r
    # both stop at the same fixed residual: same error scale against FP64
    assert guess["rel_linf_vs_fp64"]["max"] <= 3 * plain["rel_linf_vs_fp64"]["max"] + 1e-6, r
    net.close()


def test_fused_predict_after_other_kernels(torch):
    """The fused kernel reads no shared memory it has not written: its result
    is the same right after the per-layer kernels and the SOR solver have left
    their own data in every SM's shared memory."""
    from gpg.abi import GPG_SOR, default_params
    from gpg.lib import solve_device
    from gpg.net import Net
    n = 592
    d = make_patches(n, 1, seed=78, fluid=False)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    net = Net(max_batch=n, seed=6)
    layers = torch.empty((n, 8, 8, 8), device="cuda")
    net.predict(rho, pin, layers, float(CNST), fused=False)
    for other in ("layers", "sor"):
        if other == "sor":
            solve_device(default_params(4, 1, GPG_SOR, gra_acc=0, gra_ghost=0), rho, pin)
        else:
            net.predict(rho, pin, torch.empty_like(layers), float(CNST), fused=False)
        fused = torch.full((n, 8, 8, 8), float("nan"), device="cuda")
        net.predict(rho, pin, fused, float(CNST))
        torch.cuda.synchronize()
        net.check()
        assert torch.equal(fused, layers), other
    net.close()


def test_fused_predict_cold_weights(torch):
    """The weight ring's copies come from HBM when L2 holds other data: the
    tensor core must still only read a slot after its copy has landed (L2 is
    flushed by a 512 MB write before each call)."""
    from gpg.net import Net
    n = 1184  # 8 patches per CTA on 148 SMs
    d = make_patches(n, 1, seed=77, fluid=False)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    net = Net(max_batch=n, seed=4)
    layers = torch.empty((n, 8, 8, 8), device="cuda")
    net.predict(rho, pin, layers, float(CNST), fused=False)
    flush = torch.empty(128 * 2 ** 20, dtype=torch.float32, device="cuda")
    for _ in range(3):
        flush.fill_(1.0)
        fused = torch.full((n, 8, 8, 8), float("nan"), device="cuda")
        net.predict(rho, pin, fused, float(CNST))
        torch.cuda.synchronize()
        net.check()
        assert torch.equal(fused, layers)
    net.close()


def test_net_rejects_bad_input(torch):
    """Invalid sizes and NULL arrays come back as status codes with a message,
    never as a launch; zero patches is a no-op."""
    import ctypes as C
    from gpg.lib import GpgError
    from gpg.net import Net, _net_lib
    lib = _net_lib()
    bad = C.c_void_p()
    assert lib.gpg_net_create(C.byref(bad), 0, 1, 0) != 0
    assert b"max_batch" in lib.gpg_net_last_error()
    net = Net(max_batch=4, seed=2)
    assert lib.gpg_net_predict(net._n, 3, None, None, None, 1.0, None) != 0
    assert b"NULL" in lib.gpg_net_last_error()
    assert lib.gpg_net_predict(net._n, -1, None, None, None, 1.0, None) != 0
    assert lib.gpg_net_predict(net._n, 0, None, None, None, 1.0, None) == 0
    d = make_patches(8, 1, seed=3, fluid=False)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    with pytest.raises(GpgError):
        net.train_step(rho, pin, torch.zeros((8, 8, 8, 8), device="cuda"), float(CNST), 1e-3)   # 8 > max_batch
    assert lib.gpg_net_predict(None, 1, None, None, None, 1.0, None) != 0
    guess = torch.empty((8, 8, 8, 8), device="cuda")
    net.predict(rho, pin, guess, float(CNST))   # predict has no max_batch limit
    torch.cuda.synchronize()
    net.check()
    assert torch.isfinite(guess).all()
    net.close()


def test_gradient_then_apply_equals_train_step(torch):
    """gpg_net_gradients + gpg_net_apply_gradient (the data-parallel split,
    with the all-reduce in between) reproduces gpg_net_train_step bit for bit."""
    from gpg.net import Net
    d = make_patches(32, 1, seed=12, fluid=False)
    rho, pin = torch.from_numpy(d["rho"]).cuda(), torch.from_numpy(d["pot_in"]).cuda()
    tgt = (pin.mean() * (1 + 0.05 * torch.randn((32, 8, 8, 8), device="cuda",
                                                generator=torch.Generator(device="cuda").manual_seed(1)))).contiguous()
    a, b = Net(max_batch=32, seed=8), Net(max_batch=32, seed=8)
    grad = torch.empty(a.nparams, device="cuda")
    for it in range(3):
        a.train_step(rho, pin, tgt, float(CNST), 1e-3)
        b.gradients(rho, pin, tgt, float(CNST), grad=grad)
        b.apply_gradient(grad, 1e-3)
    torch.cuda.synchronize()
    a.check()
    b.check()
    assert np.array_equal(a.params(), b.params())
    with pytest.raises(ValueError):
        b.apply_gradient(grad[:10], 1e-3)
    a.close()
    b.close()


def test_data_parallel_training_under_torchrun(torch, tmp_path):
    """learned.py train under torchrun (NCCL process group, one rank here: the
    all-reduce runs, over a world of one) saves the same weights as the
    single-process run of the same configuration."""
    import os
    import subprocess
    import sys
    import learned
    script = os.path.join(os.path.dirname(learned.__file__), "learned.py")
    args = ["train", "--npatch", "65536", "--epochs", "1", "--batch", "2048", "--eval", "0"]
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r1 = subprocess.run([sys.executable, script] + args + ["--out", str(tmp_path / "single")], env=env,
                        capture_output=True, text=True, timeout=600)
    assert r1.returncode == 0, r1.stderr[-2000:]
    import socket
    with socket.socket() as so:   # a free rendezvous port
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    r2 = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "1",
                         "--master-addr", "127.0.0.1", "--master-port", str(port), script] + args +
                        ["--out", str(tmp_path / "dp")], env=env, capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0, r2.stderr[-2000:]
    w1 = np.fromfile(str(tmp_path / "single.bin"), dtype=np.float32)
    w2 = np.fromfile(str(tmp_path / "dp.bin"), dtype=np.float32)
    assert w1.size == w2.size and np.array_equal(w1, w2)


def test_bounded_wait_reports_timeout_and_recovers(torch):
    """The inference kernel's bounded tensor-core wait: a wait on a barrier
    nothing signals gives up after a few polls, every thread leaves through
    the normal path (the prediction is unchanged), gpg_net_check reports
    GPG_ERR_CUDA once, and the next call is clean."""
    from gpg.lib import GpgError
    from gpg.net import Net
    rho, pin, _ = _data(24, 5)
    rho, pin = torch.from_numpy(rho).cuda(), torch.from_numpy(pin).cuda()
    net = Net(max_batch=32, seed=2)
    ref = torch.empty((24, 8, 8, 8), device="cuda")
    net.predict(rho, pin, ref, float(CNST))
    torch.cuda.synchronize()
    net.check()
    net.set_wait_probe(4)
    got = torch.empty_like(ref)
    net.predict(rho, pin, got, float(CNST))
    torch.cuda.synchronize()
    with pytest.raises(GpgError) as ei:
        net.check()
    assert ei.value.status == 2  # GPG_ERR_CUDA
    assert torch.equal(got, ref)
    net.set_wait_probe(0)
    net.predict(rho, pin, got, float(CNST))
    torch.cuda.synchronize()
    net.check()
    assert torch.equal(got, ref)
    net.close()
