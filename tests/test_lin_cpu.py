"""CPU checks of the learned correction's restatement and of the calibrated
fixed residual (no GPU): the equivariant block model with the Green's
function weights is the exact correction, the FP64 gradient is the
derivative of the loss, the tolerance table of the C library and the Python
mirror agree with a fresh calibration, and every patch reaches it."""
import ctypes as C

import numpy as np
import pytest

from gpg.abi import GPG_INIT_INTERP, GPG_INIT_ZERO, POT_TOL, fixed_residual_params
from gpg.inputs import make_patches
from gpg.lib import check, library
from oracle import lin_oracle as lo


def test_block_model_with_green_weights_is_the_exact_correction():
    w = lo.green_params()
    G = -np.linalg.inv(lo.laplacian_interior())
    r0 = np.random.default_rng(0).standard_normal((6, 512))
    u = lo.fold(r0)
    v = np.stack([u[:, b] @ w[lo.class_of(b)].T for b in range(8)], 1)
    d = lo.unfold(v)
    want = r0 @ G.T
    assert np.abs(d - want).max() <= 1e-12 * np.abs(want).max()


def test_fold_unfold_and_orbit_tables():
    x = np.random.default_rng(1).standard_normal((3, 512))
    assert np.allclose(lo.unfold(lo.fold(x)), 8 * x, rtol=0, atol=1e-12)
    assert sorted(lo.CELL.reshape(-1)) == list(range(512))        # orbits tile the interior
    for b in range(8):
        assert sorted(lo.PERM[b]) == list(range(64))
        assert all(lo.perm_orbit(lo.perm_orbit(o, lo.perm_of(b)), lo.perm_of(b)) == o for o in range(64))


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    a = (np.random.default_rng(2).standard_normal(4096) * 10.0 ** np.random.default_rng(3).uniform(-9, 3, 4096)
         ).astype(np.float32)
    want = torch.from_numpy(a).bfloat16().double().numpy()
    assert np.array_equal(lo.bf16(a), want)


def test_gradient_is_the_derivative_of_the_loss():
    rng = np.random.default_rng(4)
    w = 0.03 * rng.standard_normal((4, 64, 64))
    u = rng.standard_normal((5, 8, 64)) * 10.0 ** rng.uniform(-4, 0, (5, 1, 1))
    t = rng.standard_normal((5, 8, 64)) * 0.01
    loss, grad = lo.gradients(w, u, t)
    for c, r, k in ((0, 3, 7), (1, 60, 2), (2, 17, 33), (3, 63, 63)):
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[c, r, k] += h
        wm[c, r, k] -= h
        fd = (lo.gradients(wp, u, t)[0] - lo.gradients(wm, u, t)[0]) / (2 * h)
        assert abs(fd - grad[c, r, k]) <= 1e-6 * max(1e-12, abs(grad).max())


@pytest.mark.parametrize("rs", [4, 8])
@pytest.mark.parametrize("g", [1, 2, 3, 4, 5])
def test_c_tolerance_table_equals_python(rs, g):
    tol = C.c_double()
    check(library().gpg_pot_tolerance(rs, g, C.byref(tol)))
    assert tol.value == POT_TOL[(rs, g)]


@pytest.mark.parametrize("rs", [4, 8])
@pytest.mark.parametrize("g", [1, 3, 5])
def test_calibration_reproduces_the_table(rs, g):
    from oracle.calibrate_tol import floor_ratios
    r = floor_ratios(rs, g, 256, 11)
    assert abs(r["tol"] - POT_TOL[(rs, g)]) <= 0.15 * POT_TOL[(rs, g)], r
    assert r["max"] < 0.7 * POT_TOL[(rs, g)], r


@pytest.mark.parametrize("rs", [4, 8])
@pytest.mark.parametrize("g", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("start", [GPG_INIT_ZERO, GPG_INIT_INTERP])
def test_every_patch_reaches_the_fixed_residual(rs, g, start):
    """Held-out inputs (other seed, rho0 over 4 decades, power index 1.5-2.5):
    no patch runs into Max_Iter from either start."""
    from oracle.oracle import run_oracle
    n = 128
    rng = np.random.default_rng(99 + g)
    d = make_patches(n, g, seed=99 + g, rho0=10.0 ** rng.uniform(0, 4, n), index=rng.uniform(1.5, 2.5, n),
                     dtype=np.float32 if rs == 4 else np.float64, fluid=False)
    p = fixed_residual_params(rs, g, init_mode=start, max_iter=300)
    _, _, it, res = run_oracle(p, d["rho"], d["pot_in"])
    assert it.max() < 300, (it.max(), np.argmax(it))
