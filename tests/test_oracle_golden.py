"""The C restatement (oracle/) against the reference's own CPU code.

Golden vectors in tests/golden/ were produced by the reference's unmodified
CPU solver (tests/golden/make_golden.py); the restatement must reproduce them
bit for bit, including every per-patch SOR iteration count.  When the
reference objects (oracle/_ref/) are present, a second test compares larger
seeded batches live.
"""
import json
import os

import numpy as np
import pytest

from gpg.abi import GPG_MG, GPG_SOR, GPG_INIT_ZERO, GPG_STOP_TOLERANCE, default_params
from gpg.inputs import make_patches
from oracle.oracle import interp_cube, ref_available, run_oracle, run_reference

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")

with open(os.path.join(GOLD, "index.json")) as f:
    INDEX = json.load(f)

import sys  # noqa: E402
sys.path.insert(0, GOLD)
from make_golden import case_inputs, input_sha  # noqa: E402


@pytest.mark.parametrize("name", sorted(INDEX["cases"]))
def test_oracle_matches_reference_golden(name):
    c = INDEX["cases"][name]
    d, seed = case_inputs(name, c["real_size"], c["ghost"], c["gra_ghost"])
    assert seed == c["seed"]
    gold = np.load(os.path.join(GOLD, name + ".npz"))
    assert str(gold["input_sha"]) == input_sha(d), "input generator drifted"
    p = default_params(c["real_size"], c["ghost"], c["scheme"], gra_ghost=c["gra_ghost"],
                       int_scheme=c["int_scheme"], p5_gradient=c["p5_gradient"])
    pot, flu, iters, _ = run_oracle(p, d["rho"], d["pot_in"], flu=d["flu"].copy(),
                                    accum_f64=False, nthreads=2)
    keep = INDEX["keep_pot"]
    assert np.array_equal(pot[keep], gold["pot_out"])          # bit-exact
    assert np.array_equal(flu[:1], gold["flu"])
    if c["scheme"] == GPG_SOR:
        assert iters.tolist() == gold["iters"].tolist()


@pytest.mark.skipif(not ref_available("sor", 3, 1, "f32"), reason="oracle/_ref not built")
@pytest.mark.parametrize("scheme", [GPG_SOR, GPG_MG])
@pytest.mark.parametrize("rs", [4, 8])
@pytest.mark.parametrize("g", [1, 2, 3, 4, 5])
def test_oracle_matches_reference_live(scheme, rs, g):
    dt = np.float32 if rs == 4 else np.float64
    d = make_patches(64, g, seed=7000 + g, dtype=dt)
    p = default_params(rs, g, scheme)
    po, fo, io, _ = run_oracle(p, d["rho"], d["pot_in"], flu=d["flu"].copy(), accum_f64=False)
    pr, fr, ir = run_reference(p, d["rho"], d["pot_in"].copy(), flu=d["flu"].copy())
    assert np.array_equal(po, pr)
    assert np.array_equal(fo, fr)
    if scheme == GPG_SOR:
        assert np.array_equal(io, ir)


def test_interp_reproduces_quadratic_exactly():
    """CQUAD and QUAD interpolation reproduce a linear coarse field exactly at
    fine-cell centres (both schemes are exact for linear data)."""
    for g in range(1, 6):
        pn = 4 + 2 * ((g + 3) // 2)
        pint = (g + 3) // 2
        k, j, i = np.meshgrid(np.arange(pn), np.arange(pn), np.arange(pn), indexing="ij")
        # coarse cell centres in fine units relative to the fine cube origin
        cz, cy, cx = [2.0 * a + 1.0 - 2 * pint + g for a in (k, j, i)]
        coarse = (0.5 + 0.25 * cx - 0.125 * cy + 0.0625 * cz).astype(np.float64)
        n = 8 + 2 * g
        fz, fy, fx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        want = 0.5 + 0.25 * (fx + 0.5) - 0.125 * (fy + 0.5) + 0.0625 * (fz + 0.5)
        for s in (4, 5):
            got = interp_cube(coarse, g, s)
            assert np.allclose(got, want, rtol=0, atol=1e-12), (g, s)


def test_sor_converges_to_discrete_solution():
    """Zero-start SOR run to a tight tolerance solves the 7-point system."""
    g = 2
    d = make_patches(8, g, seed=11, dtype=np.float64)
    p = default_params(8, g, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_TOLERANCE,
                       sor_tolerance=1e-10, sor_min_iter=1, sor_max_iter=500, gra_acc=0,
                       gra_ghost=2)
    pot, _, iters, resid = run_oracle(p, d["rho"], d["pot_in"])
    assert (iters < 500).all()
    c = pot  # GRA_NXT == cube edge (12) when gra_ghost == ghost
    lap = (c[:, 2:, 1:-1, 1:-1] + c[:, :-2, 1:-1, 1:-1] + c[:, 1:-1, 2:, 1:-1] + c[:, 1:-1, :-2, 1:-1]
           + c[:, 1:-1, 1:-1, 2:] + c[:, 1:-1, 1:-1, :-2] - 6 * c[:, 1:-1, 1:-1, 1:-1])
    rhs = p.poi_coeff * d["rho"]
    assert np.abs(lap - rhs).max() < 1e-6 * np.abs(rhs).max()
    assert (resid <= 1e-10 * np.abs(rhs).reshape(len(rhs), -1).sum(1)).all()
