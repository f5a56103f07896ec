"""CPU checks of the same-box GPU comparison's recipe (no GPU): every case's
driver arguments carry the reference's defaults (Main.cpp:1142-1223), and
the build recipe names sources that exist in the reference tree when it is
present."""
import os

import pytest

from gpg.abi import SOR_OMEGA
from oracle import build as ob
from oracle.cuapi_bench_inputs import CASES, case_id, driver_args


def _kv(args):
    return dict(zip(args[::2], args[1::2]))


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_driver_arguments_follow_the_reference_defaults(case):
    scheme, g, G, prec, npatch, p5 = case
    assert case[:4] in ob.REF_GPU_CONFIGS
    a = _kv(driver_args(case, "in.bin", "out.bin"))
    assert int(a["--npg"]) * 8 == npatch
    assert a["--max-iter"] == ("100" if prec == "f64" else "60") and a["--min-iter"] == "10"
    assert float(a["--omega"]) == SOR_OMEGA[g]
    assert a["--mg-max-iter"] == ("20" if prec == "f64" else "10")
    assert float(a["--mg-tol"]) == (1e-15 if prec == "f64" else 1e-6)
    assert a["--int-scheme"] == "4" and a["--p5"] == str(p5)
    assert a["--nstream"] == "4"


def test_cases_leave_out_device_malloc_configurations():
    """MG in FP64 and at 18^3 allocates device memory per block in the
    reference (CUPOT_PoissonSolver_MG.cu:136-145,186-187): never run."""
    for scheme, g, G, prec in ob.REF_GPU_CONFIGS:
        if scheme == "mg":
            assert prec == "f32" and g < 5


def test_recipe_sources_exist_in_the_reference_tree():
    root = ob.DEFAULT_REF
    if not os.path.isdir(os.path.join(root, "GPU_Solver")):
        pytest.skip("reference tree absent")
    for f in ob.REF_GPU_API:
        assert os.path.exists(os.path.join(root, "GPU_API", f)), f
    for f in ob.REF_GPU_SOLVER:
        assert os.path.exists(os.path.join(root, "GPU_Solver", f)), f
    assert os.path.exists(ob.BENCH_DRIVER) and os.path.exists(ob.GPU_COMPAT)
