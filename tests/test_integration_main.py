"""The reference's own driver, relinked on this library (needs a B200).

oracle/build.py links the reference's unmodified Main.cpp, CPU solvers and
Auxiliary code against the CUAPI_* shim (include/gpg_cuapi.h) and libgpg.so.
`-P` runs the reference CPU solver and the library on the same inputs and
prints the reference's own DataCompare verdicts (Main.cpp:1007-1061), with
its Makefile thresholds (Makefile:56-70).  Both must read "Passed".
"""
import os
import subprocess

import pytest

from oracle.build import INTEGRATION_CONFIGS, integration_exe

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scheme,g,G,prec", INTEGRATION_CONFIGS)
def test_reference_main_passes_against_library(tmp_path, scheme, g, G, prec):
    exe = integration_exe(scheme, g, G, prec)
    if not os.path.exists(exe):
        pytest.skip("integration executables not built (reference sources absent at build time)")
    args = [exe, "-P", "-n", "16", "-s", "2", "-t", "4"]
    if G == 2:
        args += ["-p", "1"]  # 5-point gradient
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    out = r.stdout
    assert r.returncode == 0, r.stderr[-2000:]
    assert out.count("Passed !!") == 2, out[-3000:] + r.stderr[-3000:]
    assert "Failed" not in out
