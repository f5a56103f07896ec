"""Shared test set-up: import paths and the `gpu` marker.

`-m "not gpu"` tests run on any CPU host (oracle vs golden vectors, host-side
logic, the C-ABI library's exported symbols, multi-rank CPU paths).
`-m gpu` tests call the CUDA library through its C-ABI on cuda:0.
"""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gpu_testbed_poisson-gravity_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
