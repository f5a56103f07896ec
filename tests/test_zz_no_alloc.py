"""Allocation-free batched SOR entry point (needs a B200).

Callers that may not allocate device memory while they solve (a code that
hands all device memory to its own pool at start-up, or whose allocator
belongs to another runtime) use gpg_solve_batch_device_noalloc: the work-queue
counter lives in a static device array inside libgpg instead of a caller
buffer.  Called through the C-ABI twice in a row, it must return exactly what
gpg_solve_batch_device returns with a caller-provided counter.  This file is
collected last; it passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from gpg.abi import (GPG_ERR_INVALID, GPG_INIT_ZERO, GPG_OK, GPG_SOR, GPG_STOP_ABS_TOLERANCE, GpgBatchGroup,
                     GpgParams, default_params)
from gpg.inputs import log_uniform, make_patches, mixed_ghost_assignment

pytestmark = pytest.mark.gpu


def _groups(torch, rs, npatch, seed, dev):
    gh = mixed_ghost_assignment(npatch, seed)
    rho0 = log_uniform(npatch, seed + 1)
    dt = np.float32 if rs == 4 else np.float64
    tdt = torch.float32 if rs == 4 else torch.float64
    out = []
    for g in range(1, 6):
        idx = np.flatnonzero(gh == g)
        n = len(idx)
        d = make_patches(n, g, seed=seed + 10 * g, rho0=rho0[idx], dtype=dt)
        out.append({"ghost": g, "rho": torch.from_numpy(d["rho"]).to(dev),
                    "pot_in": torch.from_numpy(d["pot_in"]).to(dev),
                    "flu0": torch.from_numpy(d["flu"]).to(dev),
                    "flu": torch.empty((n, 5, 8, 8, 8), dtype=tdt, device=dev),
                    "pot_out": torch.empty((n, 10, 10, 10), dtype=tdt, device=dev),
                    "iters": torch.empty(n, dtype=torch.int32, device=dev),
                    "resid": torch.empty(n, dtype=torch.float64, device=dev)})
    return out


def _c_groups(groups):
    arr = (GpgBatchGroup * len(groups))()
    for a, g in zip(arr, groups):
        a.ghost = g["ghost"]
        a.npatch = int(g["rho"].shape[0])
        a.d_rho, a.d_pot_in = g["rho"].data_ptr(), g["pot_in"].data_ptr()
        a.d_pot_out, a.d_flu = g["pot_out"].data_ptr(), g["flu"].data_ptr()
        a.d_guess = None
        a.d_iters, a.d_resid = g["iters"].data_ptr(), g["resid"].data_ptr()
        a.sor_omega = 0.0
    return arr


def _snapshot(groups):
    return [(g["pot_out"].clone(), g["flu"].clone(), g["iters"].clone(), g["resid"].clone()) for g in groups]


@pytest.mark.parametrize("rs", [4, 8])
def test_noalloc_batch_matches_allocating_entry_point(rs):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpg.lib import library
    lib = library()
    noalloc = lib.gpg_solve_batch_device_noalloc
    noalloc.restype = C.c_int
    noalloc.argtypes = [C.POINTER(GpgParams), C.c_int, C.POINTER(GpgBatchGroup), C.c_void_p]
    alloc = lib.gpg_solve_batch_device
    alloc.restype = C.c_int
    alloc.argtypes = [C.POINTER(GpgParams), C.c_int, C.POINTER(GpgBatchGroup), C.c_void_p, C.c_void_p]

    dev = torch.device("cuda:0")
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = default_params(rs, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_ABS_TOLERANCE,
                       sor_tolerance=1e-4 if rs == 4 else 1e-10, sor_min_iter=1, sor_max_iter=200)
    groups = _groups(torch, rs, 301, seed=123, dev=dev)
    arr = _c_groups(groups)

    # the existing entry point, with a counter the caller allocated
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    for g in groups:
        g["flu"].copy_(g["flu0"])
    assert alloc(C.byref(p), len(groups), arr, C.c_void_p(counter.data_ptr()), stream) == 0
    torch.cuda.synchronize()
    want = _snapshot(groups)

    for call in range(2):  # two calls in a row share (and re-zero) the static counter
        for g in groups:
            g["flu"].copy_(g["flu0"])
            g["pot_out"].fill_(float("nan"))
            g["iters"].fill_(-7)
        rc = noalloc(C.byref(p), len(groups), arr, stream)
        assert rc == 0, lib.gpg_last_error()
        torch.cuda.synchronize()
        for (wp, wf, wi, wr), g in zip(want, groups):
            assert torch.equal(g["pot_out"], wp), (call, g["ghost"])
            assert torch.equal(g["flu"], wf), (call, g["ghost"])
            assert torch.equal(g["iters"], wi) and torch.equal(g["resid"], wr), (call, g["ghost"])


def test_noalloc_rejects_batches_beyond_its_limit():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpg.lib import library
    lib = library()
    noalloc = lib.gpg_solve_batch_device_noalloc
    noalloc.restype = C.c_int
    noalloc.argtypes = [C.POINTER(GpgParams), C.c_int, C.POINTER(GpgBatchGroup), C.c_void_p]
    dev = torch.device("cuda:0")
    groups = _groups(torch, 4, 40, seed=5, dev=dev)[:1]
    arr = _c_groups(groups)
    arr[0].npatch = (1 << 30) + 1  # more than one call may queue; rejected on the host, nothing launched
    p = default_params(4, 1, GPG_SOR)
    rc = noalloc(C.byref(p), 1, arr, C.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    assert rc == GPG_ERR_INVALID
    assert b"exceeds" in lib.gpg_last_error()


def test_noalloc_empty_batches_launch_nothing():
    """No groups, or groups without patches: the call succeeds, writes no
    output and a following full call still matches the allocating entry point."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gpg.lib import library
    lib = library()
    noalloc = lib.gpg_solve_batch_device_noalloc
    noalloc.restype = C.c_int
    noalloc.argtypes = [C.POINTER(GpgParams), C.c_int, C.POINTER(GpgBatchGroup), C.c_void_p]
    dev = torch.device("cuda:0")
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = default_params(4, 1, GPG_SOR, init_mode=GPG_INIT_ZERO, stop_mode=GPG_STOP_ABS_TOLERANCE,
                       sor_tolerance=1e-4, sor_min_iter=1, sor_max_iter=200)
    assert noalloc(C.byref(p), 0, None, stream) == GPG_OK, lib.gpg_last_error()
    groups = _groups(torch, 4, 60, seed=9, dev=dev)
    arr = _c_groups(groups)
    for a in arr:
        a.npatch = 0
    for g in groups:
        g["iters"].fill_(-7)
    assert noalloc(C.byref(p), len(groups), arr, stream) == GPG_OK, lib.gpg_last_error()
    torch.cuda.synchronize()
    assert all(bool((g["iters"] == -7).all()) for g in groups)
    arr = _c_groups(groups)
    for g in groups:
        g["flu"].copy_(g["flu0"])
    assert noalloc(C.byref(p), len(groups), arr, stream) == GPG_OK, lib.gpg_last_error()
    torch.cuda.synchronize()
    got = _snapshot(groups)
    counter = torch.zeros(1, dtype=torch.int32, device=dev)
    for g in groups:
        g["flu"].copy_(g["flu0"])
    alloc = lib.gpg_solve_batch_device
    alloc.restype = C.c_int
    alloc.argtypes = [C.POINTER(GpgParams), C.c_int, C.POINTER(GpgBatchGroup), C.c_void_p, C.c_void_p]
    assert alloc(C.byref(p), len(groups), arr, C.c_void_p(counter.data_ptr()), stream) == GPG_OK
    torch.cuda.synchronize()
    for (gp, gf, gi, gr), g in zip(got, groups):
        assert torch.equal(g["pot_out"], gp) and torch.equal(g["flu"], gf)
        assert torch.equal(g["iters"], gi) and torch.equal(g["resid"], gr)
