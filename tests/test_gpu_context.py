"""Reference-shaped host API (CUAPI_* flow) through the C-ABI (needs a B200):
allocate -> fill pinned buffers -> asynchronous solve over streams ->
synchronize -> read, compared with the stream-ordered device API."""
import numpy as np
import pytest

from gpg.abi import GPG_MG, GPG_SOR, default_params
from gpg.inputs import make_patches

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = pytest.importorskip("torch")
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def device_result(torch, p, d):
    from gpg.lib import solve_device
    dev = torch.device("cuda:0")
    pot, flu, it, _ = solve_device(p, torch.from_numpy(d["rho"]).to(dev), torch.from_numpy(d["pot_in"]).to(dev),
                                   flu=torch.from_numpy(d["flu"].copy()).to(dev))
    torch.cuda.synchronize()
    return pot.cpu().numpy(), flu.cpu().numpy(), it.cpu().numpy()


@pytest.mark.parametrize("scheme,rs,g,G", [(GPG_SOR, 4, 1, 1), (GPG_SOR, 8, 3, 2), (GPG_MG, 4, 3, 2),
                                           (GPG_MG, 8, 2, 1)])
@pytest.mark.parametrize("nstream", [1, 3])
def test_async_context_matches_device_api(torch, scheme, rs, g, G, nstream):
    from gpg.lib import Context
    npg = 5  # 40 patches: uneven split over 3 streams
    dt = np.float32 if rs == 4 else np.float64
    d = make_patches(8 * npg, g, seed=800 + g, gra_ghost=G, dtype=dt)
    p = default_params(rs, g, scheme, gra_ghost=G, p5_gradient=1 if G == 2 else 0)
    with Context(0, nstream=4) as ctx:
        rho, pin, pout, flu = ctx.allocate(p, npg)
        rho[...] = d["rho"]
        pin[...] = d["pot_in"]
        flu[...] = d["flu"]
        ctx.asyn_solve(p, npg, nstream=nstream)
        ctx.synchronize()
        it, _ = ctx.iterations(8 * npg)
        ref_pot, ref_flu, ref_it = device_result(torch, p, d)
        assert np.array_equal(pout, ref_pot)
        assert np.array_equal(flu, ref_flu)
        assert np.array_equal(it, ref_it)
        # gravity alone on the potential just produced (Poisson off): h_pot_out is input
        p2 = p.copy(poisson=0)
        flu_before = flu.copy()
        ctx.asyn_solve(p2, npg, nstream=nstream)
        ctx.synchronize()
        from oracle.oracle import run_oracle
        _, of, _, _ = run_oracle(p2, None, None, pot_out=pout.copy(), flu=flu_before)
        assert np.array_equal(flu, of)


def test_context_errors(torch):
    from gpg.lib import Context, GpgError
    p = default_params(4, 2, GPG_SOR)
    with Context(0, nstream=2) as ctx:
        with pytest.raises(GpgError) as e:
            ctx.asyn_solve(p, 1)              # no buffers yet
        assert e.value.status == 6
        ctx.allocate(p, 2)
        with pytest.raises(GpgError):
            ctx.asyn_solve(p, 3)              # more groups than allocated
        with pytest.raises(GpgError):
            ctx.asyn_solve(p, 2, nstream=5)   # more streams than the context has
        with pytest.raises(GpgError):
            ctx.asyn_solve(p.copy(ghost=3), 2)  # shape differs from the allocation
        with pytest.raises(GpgError):
            ctx.allocate(p, 2)                # double allocation
    with Context(0, nstream=1) as ctx:
        ctx.allocate(p, 0)                    # empty allocation still counts as allocated
        with pytest.raises(GpgError) as e:
            ctx.allocate(p, 1)
        assert e.value.status == 6
        ctx.free()
        bufs = ctx.allocate(p, 1)             # allowed again after gpg_mem_free
        assert bufs[0].shape[0] == 8
        for b in bufs:
            b[...] = 0
        ctx.asyn_solve(p, 1)
        ctx.synchronize()
        it, _ = ctx.iterations(8)
        assert it.shape == (8,)
        ctx.free()
        with pytest.raises(GpgError):
            ctx.iterations(8)                 # buffers released: nothing left to read
