"""The batch engine on the GPU, through the C ABI: uneven slices (grid,
views, channels, spectrum) in one captured graph give the plain one-slice
path's results -- sinograms bit for bit (same per-ray code), FBP images to
float rounding (the tuner may pick another view split of the
backprojector) -- on every replay, after the maps change in place, and for
adjoint batches."""
import numpy as np
import pytest

import virtualct_b200 as vct
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu


def _specs():
    # small grids so the test stays quick; views both divisible by 4 and not
    return phantoms.batch_specs(7, seed=3, grids=(64, 96, 128), rate=(3, 9), channels=(512, 800))


def _tables():
    return {k: phantoms.kramers_tables(k) for k in (80, 100, 120, 140)}


def _geo(sp):
    return vct.Geometry.with_channels(sp["channels"], views=sp["views"], recon_size=sp["N"], pixel_cm=0.1)


def _plain(sp, maps, tab, sigma, seed, filt):
    import torch

    g = _geo(sp)
    with vct.Context(g) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(*tab)
        sino = torch.zeros((g.views, g.width), dtype=torch.float32, device="cuda")
        img = torch.zeros((g.recon_size, g.recon_size), dtype=torch.float32, device="cuda")
        ctx.mbfpa_dev(sigma, seed, sino)
        ctx.fbp_dev(sino, img, filter=filt)
        ctx.synchronize()
        return sino.cpu().numpy(), img.cpu().numpy()


@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_plain(cuda_device, tune):
    import torch

    specs, tabs = _specs(), _tables()
    jobs, host_maps = [], []
    for i, sp in enumerate(specs):
        m = phantoms.ellipse_phantom(sp["seed"], sp["N"], border_px=2)
        host_maps.append(m)
        g = _geo(sp)
        jobs.append(vct.Job(g, torch.from_numpy(m).cuda(), *tabs[sp["kvp"]],
                            sino=torch.zeros((g.views, g.width), dtype=torch.float32, device="cuda"),
                            img=torch.zeros((g.recon_size, g.recon_size), dtype=torch.float32, device="cuda"),
                            filter=1 + i % 2, sigma=5.37e-5 if i % 3 else 0.0, seed=11 + i))
    with vct.Batch(jobs, tune=tune) as b:
        cfg = b.config()
        # one launch per stage over all jobs: packing, statistics reset,
        # forward, normalisation + noise, weight, filter, two backprojectors
        assert 1 <= cfg["kernels_per_run"] <= 8, cfg
        for rep in range(2):
            b.run()
            b.synchronize()
            for i, (sp, j) in enumerate(zip(specs, jobs)):
                s_ref, i_ref = _plain(sp, host_maps[i], tabs[sp["kvp"]], j.sigma, j.seed, j.filter)
                assert np.array_equal(j.sino.cpu().numpy().view(np.uint32), s_ref.view(np.uint32)), (rep, i)
                img = j.img.cpu().numpy()
                assert np.abs(img - i_ref).max() <= 1e-5 * np.abs(i_ref).max(), (rep, i)
        # maps changed in place are picked up by the next run
        j0 = jobs[0]
        new = (host_maps[0].astype(np.float64) * 0.9).astype(np.int16)
        j0.maps.copy_(torch.from_numpy(new).cuda())
        b.run()
        b.synchronize()
        s_ref, _ = _plain(specs[0], new, tabs[specs[0]["kvp"]], j0.sigma, j0.seed, j0.filter)
        assert np.array_equal(j0.sino.cpu().numpy().view(np.uint32), s_ref.view(np.uint32))


def test_adjoint_batch_matches_plain(cuda_device):
    import torch

    specs, tabs = _specs()[:4], _tables()
    jobs, ref = [], []
    for sp in specs:
        m = phantoms.ellipse_phantom(sp["seed"], sp["N"], border_px=2)
        g = _geo(sp)
        with vct.Context(g) as ctx:
            ctx.set_maps(m)
            ctx.set_spectrum(*tabs[sp["kvp"]])
            meas = ctx.mbfpa(sigma=5.37e-5, seed=5)
            at = (m.astype(np.float64) * 0.95).astype(np.int16)
            ctx.set_maps(at)
            loss, grad = ctx.forward_adjoint(meas)
        ref.append((loss, grad))
        jobs.append(vct.Job(g, torch.from_numpy(at).cuda(), *tabs[sp["kvp"]],
                            meas=torch.from_numpy(meas).cuda(),
                            grad=torch.zeros((6, g.recon_size, g.recon_size), dtype=torch.float32, device="cuda"),
                            loss=torch.zeros(1, dtype=torch.float64, device="cuda")))
    with vct.Batch(jobs) as b:
        # packing, reset, persistent forward, loss sums, exact-walk scatter,
        # gather (one launch per tile shape present) and fold, for every job
        assert 1 <= b.config()["kernels_per_run"] <= 10, b.config()
        b.run()
        b.synchronize()
        for j, (loss, grad) in zip(jobs, ref):
            assert float(j.loss.cpu()[0]) == loss
            assert np.array_equal(j.grad.cpu().numpy().view(np.uint32), grad.view(np.uint32))
