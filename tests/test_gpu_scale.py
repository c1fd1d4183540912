"""The scale configuration on the GPU: dual-energy (80/140 kVp) material
decomposition of 8-element maps by projected gradient descent, every
(slice, spectrum) gradient in one adjoint batch, densities at 16384 units
per g/cm^3.  Checks: the loss falls at every iteration; the batched
gradients equal the FP64 oracle's; and at the full scale geometry (1024^2 at
0.05 cm, 1440 views x 1600 channels, 8 elements) the device loss and
gradient match the FP64 oracle (the walk's exact transpose)."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from virtualct_b200 import phantoms
from virtualct_b200.decomposition import Decomposition

pytestmark = pytest.mark.gpu

UNITS = 16384.0


def _measured(geo, maps, tabs, sigma, seed):
    import torch

    out = []
    with vct.Context(geo) as ctx:
        ctx.set_maps(maps)
        for e, (mu, pdf) in enumerate(tabs):
            ctx.set_spectrum(mu, pdf)
            s = torch.empty((geo.views, geo.width), dtype=torch.float32, device="cuda")
            ctx.mbfpa_dev(sigma, seed + e, s)
            out.append(s)
        ctx.synchronize()
    return out


def _oracle_geom(geo):
    return O.geom(views=geo.views, channels=geo.width, recon_size=geo.recon_size, pixel_cm=geo.pixel_cm)


def test_dual_energy_descent_small(cuda_device):
    import torch

    el = phantoms.ELEMENTS8
    tabs = [phantoms.kramers_tables(k, el) for k in (80, 140)]
    geo = vct.Geometry(views=120, recon_size=96, pixel_cm=0.1)
    S = 3
    true = [phantoms.ellipse_phantom(40 + s, 96, elements=el, border_px=2) for s in range(S)]
    meas = [_measured(geo, m, tabs, 0.0, 10 * s) for s, m in enumerate(true)]
    rho0 = torch.from_numpy(np.stack([m.astype(np.float32) / 1000.0 * 0.9 for m in true])).cuda()
    dec = Decomposition(geo, tabs, meas, rho0, units=UNITS, tune=False)
    try:
        # the first batched gradients against the FP64 oracle (slice 0, 80 kVp)
        dec.iterate(1)
        torch.cuda.synchronize()
        g = _oracle_geom(geo)
        c, s = O.trig_tables(geo.views)
        rho_q = dec.maps[0].cpu().numpy().astype(np.float64) / UNITS
        ref_loss, ref = O.loss_grad(g, c, s, rho_q, tabs[0][0], tabs[0][1], meas[0][0].cpu().numpy())
        dev = dec.grads[0, 0].cpu().numpy().astype(np.float64)
        assert abs(float(dec.loss[0, 0]) - ref_loss) <= 1e-6 * ref_loss
        assert np.abs(dev - ref).max() <= 1e-5 * np.abs(ref).max()
        dec.iterate(8)
        h = dec.history
        assert len(h) == 9 and all(b <= a for a, b in zip(h, h[1:])), h
        assert h[-1] < 0.9 * h[0], h
        assert dec.accepted > 0
    finally:
        dec.close()


def test_scale_geometry_gradient_vs_fp64(cuda_device):
    """One slice of the scale configuration: 1024^2 at 0.05 cm, 8 elements,
    1440 views x 1600 channels, 80 kVp, densities at 16384 units."""
    import torch

    el = phantoms.ELEMENTS8
    mu, pdf = phantoms.kramers_tables(80, el)
    geo = vct.Geometry.with_channels(1600, views=1440, recon_size=1024, pixel_cm=0.05)
    true = phantoms.ellipse_phantom(7, 1024, elements=el)
    meas = _measured(geo, true, [(mu, pdf)], 5.37e-5, 3)[0]
    at = np.round(true.astype(np.float64) / 1000.0 * 0.95 * UNITS).astype(np.int16)
    with vct.Context(geo) as ctx:
        ctx.set_density_scale(UNITS)
        ctx.set_maps(at)
        ctx.set_spectrum(mu, pdf)
        grad = torch.empty((8, 1024, 1024), dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        ctx.forward_adjoint_dev(meas, grad, loss=loss)
        ctx.synchronize()
        grad, loss = grad.cpu().numpy().astype(np.float64), float(loss.cpu()[0])
    g = _oracle_geom(geo)
    c, s = O.trig_tables(geo.views)
    ref_loss, ref = O.loss_grad(g, c, s, at.astype(np.float64) / UNITS, mu, pdf, meas.cpu().numpy())
    assert abs(loss - ref_loss) <= 1e-6 * ref_loss
    d = grad - ref
    assert np.abs(d).max() <= 1e-5 * np.abs(ref).max()
    assert np.linalg.norm(d) <= 1e-5 * np.linalg.norm(ref)


def test_decomposition_checkpoint_resume(cuda_device, tmp_path):
    """save() after three iterations and load() into a fresh decomposition:
    the next iteration equals the uninterrupted run's bit for bit."""
    import torch

    el = phantoms.ELEMENTS8
    tabs = [phantoms.kramers_tables(k, el) for k in (80, 140)]
    geo = vct.Geometry(views=80, recon_size=64, pixel_cm=0.1)
    true = [phantoms.ellipse_phantom(60 + s, 64, elements=el, border_px=2) for s in range(2)]
    meas = [_measured(geo, m, tabs, 0.0, 10 * s) for s, m in enumerate(true)]
    start = np.stack([m.astype(np.float32) / 1000.0 * 0.9 for m in true])
    a = Decomposition(geo, tabs, meas, torch.from_numpy(start.copy()).cuda(), units=UNITS, tune=False)
    b = Decomposition(geo, tabs, meas, torch.from_numpy(start.copy()).cuda(), units=UNITS, tune=False)
    c = Decomposition(geo, tabs, meas, torch.from_numpy(np.zeros_like(start)).cuda(), units=UNITS, tune=False)
    try:
        a.iterate(4)
        b.iterate(3)
        b.save(tmp_path / "ckpt")
        c.load(tmp_path / "ckpt")
        c.iterate(1)
        assert c.history == a.history
        assert torch.equal(c.rho, a.rho)
        assert torch.equal(c.maps, a.maps)
        assert np.array_equal(c.step_size, a.step_size)
    finally:
        a.close()
        b.close()
        c.close()
