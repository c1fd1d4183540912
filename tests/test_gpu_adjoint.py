"""Adjoint of the forward projector on the GPU, through the C ABI: loss and
gradient against the FP64 oracle (the exact transpose of the reference walk),
central finite differences of the FP64 loss (h = 1e-3 relative), the
dot-product test of the device A and A^T, the VJP entry point, and
run-to-run determinism.  The reference has no gradient, so these checks pin
the adjoint instead of a reference output."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import golden
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu

# Device against FP64: the ray factors and chords are FP32, sums over the
# views are FP64.  Max error relative to the largest gradient entry, and
# relative L2 error.
GRAD_MAX_REL = 1e-5
GRAD_L2_REL = 1e-5
LOSS_RTOL = 1e-6


def _case(N, views, channels, seed, noise=0.02, border_px=1):
    t = golden("mu_tables.npz")
    mu, pdf = t["kramers120_mu"], t["kramers120_pdf"]
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.1)
    c, s = O.trig_tables(views)
    maps = phantoms.ellipse_phantom(seed, N, border_px=border_px)
    full = O.forward_fp64_maps(g, c, s, maps, mu, pdf)
    ynorm = float(np.asarray(pdf, np.float32).astype(np.float64).sum())
    rng = np.random.default_rng(seed)
    meas = (full / ynorm * np.exp(noise * rng.standard_normal(full.shape))).astype(np.float32)
    # the gradient is taken away from the phantom that made the data
    at = np.round(maps.astype(np.float64) * 0.95).astype(np.int16)
    return g, c, s, at, mu, pdf, meas


def _ctx(g, at, mu, pdf):
    geo = vct.Geometry.with_channels(g.width, views=g.views, recon_size=g.recon_size, pixel_cm=g.pixel_cm)
    ctx = vct.Context(geo)
    ctx.set_maps(at)
    ctx.set_spectrum(mu, pdf)
    return ctx


def _grad_errors(dev, ref):
    d = np.asarray(dev, np.float64) - ref
    return float(np.abs(d).max() / np.abs(ref).max()), float(np.linalg.norm(d) / np.linalg.norm(ref))


@pytest.mark.parametrize("N,views,channels", [(64, 40, 609), (63, 36, 609), (64, 40, 512), (128, 120, 609),
                                              (96, 60, 800)])
def test_gradient_matches_fp64_oracle(cuda_device, N, views, channels):
    g, c, s, at, mu, pdf, meas = _case(N, views, channels, seed=N + views)
    with _ctx(g, at, mu, pdf) as ctx:
        loss, grad = ctx.forward_adjoint(meas)
    ref_loss, ref = O.loss_grad(g, c, s, at.astype(np.float64) / 1000.0, mu, pdf, meas)
    assert abs(loss - ref_loss) <= LOSS_RTOL * ref_loss
    mx, l2 = _grad_errors(grad, ref)
    assert mx < GRAD_MAX_REL and l2 < GRAD_L2_REL, (mx, l2)


def test_gradient_with_weights(cuda_device):
    g, c, s, at, mu, pdf, meas = _case(64, 40, 609, seed=11)
    w = np.random.default_rng(4).uniform(0.5, 2.0, meas.shape).astype(np.float32)
    with _ctx(g, at, mu, pdf) as ctx:
        loss, grad = ctx.forward_adjoint(meas, weights=w)
    ref_loss, ref = O.loss_grad(g, c, s, at.astype(np.float64) / 1000.0, mu, pdf, meas, weights=w)
    assert abs(loss - ref_loss) <= LOSS_RTOL * ref_loss
    mx, l2 = _grad_errors(grad, ref)
    assert mx < GRAD_MAX_REL and l2 < GRAD_L2_REL, (mx, l2)


@pytest.mark.parametrize("channels", [609, 512])
def test_dot_product_device_pair(cuda_device, channels):
    """<A x, g> = <x, A^T g> with A = vct_line_integrals_dev and
    A^T = vct_adjoint_rays_dev, both on the device."""
    import torch

    N, views = 96, 60
    g, c, s, _, mu, pdf, _ = _case(N, views, channels, seed=3)
    rng = np.random.default_rng(8)
    x = rng.integers(0, 1000, (6, N, N)).astype(np.int16)
    w = rng.standard_normal((views, channels, 6)).astype(np.float32)
    with _ctx(g, x, mu, pdf) as ctx:
        L = torch.zeros((views, channels, 6), dtype=torch.float64, device="cuda")
        ctx.line_integrals_dev(L)
        wt = torch.from_numpy(w).cuda()
        out = torch.zeros((6, N, N), dtype=torch.float32, device="cuda")
        ctx.adjoint_rays_dev(wt, out)
        torch.cuda.synchronize()
        lhs = float((L.cpu().numpy() * w).sum())
        rhs = float((x.astype(np.float64) / 1000.0 * out.cpu().numpy()).sum())
    assert abs(lhs - rhs) <= 1e-5 * np.abs(L.cpu().numpy() * w).sum()
    ref = O.walk_backproject(g, c, s, w.astype(np.float64))
    mx, l2 = _grad_errors(out.cpu().numpy(), ref)
    assert mx < GRAD_MAX_REL and l2 < GRAD_L2_REL, (mx, l2)


def test_vjp_matches_loss_gradient(cuda_device):
    """dl/d(y/ynorm) of the loss, fed to the VJP entry point, gives the loss's
    gradient."""
    import torch

    g, c, s, at, mu, pdf, meas = _case(64, 40, 609, seed=21)
    with _ctx(g, at, mu, pdf) as ctx:
        loss, grad = ctx.forward_adjoint(meas)
        y = ctx.forward().astype(np.float64)
        ynorm = float(np.asarray(pdf, np.float32).astype(np.float64).sum())
        p = meas.astype(np.float64)
        ok = p > 0
        r = np.where(ok, np.log(y / ynorm) - np.log(np.where(ok, p, 1.0)), 0.0)
        dy = np.where(ok, p * r / (y / ynorm), 0.0).astype(np.float32)
        out = torch.zeros((6, 64, 64), dtype=torch.float32, device="cuda")
        ctx.forward_vjp_dev(torch.from_numpy(dy).cuda(), out)
        torch.cuda.synchronize()
        vjp = out.cpu().numpy()
    mx, l2 = _grad_errors(vjp, grad.astype(np.float64))
    assert mx < 1e-4 and l2 < 1e-4, (mx, l2)


@pytest.mark.parametrize("channels", [609, 512])
def test_deterministic(cuda_device, channels):
    g, c, s, at, mu, pdf, meas = _case(128, 120, channels, seed=2)
    with _ctx(g, at, mu, pdf) as ctx:
        l1, g1 = ctx.forward_adjoint(meas)
        l2, g2 = ctx.forward_adjoint(meas)
    assert l1 == l2
    assert np.array_equal(g1.view(np.uint32), g2.view(np.uint32))


def test_adjoint_c4_full_size(cuda_device):
    """512^2, 6 elements, 120 kV, 800 views x 609 channels, noisy measured
    sinogram: the device gradient against the FP64 oracle everywhere, and
    against central finite differences (h = 1e-3 relative) of the FP64 loss
    on 64 random pixels inside the object."""
    t = golden("mu_tables.npz")
    mu, pdf = t["kramers120_mu"], t["kramers120_pdf"]
    g = O.geom()
    c, s = O.trig_tables(g.views)
    maps = phantoms.ellipse_phantom(0, 512)
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(mu, pdf)
        meas = ctx.mbfpa(sigma=5.37e-5, seed=7)  # max-normalised, noisy
        at = np.round(maps.astype(np.float64) * 0.97).astype(np.int16)
        ctx.set_maps(at)
        loss, grad = ctx.forward_adjoint(meas)
    rho = at.astype(np.float64) / 1000.0
    ref_loss, ref = O.loss_grad(g, c, s, rho, mu, pdf, meas)
    assert abs(loss - ref_loss) <= LOSS_RTOL * ref_loss
    mx, l2 = _grad_errors(grad, ref)
    assert mx < GRAD_MAX_REL and l2 < GRAD_L2_REL, (mx, l2)
    rng = np.random.default_rng(64)
    scale = np.abs(ref).max()
    inside = np.argwhere(rho.sum(0) > 0.2)
    for k in range(64):
        m = int(rng.integers(6))
        row, col = inside[rng.integers(len(inside))]
        h = 1e-3 * max(rho[m, row, col], 1e-3)
        fd = O.fd_pixel(g, c, s, rho, m, int(col), int(row), h, mu, pdf, meas)
        assert abs(grad[m, row, col] - fd) <= 1e-3 * abs(fd) + 1e-5 * scale, (m, row, col, grad[m, row, col], fd)
