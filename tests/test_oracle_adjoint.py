"""The FP64 adjoint oracle (no counterpart in the reference, which has no
gradient): the walk operator A and its transpose pass the dot-product test,
and the gradient of the weighted log least-squares loss matches central
finite differences of the FP64 loss, including the border pixels that the
reference walk's lumped first segment and folded cells reach."""
import numpy as np
import pytest

import oracle as O
from conftest import golden
from virtualct_b200 import phantoms


def _setup(N=48, views=24, channels=609, seed=5):
    t = golden("mu_tables.npz")
    mu, pdf = t["kramers120_mu"], t["kramers120_pdf"]
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.1)
    c, s = O.trig_tables(views)
    maps = phantoms.ellipse_phantom(seed, N, border_px=1)
    full = O.forward_fp64_maps(g, c, s, maps, mu, pdf)
    ynorm = float(np.asarray(pdf, np.float32).astype(np.float64).sum())
    rng = np.random.default_rng(seed)
    meas = (full / ynorm * np.exp(0.02 * rng.standard_normal(full.shape))).astype(np.float32)
    rho = (maps.astype(np.float64) / 1000.0) * 0.95
    return g, c, s, rho, mu, pdf, meas


@pytest.mark.parametrize("channels", [609, 512])
def test_walk_operator_dot_product(channels):
    g, c, s, _, _, _, _ = _setup(channels=channels)
    rng = np.random.default_rng(1)
    x = rng.random((3, g.recon_size, g.recon_size))
    w = rng.standard_normal((g.views, g.width, 3))
    lhs = float((O.walk_project(g, c, s, x) * w).sum())
    rhs = float((x * O.walk_backproject(g, c, s, w)).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_walk_project_equals_forward_line_integrals():
    g, c, s, _, mu, pdf, _ = _setup()
    maps = phantoms.ellipse_phantom(2, g.recon_size, border_px=0)
    _, lint = O.forward_fp64_maps(g, c, s, maps, mu, pdf, want_lint=True)
    L = O.walk_project(g, c, s, maps.astype(np.float64) / 1000.0)
    assert np.abs(L - lint).max() <= 1e-12 * np.abs(lint).max()


@pytest.mark.parametrize("channels", [609, 512])
def test_fp64_gradient_matches_central_differences(channels):
    g, c, s, rho, mu, pdf, meas = _setup(channels=channels)
    loss, grad = O.loss_grad(g, c, s, rho, mu, pdf, meas)
    assert loss > 0
    N = g.recon_size
    rng = np.random.default_rng(3)
    picks = [(0, 0, 0), (3, 0, N // 2), (3, N // 2, 0), (5, N - 1, N // 2), (1, N // 2, N - 1)]
    picks += [(int(rng.integers(6)), int(rng.integers(N)), int(rng.integers(N))) for _ in range(11)]
    scale = np.abs(grad).max()
    for m, row, col in picks:
        h = 1e-3 * max(rho[m, row, col], 1e-3)
        fd = O.fd_pixel(g, c, s, rho, m, col, row, h, mu, pdf, meas)
        # the full-loss difference gives the same number: rays that cannot
        # touch the pixel cancel exactly
        assert abs(fd - grad[m, row, col]) <= 1e-6 * abs(fd) + 1e-9 * scale, (m, row, col)


@pytest.mark.parametrize("N,views,channels", [(64, 40, 609), (63, 36, 512)])
@pytest.mark.parametrize("filt", [1, 2])
def test_fbp_transpose_dot_product(N, views, channels, filt):
    """<FBP(exp(-lam)), u> = <lam, FBP^T u>: the FP64 transpose against the
    oracle FBP that is pinned to the reference."""
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.1)
    c, s = O.trig_tables(views)
    rng = np.random.default_rng(N + filt)
    p = np.exp(-rng.uniform(0.1, 3.0, (views, channels))).astype(np.float32)
    lam = -np.log(p.astype(np.float64))
    img, _ = O.fbp(g, p, filt, c, s)
    u = rng.standard_normal((N, N))
    lt = O.fbp_transpose(g, u, filt, c, s)
    lhs = float((img.astype(np.float64) * u).sum())
    rhs = float((lam * lt).sum())
    assert abs(lhs - rhs) <= 1e-7 * float(np.abs(img * u).sum())
