"""Transpose of the FBP on the GPU, through the C ABI: against the FP64
transpose of the oracle, and the dot-product test against the device FBP
(<FBP(p), u> = <-ln p, FBP^T u>) for both backprojectors (quarter-turn
symmetric and general) and both filters, up to the full 512^2, 800 x 609
size."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct

pytestmark = pytest.mark.gpu

# FP32 device against FP64: max error relative to the largest entry, L2.
T_MAX_REL = 1e-4
T_L2_REL = 1e-4
DOT_REL = 1e-5


def _case(N, views, channels, seed):
    rng = np.random.default_rng(seed)
    p = np.exp(-rng.uniform(0.1, 3.0, (views, channels))).astype(np.float32)
    u = rng.standard_normal((N, N)).astype(np.float32)
    return p, u


@pytest.mark.parametrize("N,views,channels", [(64, 40, 609), (64, 42, 609), (63, 36, 512), (128, 120, 800)])
@pytest.mark.parametrize("filt", [1, 2])
def test_fbp_transpose_matches_fp64(cuda_device, N, views, channels, filt):
    p, u = _case(N, views, channels, N + views + filt)
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.1)
    c, s = O.trig_tables(views)
    ref = O.fbp_transpose(g, u.astype(np.float64), filt, c, s)
    geo = vct.Geometry.with_channels(channels, views=views, recon_size=N, pixel_cm=0.1)
    with vct.Context(geo) as ctx:
        out = ctx.fbp_transpose(u, filter=filt)
        img = ctx.fbp(p, filter=filt)
    d = out.astype(np.float64) - ref
    assert np.abs(d).max() <= T_MAX_REL * np.abs(ref).max()
    assert np.linalg.norm(d) <= T_L2_REL * np.linalg.norm(ref)
    lam = -np.log(p.astype(np.float64))
    lhs = float((img.astype(np.float64) * u).sum())
    rhs = float((lam * out.astype(np.float64)).sum())
    assert abs(lhs - rhs) <= DOT_REL * float(np.abs(img.astype(np.float64) * u).sum())


def test_fbp_transpose_large_grid_more_parts(cuda_device):
    """1024^2 at 0.05 cm: the scatter splits each base view's 512^2 orbit
    pixels into 64 parts (at most 4096 pixels each, so a shared slot's 32-bit
    fixed-point sums cannot overflow) instead of 16."""
    views, channels, N = 40, 800, 1024
    p, u = _case(N, views, channels, 7)
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.05)
    c, s = O.trig_tables(views)
    ref = O.fbp_transpose(g, u.astype(np.float64), 1, c, s)
    geo = vct.Geometry.with_channels(channels, views=views, recon_size=N, pixel_cm=0.05)
    with vct.Context(geo) as ctx:
        out = ctx.fbp_transpose(u, filter=1)
        img = ctx.fbp(p, filter=1)
    d = out.astype(np.float64) - ref
    assert np.abs(d).max() <= T_MAX_REL * np.abs(ref).max()
    assert np.linalg.norm(d) <= T_L2_REL * np.linalg.norm(ref)
    lam = -np.log(p.astype(np.float64))
    lhs = float((img.astype(np.float64) * u).sum())
    rhs = float((lam * out.astype(np.float64)).sum())
    assert abs(lhs - rhs) <= DOT_REL * float(np.abs(img.astype(np.float64) * u).sum())


@pytest.mark.parametrize("filt", [1, 2])
def test_fbp_transpose_dot_product_full_size(cuda_device, filt):
    import torch

    p, u = _case(512, 800, 609, 99 + filt)
    with vct.Context(vct.Geometry()) as ctx:
        pt = torch.from_numpy(p).cuda()
        ut = torch.from_numpy(u).cuda()
        img = torch.zeros((512, 512), dtype=torch.float32, device="cuda")
        lt = torch.zeros((800, 609), dtype=torch.float32, device="cuda")
        ctx.fbp_dev(pt, img, filter=filt)
        ctx.fbp_transpose_dev(ut, lt, filter=filt)
        torch.cuda.synchronize()
        img, lt = img.cpu().numpy().astype(np.float64), lt.cpu().numpy().astype(np.float64)
    lam = -np.log(p.astype(np.float64))
    lhs = float((img * u).sum())
    rhs = float((lam * lt).sum())
    assert abs(lhs - rhs) <= DOT_REL * float(np.abs(img * u).sum())
