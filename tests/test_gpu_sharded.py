"""One slice split over simulated ranks on the GPU, through the C ABI: the
pieces of vct_forward_views_dev / vct_normalize_noise_rows_dev (with the
ranks' (max, min) combined) and vct_fbp_band_dev (disjoint bands summed)
equal vct_mbfpa_dev and vct_fbp_dev bit for bit, for both backprojectors;
and virtualct_b200.sharded on a single rank does too.  (The collectives are
checked on CPU with gloo in tests/test_sharded_cpu.py.)"""
import numpy as np
import pytest

import virtualct_b200 as vct
from virtualct_b200 import phantoms
from virtualct_b200.sharded import ShardedSlice, split

pytestmark = pytest.mark.gpu

SIGMA = 5.37e-5


# (N, pixel, views, channels): quarter-turn backprojector (views % 4 == 0,
# even N) and the general one (odd view count: a zero pad row; odd N)
@pytest.mark.parametrize("N,pix,views,channels", [(256, 0.2, 200, 609), (127, 0.4, 121, 512)])
@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_pieces_equal_one_gpu(cuda_device, N, pix, views, channels, world):
    import torch

    geo = vct.Geometry.with_channels(channels, views=views, recon_size=N, pixel_cm=pix)
    mu, pdf = phantoms.kramers_tables(120)
    with vct.Context(geo) as ctx:
        # one stream for the kernels and torch's ops (torch's default stream has
        # handle 0, which means the context's own stream: 1 is cudaStreamLegacy)
        ctx.set_stream(torch.cuda.current_stream().cuda_stream or 1)
        ctx.set_maps(phantoms.ellipse_phantom(5, N, border_px=2))
        ctx.set_spectrum(mu, pdf)
        ref = torch.empty((views, geo.width), device="cuda")
        ctx.mbfpa_dev(SIGMA, 9, ref)
        ref_img = torch.empty((N, N), device="cuda")
        ctx.fbp_dev(ref, ref_img, 2)
        used = views // 2 * 2
        out = torch.full((views, geo.width), -1.0, device="cuda")
        mm = torch.empty((world, 2), device="cuda")
        for r in range(world):
            r0, r1 = split(views, world, r)
            ctx.forward_views_dev(min(r0, used), min(r1, used), out, mm[r])
            if r1 > used:
                out[max(r0, used):r1].zero_()
        glob = torch.stack([mm[:, 0].max(), mm[:, 1].min()]).contiguous()
        for r in range(world):
            r0, r1 = split(views, world, r)
            ctx.normalize_noise_rows_dev(out, r0, r1, glob, SIGMA, 9)
        img = torch.zeros((N, N), device="cuda")
        nb = ctx.fbp_band_count()
        assert nb == (N // 2 if views % 4 == 0 and N % 2 == 0 else N)
        for r in range(world):
            part = torch.zeros((N, N), device="cuda")
            ctx.fbp_band_dev(ref, *split(nb, world, r), part, filter=2)
            img += part
        one = ShardedSlice(ctx)
        o1 = torch.empty_like(ref)
        one.mbfpa(SIGMA, 9, o1)
        i1 = torch.empty_like(ref_img)
        one.fbp(o1, i1, filter=2)
        torch.cuda.synchronize()
    for got in (out, o1):
        assert torch.equal(got.view(torch.int32), ref.view(torch.int32))
    for got in (img, i1):
        assert torch.equal(got.view(torch.int32), ref_img.view(torch.int32))
