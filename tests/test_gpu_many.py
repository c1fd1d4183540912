"""vct_mbfpa_many on the GPU: the pipelined many-slice call gives, slice by
slice, exactly what vct_set_maps + vct_mbfpa give (seed + i for slice i),
from pinned and from pageable host buffers, and leaves the last slice's maps
in the context."""
import numpy as np
import pytest

import virtualct_b200 as vct
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu

SIGMA = 5.37e-5


@pytest.mark.parametrize("n,pinned", [(5, True), (5, False), (2, True), (1, False), (0, True)])
def test_mbfpa_many_matches_one_slice_calls(cuda_device, n, pinned):
    import torch

    geo = vct.Geometry(views=120, recon_size=128, pixel_cm=0.4)
    mu, pdf = phantoms.kramers_tables(120)
    slices = [phantoms.ellipse_phantom(70 + i, 128, border_px=2) for i in range(n)]
    if pinned:
        slices = [torch.from_numpy(m).pin_memory().numpy() for m in slices]
    with vct.Context(geo) as ctx:
        ctx.set_spectrum(mu, pdf)
        outs, st = ctx.mbfpa_many(slices, sigma=SIGMA, seed=11, return_stats=True)
        assert len(outs) == n
        if n:
            last = ctx.forward()
        for i, m in enumerate(slices):
            ctx.set_maps(m)
            ref, rst = ctx.mbfpa(SIGMA, 11 + i, return_stats=True)
            assert np.array_equal(outs[i].view(np.uint32), ref.view(np.uint32)), i
            assert np.array_equal(st[i], rst), i
        if n:
            assert np.array_equal(last.view(np.uint32), ctx.forward().view(np.uint32))
            assert not np.array_equal(outs[0], outs[-1]) or n == 1


def test_mbfpa_many_checks_arguments(cuda_device):
    geo = vct.Geometry(views=40, recon_size=64, pixel_cm=0.8)
    with vct.Context(geo) as ctx:
        with pytest.raises(vct.VctError) as e:  # no spectrum yet
            ctx.mbfpa_many([np.zeros((6, 64, 64), np.int16)])
        assert e.value.code == vct.VCT_E_STATE
        mu, pdf = phantoms.kramers_tables(120)
        ctx.set_spectrum(mu, pdf)
        with pytest.raises(vct.VctError) as e:  # 5 maps for a 6-element spectrum
            ctx.mbfpa_many([np.zeros((5, 64, 64), np.int16)])
        assert e.value.code == vct.VCT_E_ARG
