"""FBP on the GPU against the reference's filterSinogram + reconstructImage
(fixtures from its own code) and the oracle (bit-exact restatement)."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import FBP_ATOL_REL, FBP_L2_REL, fbp_errors, golden
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu


def device_copy(ptr, shape, dtype):
    """Host copy of a device buffer given by raw pointer (via torch)."""
    import torch

    class _Dev:
        def __init__(self):
            self.__cuda_array_interface__ = {"shape": shape, "typestr": np.dtype(dtype).str,
                                             "data": (ptr, False), "version": 3}

    torch.cuda.synchronize()
    return torch.as_tensor(_Dev(), device="cuda").cpu().numpy().copy()


@pytest.mark.parametrize("filt", [1, 2])
def test_small_fbp_matches_reference(cuda_device, filt):
    d = golden("fbp_small.npz")
    with vct.Context(vct.Geometry(views=40, recon_size=64, pixel_cm=0.4)) as ctx:
        img = ctx.fbp(d["sino"], filt)
        qq = device_copy(ctx.fbp_filtered_ptr(), (40, 609), np.float32)
    a, l2 = fbp_errors(img, d[f"img_f{filt}"])
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL
    fa, fl2 = fbp_errors(qq, d[f"fltd_f{filt}"])
    assert fa < 1e-5 and fl2 < 1e-5


@pytest.mark.parametrize("filt", [1, 2])
def test_full_size_fbp_matches_oracle(cuda_device, filt):
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(3, 512)
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        sino = ctx.mbfpa(0.0, 1)
        img = ctx.fbp(sino, filt)
    g = O.geom()
    c, s = O.trig_tables(800)
    ref, _ = O.fbp(g, sino, filt, c, s)
    a, l2 = fbp_errors(img, ref)
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (a, l2)
    assert not img[O.mask(512) == 0].any()


def test_in_mode_window(cuda_device):
    """"IN" class: filtered samples outside [1000, 3e5] are zeroed (:250-255)."""
    d = golden("fbp_small.npz")
    sino = (d["sino"] * 1e-6).astype(np.float32)  # large -ln p: filtered values spread over the window
    with vct.Context(vct.Geometry(views=40, recon_size=64, pixel_cm=0.4)) as ctx:
        ctx.fbp(sino, 1, in_mode=False)
        plain = device_copy(ctx.fbp_filtered_ptr(), (40, 609), np.float32)
        ctx.fbp(sino, 1, in_mode=True)
        win = device_copy(ctx.fbp_filtered_ptr(), (40, 609), np.float32)
    keep = (plain >= 1000.0) & (plain <= 300000.0)
    assert keep.any() and (~keep).any()
    assert np.array_equal(win, np.where(keep, plain, 0).astype(np.float32))


@pytest.mark.parametrize("views,N", [(42, 64), (40, 63), (41, 96), (36, 128)])
def test_fbp_general_and_symmetric_paths(cuda_device, views, N):
    """V % 4 == 0 with even N takes the quarter-turn-symmetric backprojector;
    every other shape the general one.  Both against the oracle."""
    t = golden("mu_tables.npz")
    pix = 25.6 / N
    g = O.geom(views=views, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(views)
    maps = phantoms.ellipse_phantom(4, N, border_px=2)
    sino = O.forward_exact(g, c, s, O.rho_from_maps(maps), t["kramers120_mu"], t["kramers120_pdf"])
    sino, _ = O.normalize_noise(sino, 0.0)
    if views % 2:
        sino[-1] = 1.0  # the row the reference leaves 0 is read by the filter as p = 1
    for filt in (1, 2):
        ref, _ = O.fbp(g, sino, filt, c, s)
        with vct.Context(vct.Geometry(views=views, recon_size=N, pixel_cm=pix)) as ctx:
            img = ctx.fbp(sino, filt)
        a, l2 = fbp_errors(img, ref)
        assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (filt, a, l2)
