"""vct_fbp_noalloc: FBP for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc where they reconstruct --
their device memory belongs to another allocator or a fixed budget, they run
a real-time loop that must not wait on an allocation, or they are library code
that may not fail on one.  vct_fbp_noalloc serves them: its intermediate
buffers are static device arrays inside libvct, so the call allocates nothing.
These tests call it through the C ABI and compare it with the context FBP
(vct_fbp_dev) at the FBP tolerance, on consecutive calls, and with the CPU
oracle on a geometry that takes the general backprojector and the "IN" class
window.  The file is named
to be collected last: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import FBP_ATOL_REL, FBP_L2_REL, fbp_errors, golden
from virtualct_b200 import phantoms


def _sinogram(geo, seed):
    t = golden("mu_tables.npz")
    with vct.Context(geo) as ctx:
        ctx.set_maps(phantoms.ellipse_phantom(seed, geo.recon_size))
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        return ctx.mbfpa(0.0, 1)


def test_fbp_noalloc_rejects_sizes_beyond_its_static_scratch():
    g = vct.Geometry(views=2048, recon_size=64, pixel_cm=0.4)  # 2048 x 609 > 1048576
    rc = vct.lib().vct_fbp_noalloc(C.byref(g.to_c()), None, 1, 0, None, None)
    assert rc == vct.VCT_E_ARG  # null buffers are refused first
    rc = vct.lib().vct_fbp_noalloc(C.byref(g.to_c()), 16, 1, 0, 16, None)
    assert rc == vct.VCT_E_ARG and b"static scratch limit" in vct.lib().vct_last_error()
    # the grid limit of vct_create applies too (N*N indices stay in int)
    big = vct.Geometry(views=400, recon_size=8193, pixel_cm=0.01)
    rc = vct.lib().vct_fbp_noalloc(C.byref(big.to_c()), 16, 1, 0, 16, None)
    assert rc == vct.VCT_E_ARG and b"geometry out of range" in vct.lib().vct_last_error()


@pytest.mark.gpu
def test_fbp_noalloc_matches_context_fbp_on_consecutive_calls(cuda_device):
    import torch

    geo = vct.Geometry()  # 800 views x 609 channels, 512 x 512
    sinos = [_sinogram(geo, 21), _sinogram(geo, 22)]
    ref = []
    with vct.Context(geo) as ctx:
        for sino, filt in zip(sinos, (1, 2)):
            ref.append(ctx.fbp(sino, filt))
    gc = geo.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):  # two calls in a row, the second with other data and filter
        for sino, filt, r in zip(sinos, (1, 2), ref):
            d_sino = torch.from_numpy(sino).cuda()
            d_img = torch.full((512, 512), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            rc = vct.lib().vct_fbp_noalloc(C.byref(gc), d_sino.data_ptr(), filt, 0, d_img.data_ptr(), stream)
            assert rc == 0, vct.lib().vct_last_error()
            torch.cuda.synchronize()
            img = d_img.cpu().numpy()
            a, l2 = fbp_errors(img, r)
            assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (call, filt, a, l2)


@pytest.mark.gpu
def test_fbp_noalloc_later_calls_take_no_device_memory(cuda_device):
    """The first call on a device may make the driver allocate the static
    arrays (lazy module loading); later calls take nothing."""
    import torch

    geo = vct.Geometry()
    gc = geo.to_c()
    d_sino = torch.from_numpy(_sinogram(geo, 23)).cuda()
    d_img = torch.empty((512, 512), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert vct.lib().vct_fbp_noalloc(C.byref(gc), d_sino.data_ptr(), 1, 0, d_img.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for filt in (1, 2, 1):
        rc = vct.lib().vct_fbp_noalloc(C.byref(gc), d_sino.data_ptr(), filt, 0, d_img.data_ptr(), stream)
        assert rc == 0, vct.lib().vct_last_error()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


@pytest.mark.gpu
def test_fbp_noalloc_general_backprojector_in_mode_matches_oracle(cuda_device):
    """views % 4 != 0 and odd N (the general backprojector), 31 channels (the
    device-built filter's edge-row factors cover rows that overlap), Shepp-Logan
    and the "IN" class window (filtered values outside [1000, 3e5] zeroed),
    against the CPU oracle, on two calls in a row."""
    import torch

    V, N, CH, pix = 42, 63, 31, 0.4
    g = O.geom(views=V, channels=CH, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(5, N, border_px=2)
    sino = O.forward_exact(g, c, s, O.rho_from_maps(maps), t["kramers120_mu"], t["kramers120_pdf"])
    sino, _ = O.normalize_noise(sino, 0.0)
    # p^10: ten times the line integrals, so the filtered values straddle the
    # window's lower edge
    sino = (sino.astype(np.float64) ** 10).astype(np.float32)
    h = O.fbp_constmap(g, 2)
    q = O.fbp_filter(g, sino, h, 0)
    keep = (q >= 1000.0) & (q <= 300000.0)
    assert keep.any() and (~keep).any()
    # no filtered value so close to a window edge that rounding could move it across
    assert np.min(np.abs(q / 1000.0 - 1.0)) > 1e-5 and np.min(np.abs(q / 300000.0 - 1.0)) > 1e-5
    ref, _ = O.fbp(g, sino, 2, c, s, in_mode=1)
    gc = vct.Geometry.with_channels(CH, views=V, recon_size=N, pixel_cm=pix).to_c()
    d_sino = torch.from_numpy(sino).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        d_img = torch.full((N, N), float("nan"), dtype=torch.float32, device="cuda")
        rc = vct.lib().vct_fbp_noalloc(C.byref(gc), d_sino.data_ptr(), 2, 1, d_img.data_ptr(), stream)
        assert rc == 0, vct.lib().vct_last_error()
        torch.cuda.synchronize()
        a, l2 = fbp_errors(d_img.cpu().numpy(), ref)
        assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (call, a, l2)
