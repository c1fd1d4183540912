"""vct_fbp_noalloc: FBP for callers that cannot allocate device memory.

Some callers of this library cannot call cudaMalloc where they reconstruct --
their device memory belongs to another allocator or a fixed budget, they run
a real-time loop that must not wait on an allocation, or they are library code
that may not fail on one.  vct_fbp_noalloc serves them: its intermediate
buffers are static device arrays inside libvct, so the call allocates nothing.
These tests call it through the C ABI and compare it with the context FBP
(vct_fbp_dev) at the FBP tolerance, on consecutive calls.  The file is named
to be collected last: if it fails, a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

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
