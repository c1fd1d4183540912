"""The drop-in executables on the GPU: bin/vct_mbfpa and bin/vct_fbp run in a
scratch directory on inputs written in the reference's own formats (the
31-field and 21-field txts, int16 weights, the spectrum txt) and give the
library's results: the noise-free reprojection and the FBP image bit for
bit, npf_float.raw all zeros (lengthproj_TOMO of the virtual path's absent
measured sinogram, as the reference's shipped npf_float.raw), and the
iterative step's ReconImageRaw/ images equal to vct_ir_step's."""
import os
import subprocess

import numpy as np
import pytest

import virtualct_b200 as vct
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(vct.__file__), "bin")


def test_dropin_mbfpa_and_fbp(cuda_device, tmp_path):
    N, V = 128, 80
    os.makedirs(tmp_path / "Spectrum")
    spec = "Spectrum/kramers120.txt"
    phantoms.write_spectrum_txt(tmp_path / spec, phantoms.kramers_spectrum(120))
    maps = phantoms.ellipse_phantom(17, N, border_px=4)
    maps.tofile(tmp_path / "Weight_input_ICRU110.raw")
    phantoms.write_mb_txt(tmp_path / "mb.txt", spectrum=spec, views=V, N=N, pixel_cm=0.1, noise=0.0)
    r = subprocess.run([os.path.join(BIN, "vct_mbfpa"), "mb.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    sino = np.fromfile(tmp_path / "reprojection_float.raw", np.float32).reshape(V, 609)
    npf = np.fromfile(tmp_path / "npf_float.raw", np.float32)
    assert npf.shape == (N * N,) and not npf.any()

    mu, pdf = vct.attenuation_coefficient(tmp_path / spec)
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=0.1)) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(mu, pdf)
        ref = ctx.mbfpa(sigma=0.0)
        img_ref = ctx.fbp(ref, filter=2)
    assert np.array_equal(sino.view(np.uint32), ref.view(np.uint32))

    # the iterative step's outputs (MB/main.cpp:432-600): the first element's
    # map after one IR_ImageTOMO update, and its int16 form
    it1 = np.fromfile(tmp_path / "ReconImageRaw" / "Reconstruction_ite0001_z0000.raw", np.float32).reshape(N, N)
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=0.1)) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(mu, pdf)
        before = maps[0].astype(np.float32) / np.float32(1000)
        after, wb, obj, _ = ctx.ir_step(np.zeros((V, 609), np.float32), np.zeros((N, N), np.float32), before,
                                        ite=1, thinout=10, num_ite=500, w_tv=1e-4, w_prior=0.0, wbefore=0.0105)
    assert wb == pytest.approx(0.0106) and obj < 1e7
    assert np.array_equal(it1.view(np.uint32), after.view(np.uint32))
    s16 = np.fromfile(tmp_path / "ReconImageRaw" / "Reconstruction_512x512x1.raw", np.int16).reshape(N, N)
    assert np.array_equal(s16, (1024 * (after.astype(np.float64) - 0.0716) / 0.0716).astype(np.int16))

    phantoms.write_fbp_txt(tmp_path / "fbp.txt", sino="reprojection_float.raw", out="img.raw", filter=2, views=V,
                           N=N, pixel_cm=0.1)
    r = subprocess.run([os.path.join(BIN, "vct_fbp"), "fbp.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    img = np.fromfile(tmp_path / "img.raw", np.float32).reshape(N, N)
    assert np.array_equal(img.view(np.uint32), img_ref.view(np.uint32))
