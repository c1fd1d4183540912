"""Beam-hardening correction on the GPU: vct_beam_hardening against the
reference program's output (tests/golden/beam_hardening.npz), the vct_bhc
drop-in in a scratch directory, and the FBP with the correction folded into
its -ln step against the FBP of the separately corrected sinogram."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import FBP_ATOL_REL, FBP_L2_REL, SINO_RTOL, fbp_errors, golden
from golden_cases import BH_PARAMS, BH_ROW_STEP, bh_sino

pytestmark = pytest.mark.gpu

# The sinogram tolerance.  The device's logf and glibc's differ in the last
# bit for some inputs (glibc's is not correctly rounded either); the
# correction's alpha*beta*|y|^(beta-1) factor magnifies that up to ~2e-6 for
# the MV parameters at the most attenuated rays.
BH_RTOL = SINO_RTOL


@pytest.mark.parametrize("k", range(len(BH_PARAMS)))
def test_beam_hardening_matches_reference(cuda_device, k):
    a, b = BH_PARAMS[k]
    with vct.Context(vct.Geometry()) as ctx:
        cor = ctx.beam_hardening(bh_sino(), a, b)
    ref = golden("beam_hardening.npz")[f"rows_{k}"].astype(np.float64)
    got = cor[::BH_ROW_STEP].astype(np.float64)
    assert np.max(np.abs(got - ref) / np.abs(ref)) < BH_RTOL


def test_bhc_dropin(cuda_device, tmp_path):
    bh_sino().tofile(tmp_path / "reprojection_float.raw")
    exe = os.path.join(os.path.dirname(vct.__file__), "bin", "vct_bhc")
    r = subprocess.run([exe, "0.01", "2.00"], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    d = golden("beam_hardening.npz")
    assert r.stdout.strip() == str(d["line_0"])
    out = np.fromfile(tmp_path / "reprojection_float_cor.raw", np.float32).reshape(800, 609)
    ref = d["rows_0"].astype(np.float64)
    assert np.max(np.abs(out[::BH_ROW_STEP] - ref) / ref) < BH_RTOL
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "no alpha and beta" in r.stderr


@pytest.mark.parametrize("filt", [1, 2])
def test_fbp_with_folded_correction(cuda_device, filt):
    N, V = 128, 120
    p = np.exp(-np.random.default_rng(filt).uniform(0.05, 4.0, (V, 609))).astype(np.float32)
    a, b = 0.01, 2.0
    cor, _ = O.beam_hardening(p, a, b)
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=0.2)) as ctx:
        ref = ctx.fbp(cor, filter=filt)
        ctx.set_beam_hardening(a, b)
        img = ctx.fbp(p, filter=filt)
        ctx.set_beam_hardening(0.0, 0.0)
        plain = ctx.fbp(cor, filter=filt)
    assert np.array_equal(plain, ref)
    mx, l2 = fbp_errors(img, ref)
    assert mx < FBP_ATOL_REL and l2 < FBP_L2_REL, (mx, l2)
