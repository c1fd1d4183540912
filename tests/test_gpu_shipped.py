"""The CUDA path on the reference's own shipped cases, and on the 6 MV
configuration at full size.

Fixtures (tests/golden/make_golden.py, from the reference compiled from its
sources and the pinned oracle):
  icru_shipped.npz  Weight_input_ICRU110.raw with the shipped 100-bin 120 kV and
                    650-bin 6 MV spectra (MB/main.cpp:421-530, noise-free), and
                    rows of the shipped noisy reprojection_float.raw;
  fbp_human.npz     Release_FBP_CPU/reprojection_float.raw and rows of the
                    shipped FBP_virtual_projection_512x512_human.raw (Shepp-Logan,
                    FBP/main.cpp:137-167);
  c2_subset.npz     512^2, 8 elements, 16-insert cylinder, 60-bin 6 MV, 800 x 609.
Tolerances: sinograms 1e-5 relative per element against the reference, 1e-6
against the FP64 sum; FBP images 1e-4 of max|ref| per pixel and 1e-4 relative
L2 against the reference and against the FBP with every sum in FP64.
"""
import math

import numpy as np
import pytest

import virtualct_b200 as vct
from conftest import FBP_ATOL_REL, FBP_L2_REL, SINO_RTOL, fbp_errors, golden, max_rel
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu

# Device forward against the FP64 sum of the same walk (the SFU exponential of
# the compensated spectral sum and the final float rounding; the reference
# itself is up to 8e-7 from FP64 on these inputs).
FP64_RTOL = 1e-6


def _icru_forward(name):
    d = golden("icru_shipped.npz")
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(d["maps"])
        ctx.set_spectrum(d[f"{name}_mu"], d[f"{name}_pdf"])
        out = ctx.forward()
        norm, stats = ctx.mbfpa(0.0, 1, return_stats=True)
    return d, out, norm, stats


@pytest.mark.parametrize("name,nbins", [("kv120", 100), ("mv6", 650)])
def test_icru110_shipped_spectra_match_reference(cuda_device, name, nbins):
    """The shipped ICRU-110 phantom with the shipped spectrum, noise-free:
    every 20th view against reprojection_TOMO summed over all bins."""
    d, out, norm, stats = _icru_forward(name)
    assert d[f"{name}_pdf"].shape == (nbins,)
    rows = d["rows"]
    assert max_rel(out[rows], d[f"{name}_rows"]) < SINO_RTOL
    assert max_rel(out[rows], d[f"{name}_fp64_rows"]) < FP64_RTOL
    if name == "kv120":
        assert abs(float(stats[0]) / float(d["kv120_max"]) - 1) < SINO_RTOL
        ref_min = float(d["kv120_min"]) / float(d["kv120_max"])
        assert abs(float(stats[1]) / ref_min - 1) < 2 * SINO_RTOL


def test_icru110_shipped_noisy_sinogram_statistics(cuda_device):
    """The shipped noisy sinogram (sigma 5.37e-5, glibc rand()) against the
    device's noise-free normalised sinogram of the same inputs: unclamped
    residuals are N(0, sigma^2) and the two clamps of gaussiannoise0
    (MB/main.cpp:51-76: p < 0 -> projection_min/10, p > 1 -> 1) fire as often
    as the noise-free values predict."""
    d, out, norm, stats = _icru_forward("kv120")
    sigma = float(d["sigma"])
    clean = norm[d["noisy_rows"]].astype(np.float64)
    gold = d["noisy"]
    floor = np.float32(float(stats[1]) / 10.0)
    hi, lo = gold == np.float32(1.0), np.isclose(gold, floor, rtol=1e-5, atol=0)
    # residual statistics on the rays whose noise-free value is away from both
    # clamps (near one, the unclamped samples are a truncated distribution)
    away = (clean > 8 * sigma) & (clean < 1 - 8 * sigma)
    assert not (hi | lo)[away].any()
    r = (gold[away].astype(np.float64) - clean[away]) / sigma
    n = r.size
    assert n > 20000
    assert abs(r.mean()) < 6 / math.sqrt(n)
    assert abs(r.var() - 1) < 6 * math.sqrt(2 / (n - 1))
    # clamp counts against their expectations sum Phi(.) over the samples
    phi = np.vectorize(lambda x: 0.5 * math.erfc(-x / math.sqrt(2)))
    e_hi = float(phi((clean - 1.0) / sigma).sum())
    e_lo = float(phi(-clean / sigma).sum())
    assert e_hi > 100 and e_lo > 0
    assert abs(hi.sum() - e_hi) < 6 * math.sqrt(e_hi) + 3, (hi.sum(), e_hi)
    assert abs(lo.sum() - e_lo) < 6 * math.sqrt(e_lo) + 3, (lo.sum(), e_lo)


def test_shipped_human_fbp_matches_reference(cuda_device):
    """FBP/reprojection_float.raw -> FBP_virtual_projection_512x512_human.raw
    (Shepp-Logan, 800 x 609 -> 512^2) on the device, every 8th row."""
    d = golden("fbp_human.npz")
    with vct.Context(vct.Geometry()) as ctx:
        img = ctx.fbp(d["sino"], int(d["filter"]))
    rows = d["rows"]
    a, l2 = fbp_errors(img[rows], d["golden_rows"])
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (a, l2)
    a, l2 = fbp_errors(img[rows], d["fp64_rows"])
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (a, l2)


def test_c2_full_size_matches_oracle(cuda_device):
    """The 6 MV configuration at its stated size: 512^2 at 0.1 cm, 8 elements
    (H C N O P Ca Mg Si), the seeded 33 cm cylinder with 16 inserts, the
    synthetic 60-bin 6 MV spectrum, 800 x 609; the forward against the pinned
    oracle (reference arithmetic) and FP64, then the Shepp-Logan FBP of the
    max-normalised, noise-free sinogram."""
    d = golden("c2_subset.npz")
    maps = phantoms.gammex_cylinder_phantom(int(d["seed"]), 512)
    import hashlib

    assert hashlib.sha256(maps.tobytes()).digest() == d["maps_sha"].tobytes()
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(d["mu"], d["pdf"])
        out = ctx.forward()
        norm, stats = ctx.mbfpa(0.0, 1, return_stats=True)
        img = ctx.fbp(norm, 2)
    rows = d["rows"]
    assert max_rel(out[rows], d["full_rows"]) < SINO_RTOL
    assert max_rel(out[rows], d["fp64_rows"]) < FP64_RTOL
    assert abs(float(stats[0]) / float(d["max"]) - 1) < SINO_RTOL
    step = 512 // d["fbp_sl_rows"].shape[0]
    a, l2 = fbp_errors(img[::step], d["fbp_sl_rows"])
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (a, l2)
    a, l2 = fbp_errors(img[::step], d["fbp_sl_fp64_rows"])
    assert a < FBP_ATOL_REL and l2 < FBP_L2_REL, (a, l2)
