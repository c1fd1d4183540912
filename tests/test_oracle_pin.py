"""The oracle (oracle/vct_oracle.c) against the reference itself.

Pins: (1) golden fixtures produced by the reference compiled from its own
sources (tests/golden/make_golden.py); (2) when the reference checkout is
present, the golden outputs it ships, bit for bit."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, REF_FBP, REF_MB, golden, have_reference_sources
from virtualct_b200 import phantoms


def test_kramers_tables_match_reference():
    t = golden("mu_tables.npz")
    pdf, e = O.spectrum(os.path.join(GOLDEN, "kramers_120kvp.txt"))
    mu = O.attenuation(e)
    assert len(pdf) == 110
    assert np.array_equal(pdf, t["kramers120_pdf"])
    assert np.array_equal(mu, t["kramers120_mu"])


@pytest.mark.skipif(not have_reference_sources(), reason="reference checkout absent")
@pytest.mark.parametrize("name,fname", [("kv120", "PhaseSpace_photon_120kV_0cm.txt"),
                                        ("mv6", "PhaseSpace_photon_6MV_0cm.txt")])
def test_shipped_spectra_tables_match_reference(name, fname):
    t = golden("mu_tables.npz")
    pdf, e = O.spectrum(os.path.join(REF_MB, "Spectrum", fname))
    assert np.array_equal(pdf, t[f"{name}_pdf"])
    assert np.array_equal(O.attenuation(e), t[f"{name}_mu"])


@pytest.mark.parametrize("views", [40, 41])
def test_small_forward_bit_exact(views):
    d = golden("mb_small.npz")
    t = golden("mu_tables.npz")
    g = O.geom(views=views, recon_size=int(d["N"]), pixel_cm=float(d["pixel_cm"]))
    c, s = O.trig_tables(views)
    full = O.forward_exact(g, c, s, O.rho_from_maps(d["maps"]), t["kv120_mu"], t["kv120_pdf"])
    assert np.array_equal(full, d[f"full_v{views}"])
    if views % 2:
        assert not full[-1].any()  # odd view counts leave the last row 0 (reprojection_TOMO.cpp:35)


@pytest.mark.parametrize("filt", [1, 2])
def test_small_fbp_bit_exact(filt):
    d = golden("fbp_small.npz")
    g = O.geom(views=40, recon_size=64, pixel_cm=0.4)
    c, s = O.trig_tables(40)
    img, q = O.fbp(g, d["sino"], filt, c, s)
    assert np.array_equal(q, d[f"fltd_f{filt}"])
    assert np.array_equal(img, d[f"img_f{filt}"])


def test_c1_phantom_generator_is_the_fixtures():
    import hashlib

    d = golden("c1_subset.npz")
    maps = phantoms.ellipse_phantom(int(d["seed"]), 512)
    assert hashlib.sha256(maps.tobytes()).digest() == d["maps_sha"].tobytes()


@pytest.mark.skipif(not have_reference_sources(), reason="reference checkout absent")
def test_shipped_fbp_golden_bit_exact():
    sino = np.fromfile(os.path.join(REF_FBP, "reprojection_float.raw"), np.float32).reshape(800, 609)
    gold = np.fromfile(os.path.join(REF_FBP, "FBP_virtual_projection_512x512_human.raw"), np.float32)
    g = O.geom()
    c, s = O.trig_tables(800)
    img, _ = O.fbp(g, sino, 2, c, s)
    assert np.array_equal(img.reshape(-1), gold)


@pytest.mark.skipif(not have_reference_sources(), reason="reference checkout absent")
def test_shipped_mbfpa_golden_bit_exact():
    """The shipped noisy sinogram (ICRU110, 120 kV, sigma 5.37e-5, glibc rand()
    seed 1) is reproduced bit for bit (about 40 s on 8 cores)."""
    pdf, e = O.spectrum(os.path.join(REF_MB, "Spectrum", "PhaseSpace_photon_120kV_0cm.txt"))
    mu = O.attenuation(e)
    maps = np.fromfile(os.path.join(REF_MB, "Weight_input_ICRU110.raw"), np.int16).reshape(6, 512, 512)
    g = O.geom()
    c, s = O.trig_tables(800)
    full = O.forward_exact(g, c, s, O.rho_from_maps(maps), mu, pdf)
    noisy, pmin = O.normalize_noise(full, 0.0000537, seed=1, order=0)
    gold = np.fromfile(os.path.join(REF_MB, "reprojection_float.raw"), np.float32).reshape(800, 609)
    assert np.array_equal(noisy, gold)
    assert abs(pmin - 1.2622175745491404e-05) < 1e-12
