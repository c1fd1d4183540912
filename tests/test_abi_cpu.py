"""Host-side checks of libvct.so that need no GPU: the library loads, exports
every entry point include/*.h declares, and its host logic (spectrum model,
txt parsers, Philox) matches the reference / published vectors."""
import os
import re

import numpy as np
import pytest

import virtualct_b200 as vct
from conftest import GOLDEN, REF_MB, ROOT, golden, have_reference_sources
from virtualct_b200 import phantoms


def declared_symbols():
    names = set()
    for h in ("vct.h", "vct_io.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(vct_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    L = vct.lib()
    decl = declared_symbols()
    assert decl == set(vct.EXPORTED_SYMBOLS), decl ^ set(vct.EXPORTED_SYMBOLS)
    for name in decl:
        assert hasattr(L, name), name


def test_index_checked_library_exports_the_same_symbols():
    import ctypes

    path = os.path.join(ROOT, "virtualct_b200", "lib", "libvct_bounds.so")
    assert os.path.exists(path), "libvct_bounds.so not built"
    B = ctypes.CDLL(path)
    for name in declared_symbols():
        assert hasattr(B, name), name
    # the product library carries no index checks and says so
    with pytest.raises(vct.VctError) as e:
        vct.bounds_violations()
    assert e.value.code == vct.VCT_E_UNSUPPORTED


def test_attenuation_matches_reference_tables():
    t = golden("mu_tables.npz")
    mu, pdf = vct.attenuation_coefficient(os.path.join(GOLDEN, "kramers_120kvp.txt"))
    assert np.array_equal(pdf, t["kramers120_pdf"]) and np.array_equal(mu, t["kramers120_mu"])


@pytest.mark.skipif(not have_reference_sources(), reason="reference checkout absent")
def test_attenuation_matches_reference_shipped_spectra():
    t = golden("mu_tables.npz")
    for name, f in (("kv120", "PhaseSpace_photon_120kV_0cm.txt"), ("mv6", "PhaseSpace_photon_6MV_0cm.txt")):
        mu, pdf = vct.attenuation_coefficient(os.path.join(REF_MB, "Spectrum", f))
        assert np.array_equal(pdf, t[f"{name}_pdf"]) and np.array_equal(mu, t[f"{name}_mu"])


def test_attenuation_eight_elements_extends_table():
    mu6, _ = vct.attenuation_coefficient(os.path.join(GOLDEN, "kramers_120kvp.txt"))
    mu8, _ = vct.attenuation_coefficient(os.path.join(GOLDEN, "kramers_120kvp.txt"), vct.GAMMEX_ELEMENTS)
    assert mu8.shape == (8, 110) and np.array_equal(mu8[:6], mu6)
    assert np.all(mu8[6] > 0) and np.all(mu8[7] > mu8[6])  # Si attenuates more than Mg


def test_attenuation_c2_tables_match_fixture(tmp_path):
    """The 60-bin 6 MV spectrum through its txt form, 8 elements: the product's
    host model gives the C2 fixture's (oracle) mu and pdf bit for bit."""
    from virtualct_b200 import phantoms

    d = golden("c2_subset.npz")
    p = str(tmp_path / "mv6_60.txt")
    phantoms.write_spectrum_txt(p, phantoms.mv_spectrum())
    mu, pdf = vct.attenuation_coefficient(p, vct.GAMMEX_ELEMENTS)
    assert np.array_equal(pdf, d["pdf"]) and np.array_equal(mu, d["mu"])


def test_attenuation_errors():
    with pytest.raises(vct.VctError) as e:
        vct.attenuation_coefficient("/nonexistent/spectrum.txt")
    assert e.value.code == vct.VCT_E_IO
    with pytest.raises(KeyError):
        vct.attenuation_coefficient(os.path.join(GOLDEN, "kramers_120kvp.txt"), ("H", "Fe"))


def test_philox_known_answers():
    # Known-answer vectors of Philox4x32-10 (Salmon et al., SC'11, Random123 KAT).
    assert vct.philox4x32_10([0, 0, 0, 0], [0, 0]).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    ff = 0xFFFFFFFF
    assert vct.philox4x32_10([ff] * 4, [ff, ff]).tolist() == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert vct.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]).tolist() == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_mb_config_parser_generated_txt(tmp_path):
    import ctypes as C

    p = tmp_path / "in.txt"
    phantoms.write_mb_txt(str(p), spectrum="spec.txt", width=609, views=360, N=256, pixel_cm=0.2, noise=1e-4)
    L = vct.lib()
    cfg = (C.c_byte * 8192)()
    assert L.vct_load_mb_config(str(p).encode(), cfg) == 0
    g = vct._CGeometry()
    L.vct_mb_geometry(cfg, C.byref(g))
    assert (g.views, g.width, g.recon_size, g.xfactor) == (360, 609, 256, 1)
    assert g.pixel_cm == 0.2 and g.sid_cm == 85.0 and g.iso_channel == 304.5


@pytest.mark.skipif(not have_reference_sources(), reason="reference checkout absent")
def test_mb_config_parser_shipped_txt():
    import ctypes as C

    L = vct.lib()
    cfg = (C.c_byte * 8192)()
    assert L.vct_load_mb_config(os.path.join(REF_MB, "IR_TOMO_input_virtual_projection_120kV.txt").encode(), cfg) == 0
    g = vct._CGeometry()
    L.vct_mb_geometry(cfg, C.byref(g))
    assert (g.views, g.width, g.recon_size, g.pixel_cm, g.xfactor) == (800, 609, 512, 0.1, 1)


def test_config_missing_file_is_io_error():
    import ctypes as C

    cfg = (C.c_byte * 8192)()
    assert vct.lib().vct_load_mb_config(b"/nonexistent.txt", cfg) == vct.VCT_E_IO
    assert vct.lib().vct_load_fbp_config(b"/nonexistent.txt", cfg) == vct.VCT_E_IO
    assert b"not found" in vct.lib().vct_last_error()


def test_create_rejects_bad_geometry():
    import torch

    for bad in (dict(views=1), dict(recon_size=1), dict(pixel_cm=0.0), dict(width=100)):
        with pytest.raises(vct.VctError) as e:
            vct.Context(vct.Geometry(**bad))
        assert e.value.code == vct.VCT_E_ARG
    if not torch.cuda.is_available():
        with pytest.raises(vct.VctError) as e:
            vct.Context(vct.Geometry())
        assert e.value.code == vct.VCT_E_CUDA
