"""Host-side failure paths, no GPU: truncated input txts, missing measured
files, energy labels the loader does not know, layouts that would take the
reference past its own buffers, and bad shapes for the helical
interpolation -- each a status code and a message, none a crash."""
import os

import numpy as np
import pytest

import virtualct_b200 as vct
from virtualct_b200 import phantoms


def _txt(tmp_path, **kw):
    p = tmp_path / "mb.txt"
    phantoms.write_mb_txt(p, spectrum="s.txt", sino="p.raw", air="a.raw", **kw)
    return p


@pytest.mark.parametrize("keep", [0.25, 0.5, 0.98])
def test_truncated_txts_are_refused(tmp_path, keep):
    full = _txt(tmp_path).read_text()
    short = tmp_path / "short.txt"
    short.write_text(full[: int(len(full) * keep)])
    with pytest.raises(vct.VctError) as e:
        vct.MbConfig.load(short)
    assert e.value.code == vct.VCT_E_IO and "ends before field" in str(e.value)
    fbp = tmp_path / "fbp.txt"
    phantoms.write_fbp_txt(fbp, sino="s.raw", out="o.raw")
    ftxt = fbp.read_text()
    fshort = tmp_path / "fshort.txt"
    fshort.write_text(ftxt[: int(len(ftxt) * keep)])
    import ctypes

    class FbpCfg(ctypes.Structure):  # large enough for vct_fbp_config
        _fields_ = [("raw", ctypes.c_char * 8192)]

    cfg = FbpCfg()
    rc = vct.lib().vct_load_fbp_config(str(fshort).encode(), ctypes.byref(cfg))
    assert rc == vct.VCT_E_IO
    assert vct.lib().vct_load_fbp_config(str(fbp).encode(), ctypes.byref(cfg)) == vct.VCT_OK


def test_complete_txts_still_load(tmp_path):
    cfg = vct.MbConfig.load(_txt(tmp_path, rotations=2))
    assert cfg.total_proj_number == 2 and cfg.proj_height == 800


def test_measured_data_errors(tmp_path):
    cfg = vct.MbConfig.load(_txt(tmp_path))
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        with pytest.raises(vct.VctError) as e:  # neither file exists
            vct.load_measured(cfg)
        assert e.value.code == vct.VCT_E_IO and "p.raw not found" in str(e.value)
        (tmp_path / "p.raw").write_bytes(b"\0" * 16)
        with pytest.raises(vct.VctError) as e:  # the air scan is missing
            vct.load_measured(cfg)
        assert e.value.code == vct.VCT_E_IO and "a.raw not found" in str(e.value)
        (tmp_path / "a.raw").write_bytes(b"\0" * 16)
        with pytest.raises(vct.VctError) as e:  # 27 skipped + 609 used > 609 raw channels
            vct.load_measured(cfg)
        assert e.value.code == vct.VCT_E_UNSUPPORTED
        cfg.in_pr_class = b"XX"
        with pytest.raises(vct.VctError) as e:
            vct.load_measured(cfg)
        assert e.value.code == vct.VCT_E_ARG
    finally:
        os.chdir(cwd)


@pytest.mark.parametrize("shape", [(0, 4, 3), (2, 0, 3), (2, 4, 0)])
def test_helical_rejects_empty_shapes(shape):
    with pytest.raises(vct.VctError) as e:
        vct.helical_sinogram(np.zeros(shape, np.float32))
    assert e.value.code == vct.VCT_E_ARG
