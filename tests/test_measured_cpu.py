"""Measured-data ingestion and the helical z-interpolation on the CPU: the
oracle's loader (orc_load_measured, restating MB/projectionDataTOMO.cpp:
324-508) against the reference's own loadProjectionData -- fixtures made by
it (tests/golden/make_golden.py), bit for bit, on inputs the tests
regenerate -- and the oracle's helical interpolation (MB/main.cpp:347-371)
through the reference's MBFPA program end to end: loader, interpolation and
lengthproj_TOMO give its npf_float.raw bit for bit."""
import hashlib
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden, have_reference_sources
from golden_cases import (MEAS_CASES, MEAS_E2E, MEAS_E2E_N, MEAS_E2E_PIX, MEAS_STOP, write_e2e_inputs,
                          write_measured)


def _sha(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def _oracle(d, case, **kw):
    cls, width, views, nskip, rotations, rate = case[:6]
    return O.load_measured(os.path.join(d, "proj.raw"), os.path.join(d, "air.raw"), cls == "IN", width, views, nskip,
                           rotations, rate, **kw)


@pytest.mark.parametrize("name", sorted(MEAS_CASES))
def test_loader_matches_reference(name, tmp_path):
    case = MEAS_CASES[name]
    write_measured(tmp_path, case)
    rc, vol, mask, mx = _oracle(tmp_path, case)
    g = golden("measured.npz")
    assert rc == int(g[f"{name}_rc"])
    assert np.array_equal(_sha(vol), g[f"{name}_vol_sha"])
    assert np.array_equal(_sha(mask), g[f"{name}_mask_sha"])
    assert np.array_equal(vol[:, ::37, ::41], g[f"{name}_vol_sample"], equal_nan=True)
    if case[0] == "IN":
        # only view 0 of each rotation reads the file (the reference's loop
        # indexes rows of its buffer that no read fills): later views are 0,
        # or NaN (mask 1) where the air mean is 0
        later = mask[:, 1:] == 1
        assert np.isnan(vol[:, 1:][later]).all() and mask[:, 0].any()
        assert 0.5 < mx <= 1.0


@pytest.mark.skipif(not (have_reference_sources() and O.ref_available()), reason="reference harness not built")
@pytest.mark.parametrize("name", ["pr_thin2", "in_240hz"])
def test_loader_matches_reference_directly(name, tmp_path):
    case = MEAS_CASES[name]
    write_measured(tmp_path, case)
    cls, width, views, nskip, rotations, rate = case[:6]
    cwd = os.getcwd()
    os.chdir(tmp_path)  # the reference writes projections.raw here
    try:
        rc, vol, mask = O.ref_load_measured("proj.raw", "air.raw", cls, width, views * nskip, nskip, rotations, rate)
    finally:
        os.chdir(cwd)
    orc = _oracle(tmp_path, case)
    assert rc == orc[0]
    assert np.array_equal(vol.view(np.uint32), orc[1].view(np.uint32)) and np.array_equal(mask, orc[2])


def test_loader_stop_and_missing_files(tmp_path):
    write_measured(tmp_path, MEAS_STOP)
    rc, _, _, mx = _oracle(tmp_path, MEAS_STOP)
    assert rc == -2
    assert "Maximum projection: %lf > 1.0... STOP" % mx == str(golden("measured.npz")["stop_line"])
    cls, width, views, nskip, rotations, rate = MEAS_STOP[:6]
    assert O.load_measured(tmp_path / "nothing.raw", tmp_path / "air.raw", True, width, views, nskip, rotations,
                           rate)[0] == -1
    assert O.load_measured(tmp_path / "proj.raw", tmp_path / "nothing.raw", True, width, views, nskip, rotations,
                           rate)[0] == -1
    # PR at the full 609 channels: the reference would read past its raw row
    assert O.load_measured(tmp_path / "proj.raw", tmp_path / "air.raw", False, 609, 800, 1, 1, 80.0)[0] == -3


def _helical_np(vol):
    """MB/main.cpp:347-371, written out in numpy float64."""
    R, V, W = vol.shape
    out = np.zeros((V, W), np.float32)
    use = V // 2 * 2
    for j in range(use):
        iphase = 1 if j < use // 2 else (-1 if j > use // 2 else 0)
        if j + iphase * V < V:
            iphase = 0
        if j + iphase * V > (R - 1) * V:
            iphase = 0
        zw = 0.5 * abs(j - V / 2.0) / (V / 2.0)
        a = vol.reshape(R * V, W)
        out[j] = ((1.0 - zw) * a[j].astype(np.float64) + zw * a[j + iphase * V].astype(np.float64)).astype(np.float32)
    return out


@pytest.mark.parametrize("R,V", [(1, 10), (2, 10), (3, 10), (3, 7), (4, 1)])
def test_helical_restatement(R, V):
    vol = np.random.default_rng(R * 100 + V).uniform(0, 1, (R, V, 5)).astype(np.float32)
    out = O.helical(vol)
    assert np.array_equal(out.view(np.uint32), _helical_np(vol).view(np.uint32))
    if R >= 3 and V == 10:
        assert not np.array_equal(out[:5], vol[0, :5])  # the first half blends with the next rotation


def test_measured_chain_matches_reference_program(tmp_path):
    """Loader -> helical interpolation -> lengthproj_TOMO, all in the oracle,
    equals the reference program's npf_float.raw on the same files."""
    write_e2e_inputs(tmp_path)
    cls, width, views, nskip, rotations, rate = MEAS_E2E[:6]
    rc, vol, mask, mx = _oracle(tmp_path, MEAS_E2E)
    e = golden("measured_e2e.npz")
    assert rc == rotations
    assert np.array_equal(_sha(vol), e["projections_sha"])
    assert "Maximum projection: %lf" % mx == str(e["max_line"])
    proj = O.helical(vol)
    N = MEAS_E2E_N
    g = O.geom(views=views, recon_size=N, pixel_cm=MEAS_E2E_PIX)
    c, s = O.trig_tables(views)
    npf = O.lengthproj(g, c, s, proj[: views // 2 * 2], z=0.4, couch_speed=0.8)
    assert np.array_equal(npf.view(np.uint32), e["npf"].view(np.uint32))
    assert np.count_nonzero(npf) > 1000
