"""Measured-data ingestion and the helical z-interpolation on the GPU,
through the C ABI: vct_load_measured against the oracle's loader (itself
pinned to the reference's loadProjectionData) bit for bit on every seeded
case, its error paths, vct_helical_sinogram(_dev) against the oracle, and the
vct_mbfpa drop-in on measured data against the reference's own MBFPA
program (tests/golden/measured_e2e.npz)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import SINO_RTOL, golden, max_rel
from golden_cases import (MEAS_CASES, MEAS_E2E, MEAS_E2E_N, MEAS_STOP, write_e2e_inputs, write_measured,
                          write_measured_txt)

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "virtualct_b200", "bin")


def _cfg(d, case):
    write_measured(d, case)
    write_measured_txt(d, case)
    cwd = os.getcwd()
    os.chdir(d)  # the txt names the files relative to its directory
    try:
        return vct.MbConfig.load("mb.txt")
    finally:
        os.chdir(cwd)


def _load(d, cfg):
    cwd = os.getcwd()
    os.chdir(d)
    try:
        return vct.load_measured(cfg)
    finally:
        os.chdir(cwd)


def _same(a, b):
    """Bit-identical floats; NaN at the same places (CUDA and x86 write
    different NaN payloads)."""
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


@pytest.mark.parametrize("name", sorted(MEAS_CASES))
def test_loader_matches_oracle(cuda_device, name, tmp_path):
    case = MEAS_CASES[name]
    cfg = _cfg(tmp_path, case)
    vol, mask, rot, mx = _load(tmp_path, cfg)
    cls, width, views, nskip, rotations, rate = case[:6]
    rc, ovol, omask, omx = O.load_measured(tmp_path / "proj.raw", tmp_path / "air.raw", cls == "IN", width, views,
                                           nskip, rotations, rate)
    assert rot == rc == rotations and vol.shape == ovol.shape
    assert _same(vol, ovol) and np.array_equal(mask, omask)
    assert mx == omx


def test_loader_errors(cuda_device, tmp_path):
    cfg = _cfg(tmp_path, MEAS_STOP)
    with pytest.raises(vct.VctError) as e:
        _load(tmp_path, cfg)
    assert e.value.code == vct.VCT_E_RANGE
    assert str(golden("measured.npz")["stop_line"]) in str(e.value)
    missing = vct.MbConfig.load(tmp_path / "mb.txt")
    missing.proj_file = str(tmp_path / "nothing.raw").encode()
    with pytest.raises(vct.VctError) as e:
        vct.load_measured(missing)
    assert e.value.code == vct.VCT_E_IO and "nothing.raw not found" in str(e.value)
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        pr609 = vct.MbConfig.load("mb.txt")
    finally:
        os.chdir(cwd)
    pr609.proj_file = str(tmp_path / "proj.raw").encode()
    pr609.air_scan_file = str(tmp_path / "air.raw").encode()
    pr609.in_pr_class = b"PR"
    pr609.proj_width = 609
    with pytest.raises(vct.VctError) as e:  # 27 skipped + 609 used channels > a 609-channel raw row
        vct.load_measured(pr609)
    assert e.value.code == vct.VCT_E_UNSUPPORTED


@pytest.mark.parametrize("R,V,W", [(1, 10, 5), (2, 10, 7), (3, 400, 609), (3, 7, 3), (5, 800, 609)])
def test_helical_matches_oracle(cuda_device, R, V, W):
    import torch

    vol = np.random.default_rng(R * 1000 + V).uniform(0, 1, (R, V, W)).astype(np.float32)
    ref = O.helical(vol)
    out = vct.helical_sinogram(vol)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))
    d_out = torch.full((V, W), 7.0, dtype=torch.float32, device="cuda")
    vct.helical_sinogram_dev(torch.from_numpy(vol).cuda(), d_out)
    torch.cuda.synchronize()
    dev = d_out.cpu().numpy()
    use = V // 2 * 2
    assert np.array_equal(dev[:use].view(np.uint32), ref[:use].view(np.uint32))
    assert (dev[use:] == 7.0).all()  # rows past views/2*2 are left alone


def test_dropin_on_measured_data_matches_reference_program(cuda_device, tmp_path):
    write_e2e_inputs(tmp_path)
    r = subprocess.run([os.path.join(BIN, "vct_mbfpa"), "mb.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    e = golden("measured_e2e.npz")
    N = MEAS_E2E_N
    assert str(e["max_line"]) in r.stderr
    proj = np.fromfile(tmp_path / "projections.raw", np.float32)
    assert np.array_equal(np.frombuffer(hashlib.sha256(proj.tobytes()).digest(), np.uint8), e["projections_sha"])
    npf = np.fromfile(tmp_path / "npf_float.raw", np.float32).reshape(N, N)
    assert np.array_equal(npf.view(np.uint32), e["npf"].view(np.uint32))
    assert np.count_nonzero(npf) > 1000
    # the iterative step reads one energy bin of this build's forward
    # projection (within 1e-5 of the reference's), so its image agrees to
    # that order, not bit for bit
    ite1 = np.fromfile(tmp_path / "ReconImageRaw" / "Reconstruction_ite0001_z0000.raw", np.float32).reshape(N, N)
    assert np.abs(ite1 - e["ite1"]).max() <= 1e-5 * np.abs(e["ite1"]).max()
    assert not np.array_equal(ite1, np.fromfile(tmp_path / "Weight_input_ICRU110.raw", np.int16)[:N * N]
                              .reshape(N, N).astype(np.float32) / 1000)  # the measured data moved the image
    s16 = np.fromfile(tmp_path / "ReconImageRaw" / "Reconstruction_512x512x1.raw", np.int16)
    assert np.abs(s16.astype(np.int32) - e["recon16"].astype(np.int32)).max() <= 1
    views = MEAS_E2E[2]
    sino = np.fromfile(tmp_path / "reprojection_float.raw", np.float32).reshape(views, 609)
    assert max_rel(sino[::10], e["reprojection_rows"]) < SINO_RTOL
