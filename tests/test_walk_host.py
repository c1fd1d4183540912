"""The device ray walks, compiled for the CPU from the same source
(virtualct_b200/csrc/vct_forward.cu), against each other and the oracle: the
fast walk must find the exact walk's segments and line integrals."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden
from virtualct_b200 import phantoms


@pytest.fixture(scope="module")
def walk_check(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path_factory.mktemp("walk") / "walk_check"
    src = os.path.join(ROOT, "tests", "host", "walk_check.cu")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Xcompiler", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "virtualct_b200", "csrc"), src, "-o",
                    str(exe)], check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("N,pix,views,seed,channels", [(128, 0.1, 200, 3, 609), (64, 0.4, 40, 7, 609),
                                                        (96, 0.25, 61, 5, 609), (256, 0.1, 90, 11, 512),
                                                        (160, 0.1, 60, 2, 800)])
def test_fast_walk_matches_exact_walk(walk_check, tmp_path, N, pix, views, seed, channels):
    """Includes even channel counts, whose central ray passes through the origin."""
    maps = phantoms.ellipse_phantom(seed, N, border_px=2)
    mp = tmp_path / "maps.raw"
    maps.tofile(mp)
    out = tmp_path / "L.bin"
    r = subprocess.run([str(walk_check), str(mp), str(N), str(pix), str(views), str(channels), str(out)],
                       check=True, capture_output=True, text=True)
    miss, fallback, nse, nsf = map(int, r.stdout.split())
    L = np.fromfile(out, np.float64)
    n = L.size // 2
    Le, Lf = L[:n].reshape(views, channels, 6), L[n:].reshape(views, channels, 6)
    # The fast walk also visits the (zero-weight) poke-out cells past the
    # grid and closes coincident events with empty segments.
    assert nse <= nsf <= nse + 6 * views * channels
    assert np.max(np.abs(Lf - Le)) < 1e-8
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(views)
    t = golden("mu_tables.npz")
    _, lint = O.forward_fp64_maps(g, c, s, maps, t["kramers120_mu"], t["kramers120_pdf"], want_lint=True)
    assert np.max(np.abs(Le - lint)) < 1e-11 * max(1.0, lint.max())
    if pix == 0.1:
        # every first step is a pixel boundary at 0.1 cm; only rays through
        # the origin (even channel counts) take the exact walk
        assert fallback <= (0 if channels % 2 else views)


@pytest.fixture(scope="module")
def acc_check(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = tmp_path_factory.mktemp("acc") / "acc_check"
    src = os.path.join(ROOT, "tests", "host", "acc_check.cu")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "virtualct_b200", "csrc"), src, "-o", str(exe)],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("M", [1, 2, 3, 4, 5, 6, 7, 8])
def test_paired_word_accumulation_is_exact(acc_check, M):
    """Two elements per 64-bit multiply-add, the low sum recovered modulo 2^64:
    equal to the per-element sums at the extremes (65535 densities, 2^31
    weights, 20,000 segments, so the packed sums wrap many times)."""
    r = subprocess.run([str(acc_check), str(M), "20000", str(M + 100)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
