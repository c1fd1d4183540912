"""Normalisation + Philox noise (gaussiannoise0, MB/main.cpp:51-76): checked by
per-channel mean and variance, clamps and determinism, not sample by sample."""
import numpy as np
import pytest

import virtualct_b200 as vct
from conftest import golden

pytestmark = pytest.mark.gpu


def _run(sigma, seed, views=800):
    t = golden("mu_tables.npz")
    from virtualct_b200 import phantoms

    maps = phantoms.ellipse_phantom(5, 128)
    with vct.Context(vct.Geometry(views=views, recon_size=128, pixel_cm=0.4)) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        clean = ctx.mbfpa(0.0, seed)
        noisy, st = ctx.mbfpa(sigma, seed, return_stats=True)
    return clean, noisy, st


def test_noise_statistics(cuda_device):
    sigma = 2e-3
    clean, noisy, st = _run(sigma, 1234)
    assert clean.max() == 1.0
    ok = (clean > 10 * sigma) & (clean < 1 - 10 * sigma)  # away from both clamps
    d = noisy.astype(np.float64) - clean
    cols = np.flatnonzero(ok.sum(0) >= 150)
    assert len(cols) > 50
    for c in cols:
        x = d[ok[:, c], c]
        n = len(x)
        # per channel over views: mean ~ N(0, sigma^2/n), var ~ sigma^2 (1 +- sqrt(2/(n-1)))
        assert abs(x.mean()) < 6 * sigma / np.sqrt(n)
        assert abs(x.var(ddof=1) / sigma**2 - 1) < 6 * np.sqrt(2 / (n - 1))
    x = d[ok]
    assert abs(x.mean()) < 6 * sigma / np.sqrt(x.size)
    assert abs(x.var() / sigma**2 - 1) < 6 * np.sqrt(2 / (x.size - 1))


def test_noise_clamps_and_determinism(cuda_device):
    sigma = 0.05
    clean, noisy, st = _run(sigma, 7)
    assert noisy.max() <= 1.0
    pmin = float(st[1])
    assert abs(pmin - clean.min()) <= 1e-7 * max(pmin, 1e-30)
    assert noisy.min() >= 0.0
    # p + noise < 0 -> projection_min/10: with sigma = 0.05 the darkest rays
    # (p < 1e-3) go negative about half the time.
    floor = np.float32(pmin / 10)
    dark = clean < 1e-3
    assert dark.sum() > 100
    frac = float(np.mean(noisy[dark] == floor))
    assert 0.3 < frac < 0.7
    assert np.any(noisy == 1.0)
    _, again, _ = _run(sigma, 7)
    _, other, _ = _run(sigma, 8)
    assert np.array_equal(noisy, again)
    assert not np.array_equal(noisy, other)


def test_noise_at_configured_sigma_c1(cuda_device):
    """The 512^2, 800 x 609 slice at the shipped txt's sigma = 5.37e-5 (field
    31 of IR_TOMO_input_virtual_projection_120kV.txt), four seeds: per-channel
    mean and variance of the unclamped residuals, and how often each clamp of
    gaussiannoise0 (MB/main.cpp:51-76) fires against its probability from the
    noise-free values, Phi(-p/sigma) for p + noise < 0 (-> projection_min/10)
    and Phi((p-1)/sigma) for p + noise > 1 (-> 1)."""
    import math

    from virtualct_b200 import phantoms

    sigma = 0.0000537
    t = golden("mu_tables.npz")
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(phantoms.ellipse_phantom(0, 512))
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        clean, st0 = ctx.mbfpa(0.0, 1, return_stats=True)
        runs = [ctx.mbfpa(sigma, seed, return_stats=True) for seed in (11, 12, 13, 14)]
    clean = clean.astype(np.float64)
    floor = np.float32(float(st0[1]) / 10.0)
    assert clean.min() < sigma  # the darkest rays reach the lower clamp
    phi = np.vectorize(lambda x: 0.5 * math.erfc(-x / math.sqrt(2)))
    e_lo = float(phi(-clean / sigma).sum())
    e_hi = float(phi((clean - 1.0) / sigma).sum())
    assert e_lo > 20 and e_hi > 1000
    res = []
    for noisy, st in runs:
        assert abs(float(st[1]) - float(st0[1])) <= 1e-7 * float(st0[1])  # same projection_min
        lo = noisy == floor
        hi = noisy == np.float32(1.0)
        assert abs(lo.sum() - e_lo) < 6 * math.sqrt(e_lo) + 3, (lo.sum(), e_lo)
        assert abs(hi.sum() - e_hi) < 6 * math.sqrt(e_hi) + 3, (hi.sum(), e_hi)
        d = noisy.astype(np.float64) - clean
        d[lo | hi] = np.nan
        res.append(d)
    d = np.concatenate(res, axis=0)  # [4*800][609]
    # per channel, the views whose noise-free value is away from both clamps
    away = np.tile((clean > 8 * sigma) & (clean < 1 - 8 * sigma), (len(runs), 1))
    assert np.isfinite(d[away]).all()
    cols = np.flatnonzero(away.sum(axis=0) >= 2000)
    assert len(cols) > 200
    for c in cols:
        x = d[away[:, c], c]
        n = x.size
        assert abs(x.mean()) < 6 * sigma / math.sqrt(n)
        assert abs(x.var(ddof=1) / sigma**2 - 1) < 6 * math.sqrt(2 / (n - 1))
    x = d[away]
    assert abs(x.mean()) < 6 * sigma / math.sqrt(x.size)
    assert abs(x.var() / sigma**2 - 1) < 6 * math.sqrt(2 / (x.size - 1))
