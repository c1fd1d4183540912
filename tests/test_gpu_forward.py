"""MBFPA forward projection on the GPU against the reference (fixtures made by
the reference's own code) and against the oracle, through the C ABI."""
import os

import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import GOLDEN, SINO_RTOL, fbp_errors, golden, max_rel
from virtualct_b200 import phantoms

pytestmark = pytest.mark.gpu


def _ctx(views, N, pixel, **kw):
    return vct.Context(vct.Geometry(views=views, recon_size=N, pixel_cm=pixel, **kw))


# Error of the device path against the FP64 oracle (same walk, FP64 sums,
# densities s/1000): the SFU exponential of the compensated summation and the
# final float rounding.
FP64_RTOL = 1e-6


@pytest.mark.parametrize("views", [40, 41])
@pytest.mark.parametrize("mode", [vct.SUM_COMPENSATED, vct.SUM_REFERENCE])
@pytest.mark.parametrize("walk", [vct.WALK_FAST, vct.WALK_EXACT])
def test_small_forward_matches_reference(cuda_device, views, mode, walk):
    d = golden("mb_small.npz")
    t = golden("mu_tables.npz")
    ref = d[f"full_v{views}"]
    with _ctx(views, int(d["N"]), float(d["pixel_cm"])) as ctx:
        ctx.set_sum_mode(mode)
        ctx.set_walk_mode(walk)
        ctx.set_maps(d["maps"])
        ctx.set_spectrum(t["kv120_mu"], t["kv120_pdf"])
        out = ctx.forward()
    used = views // 2 * 2
    assert max_rel(out[:used], ref[:used]) < SINO_RTOL
    assert not out[used:].any()  # rows past views/2*2 stay 0, as in the reference


@pytest.mark.parametrize("mode", [vct.SUM_COMPENSATED, vct.SUM_REFERENCE])
def test_even_channels_exact_rays_by_warp(cuda_device, mode):
    """At an even channel count the central channel of every view passes
    through the grid origin and takes the exact walk; with the fast walk those
    rays are listed once and each is walked by a whole warp after the rest.
    The sinogram and line integrals against the FP64 oracle, and those rays'
    line integrals against the exact walk in one thread per ray (the same
    segments, summed in another order)."""
    import torch

    N, pix, views, C = 128, 0.1, 120, 512
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(13, N, border_px=2)
    g = O.geom(views=views, channels=C, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(views)
    f64, lint = O.forward_fp64_maps(g, c, s, maps, t["kv120_mu"], t["kv120_pdf"], want_lint=True)
    geo = vct.Geometry.with_channels(C, views=views, recon_size=N, pixel_cm=pix)
    res = {}
    for walk in (vct.WALK_FAST, vct.WALK_EXACT):
        with vct.Context(geo) as ctx:
            ctx.set_sum_mode(mode)
            ctx.set_walk_mode(walk)
            ctx.set_maps(maps)
            ctx.set_spectrum(t["kv120_mu"], t["kv120_pdf"])
            out = ctx.forward()
            L = torch.zeros((views, C, 6), dtype=torch.float64, device="cuda")
            ctx.line_integrals_dev(L)
            ctx.synchronize()
            res[walk] = (out, L.cpu().numpy())
    out_f, L_f = res[vct.WALK_FAST]
    _, L_e = res[vct.WALK_EXACT]
    scale = max(1.0, np.abs(lint).max())
    central = C // 2
    assert np.abs(L_e[:, central]).max() > 0
    assert np.max(np.abs(L_f[:, central] - L_e[:, central])) <= 1e-12 * scale
    assert np.max(np.abs(L_f - lint)) <= 1e-8 * scale
    assert max_rel(out_f, f64) < (FP64_RTOL if mode == vct.SUM_COMPENSATED else SINO_RTOL)


@pytest.mark.parametrize("walk", [vct.WALK_FAST, vct.WALK_EXACT])
@pytest.mark.parametrize("N,pix,views", [(64, 0.4, 40), (128, 0.1, 120)])
def test_line_integrals_vs_fp64_oracle(cuda_device, walk, N, pix, views):
    import torch

    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(9, N, border_px=2)
    g = O.geom(views=views, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(views)
    f64, lint = O.forward_fp64_maps(g, c, s, maps, t["kv120_mu"], t["kv120_pdf"], want_lint=True)
    with _ctx(views, N, pix) as ctx:
        ctx.set_walk_mode(walk)
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kv120_mu"], t["kv120_pdf"])
        out = ctx.forward()
        L = torch.zeros((views, 609, 6), dtype=torch.float64, device="cuda")
        ctx.line_integrals_dev(L)
        ctx.synchronize()
        L = L.cpu().numpy()
    # Exact walk: the reference's segments, FMA accumulation only.  Fast
    # walk: split fractions in 30-bit fixed point.
    tol = 1e-11 if walk == vct.WALK_EXACT else 1e-8
    assert np.max(np.abs(L - lint)) <= tol * max(1.0, np.abs(lint).max())
    assert max_rel(out, f64) < FP64_RTOL


@pytest.mark.parametrize("walk", [vct.WALK_FAST, vct.WALK_EXACT])
def test_c1_full_size_matches_reference(cuda_device, walk):
    """512^2, 800 x 609, 6 elements, 110-bin 120 kVp Kramers spectrum."""
    d = golden("c1_subset.npz")
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(int(d["seed"]), 512)
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_walk_mode(walk)
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        out = ctx.forward()
        segs = ctx.last_segment_count
        norm, stats = ctx.mbfpa(0.0, 1, return_stats=True)
    rows = d["rows"]
    assert max_rel(out[rows], d["full_rows"]) < SINO_RTOL
    if walk == vct.WALK_EXACT:
        assert segs == int(d["segments"])  # the reference's walk: same segment set
    else:  # plus zero-weight poke-out / coincident-event pieces
        assert int(d["segments"]) <= segs <= int(d["segments"]) + 6 * 800 * 609
    assert abs(float(stats[0]) / float(d["max"]) - 1) < SINO_RTOL
    assert abs(float(out.max()) / float(d["max"]) - 1) < SINO_RTOL
    ref_norm = d["full_rows"] / d["max"]
    assert max_rel(norm[rows], ref_norm) < 2 * SINO_RTOL


def test_c1_fbp_and_fp64_rows(cuda_device):
    """The 512^2, 800 x 609, 6-element slice end to end: the device forward within 1e-5 of the FP64 sum, and the
    Ram-Lak FBP of its max-normalised, noise-free sinogram within 1e-4 of the
    reference's FBP of the reference's sinogram (every 16th row)."""
    d = golden("c1_subset.npz")
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(int(d["seed"]), 512)
    with vct.Context(vct.Geometry()) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        out = ctx.forward()
        norm = ctx.mbfpa(0.0, 1)
        img = ctx.fbp(norm, filter=1)
    assert max_rel(out[d["rows"]], d["fp64_rows"]) < SINO_RTOL
    step = 512 // d["fbp_ramlak_rows"].shape[0]
    mx, l2 = fbp_errors(img[::step], d["fbp_ramlak_rows"])
    assert mx < 1e-4 and l2 < 1e-4, (mx, l2)


def test_eight_elements_and_6mv(cuda_device):
    """6 MV style: 8 elements (Mg, Si added), MV spectrum; against the FP64 oracle."""
    rows = phantoms.mv_spectrum()
    import tempfile

    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "mv.txt")
        phantoms.write_spectrum_txt(p, rows)
        mu, pdf = vct.attenuation_coefficient(p, vct.GAMMEX_ELEMENTS)
    maps = phantoms.gammex_cylinder_phantom(2, 128, pixel_cm=0.4)
    g = O.geom(views=60, recon_size=128, pixel_cm=0.4)
    c, s = O.trig_tables(60)
    f64 = O.forward_fp64_maps(g, c, s, maps, mu, pdf)
    ex = O.forward_exact(g, c, s, O.rho_from_maps(maps), mu, pdf)
    with _ctx(60, 128, 0.4) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(mu, pdf)
        out = ctx.forward()
    assert max_rel(out, ex) < SINO_RTOL
    assert max_rel(out, f64) < FP64_RTOL


@pytest.mark.parametrize("channels,views,N", [(512, 360, 256), (800, 900, 384)])
def test_runtime_geometry(cuda_device, channels, views, N):
    """Channel and view counts as runtime fields (iso = C/2, dalpha = Max_alpha/((C-1)/2))."""
    t = golden("mu_tables.npz")
    maps = phantoms.ellipse_phantom(11, N)
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=0.1)
    c, s = O.trig_tables(views)
    f64 = O.forward_fp64_maps(g, c, s, maps, t["kramers120_mu"], t["kramers120_pdf"])
    with vct.Context(vct.Geometry.with_channels(channels, views=views, recon_size=N)) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(t["kramers120_mu"], t["kramers120_pdf"])
        out = ctx.forward()
    assert max_rel(out, f64) < FP64_RTOL


def test_negative_densities_contribute_nothing(cuda_device):
    d = golden("mb_small.npz")
    t = golden("mu_tables.npz")
    maps = d["maps"].copy()
    neg = maps.copy()
    rng = np.random.default_rng(0)
    idx = rng.random(neg.shape) < 0.05
    neg[idx] = -rng.integers(1, 900, idx.sum())
    clipped = np.where(neg < 0, 0, neg).astype(np.int16)
    with _ctx(40, 64, 0.4) as ctx:
        ctx.set_spectrum(t["kv120_mu"], t["kv120_pdf"])
        ctx.set_maps(neg)
        a = ctx.forward()
        ctx.set_maps(clipped)
        b = ctx.forward()
    assert np.array_equal(a, b)


def test_empty_phantom_is_spectrum_sum(cuda_device):
    t = golden("mu_tables.npz")
    with _ctx(40, 64, 0.4) as ctx:
        ctx.set_sum_mode(vct.SUM_REFERENCE)
        ctx.set_maps(np.zeros((6, 64, 64), np.int16))
        ctx.set_spectrum(t["kv120_mu"], t["kv120_pdf"])
        out = ctx.forward()
    s = np.float32(0)
    for p in t["kv120_pdf"]:
        s = np.float32(s + p)
    assert np.all(out == s)


def test_call_order_errors(cuda_device):
    with _ctx(40, 64, 0.4) as ctx:
        with pytest.raises(vct.VctError) as e:
            ctx.forward()
        assert e.value.code == vct.VCT_E_STATE
        with pytest.raises(vct.VctError) as e:
            ctx.set_spectrum(np.zeros((9, 10), np.float32), np.zeros(10, np.float32))
        assert e.value.code == vct.VCT_E_ARG
