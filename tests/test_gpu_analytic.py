"""The forward walk against closed-form answers on the GPU, through the C
ABI (vct_line_integrals_dev), for both walks:

  * a uniform square inside an empty border ring: every ray's line integral is
    its chord through that square (the segments are bounded by grid lines, so
    the reference's midpoint rule assigns each exactly; the ring holds the
    lumped first segments, which reach at most a few pixels in);
  * a single-pixel impulse: every ray's line integral is its chord through
    that pixel.

Ray ends as MB/reprojection_TOMO.cpp:53-74 builds them: the source at
SID (sin b, cos b), channel jj's detector point on the arc of radius 142.6 cm
centred 85 cm beyond the isocentre at angle (iso - jj) * dalpha, rotated by
the view.  Chords are clipped in FP64 (Liang-Barsky)."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct

pytestmark = pytest.mark.gpu

SID, DET_R, DET_SRC_ISO, MAX_ALPHA = 85.0, 142.6, 85.0, 0.326086956


def _rays(views, channels):
    """Source and detector points, [views][channels] each (x, y) in cm."""
    c, s = O.trig_tables(views)
    half = (channels - 1) // 2
    dalpha = MAX_ALPHA / half
    iso = channels / 2.0
    jj = np.arange(channels, dtype=np.float64)
    theta = (iso - jj) * dalpha
    px0 = DET_R * np.sin(theta)
    py0 = -DET_R * np.cos(theta) + DET_SRC_ISO
    cb, sb = c[:, None], s[:, None]
    px = px0[None] * cb + py0[None] * sb
    py = -px0[None] * sb + py0[None] * cb
    sx, sy = SID * sb + 0 * px, SID * cb + 0 * py
    return sx, sy, px, py


def _chord(sx, sy, px, py, x0, x1, y0, y1):
    """Length of the segment source->detector inside [x0,x1] x [y0,y1]."""
    dx, dy = px - sx, py - sy
    t0 = np.zeros_like(dx)
    t1 = np.ones_like(dx)
    for p, q in ((-dx, sx - x0), (dx, x1 - sx), (-dy, sy - y0), (dy, y1 - sy)):
        with np.errstate(divide="ignore", invalid="ignore"):
            r = q / p
        t0 = np.where((p < 0) & (r > t0), r, t0)
        t1 = np.where((p > 0) & (r < t1), r, t1)
        t1 = np.where((p == 0) & (q < 0), -1.0, t1)  # parallel and outside
    return np.maximum(t1 - t0, 0.0) * np.hypot(dx, dy)


def _line_integrals(geo, maps, walk):
    import torch

    with vct.Context(geo) as ctx:
        ctx.set_walk_mode(walk)
        ctx.set_maps(maps)
        ctx.set_spectrum(np.ones((maps.shape[0], 1), np.float32), np.ones(1, np.float32))
        L = torch.zeros((geo.views // 2 * 2, geo.channels, maps.shape[0]), dtype=torch.float64, device="cuda")
        ctx.line_integrals_dev(L)
        ctx.synchronize()
        return L.cpu().numpy()


# (N, pixel cm, views, channels): the 512^2 grid at 0.1 cm; coarser grids; even channel
# counts, whose central ray passes through the origin; view counts whose views
# include 0, 45, 90 ... degrees exactly.  The pixel sizes divide 1 cm: the
# walk steps from the first whole-cm gridline, so for sizes that do not (say
# 0.4 cm) its segment ends are not pixel edges and the midpoint rule moves
# partial pieces between pixels -- the reference's behaviour, checked against
# the oracle elsewhere, not a chord.
CASES = [(512, 0.1, 80, 609), (128, 0.25, 72, 512), (96, 0.5, 120, 610)]


def _origin_rays(channels, shape):
    """Rays through the grid origin (even channel counts, channel C/2): the
    reference's sign test divides 0 by 0 there, and the walk follows it, so
    those rays are held to the oracle's walk instead of the chord."""
    m = np.zeros(shape, bool)
    if channels % 2 == 0:
        m[:, channels // 2] = True
    return m


@pytest.mark.parametrize("walk", [vct.WALK_EXACT, vct.WALK_FAST])
@pytest.mark.parametrize("N,pix,views,channels", CASES)
def test_uniform_square_gives_chords(cuda_device, walk, N, pix, views, channels):
    ring = max(12, int(np.ceil(1.2 / pix)) + 2)  # the lumped first segment reaches < 1 cm past the entry
    maps = np.zeros((1, N, N), np.int16)
    maps[0, ring:N - ring, ring:N - ring] = 1000  # 1 g/cm^3
    geo = vct.Geometry.with_channels(channels, views=views, recon_size=N, pixel_cm=pix)
    L = _line_integrals(geo, maps, walk)[..., 0]
    nxm = N // 2
    x0, x1 = (ring - nxm) * pix, (N - ring - nxm) * pix
    y0, y1 = (nxm - (N - ring)) * pix, (nxm - ring) * pix
    sx, sy, px, py = _rays(views // 2 * 2, channels)
    ref = _chord(sx, sy, px, py, x0, x1, y0, y1)
    tol = (1e-10 if walk == vct.WALK_EXACT else 1e-7) * ref.max()
    org = _origin_rays(channels, ref.shape)
    assert np.abs(L - ref)[~org].max() <= tol, np.abs(L - ref)[~org].max() / ref.max()
    assert (ref > 0).sum() > 0.3 * ref.size
    if org.any():
        g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=pix)
        c, s = O.trig_tables(views)
        ow = O.walk_project(g, c, s, maps.astype(np.float64) / 1000.0)[: views // 2 * 2, :channels, 0]
        assert np.abs(L - ow)[org].max() <= tol


@pytest.mark.parametrize("walk", [vct.WALK_EXACT, vct.WALK_FAST])
@pytest.mark.parametrize("N,pix,views,channels", CASES)
def test_single_pixel_impulse_gives_its_chords(cuda_device, walk, N, pix, views, channels):
    col, row = N // 2 + 3, N // 2 - 5
    maps = np.zeros((1, N, N), np.int16)
    maps[0, row, col] = 1000
    geo = vct.Geometry.with_channels(channels, views=views, recon_size=N, pixel_cm=pix)
    L = _line_integrals(geo, maps, walk)[..., 0]
    nxm = N // 2
    x0, x1 = (col - nxm) * pix, (col - nxm + 1) * pix
    y0, y1 = (nxm - row - 1) * pix, (nxm - row) * pix
    sx, sy, px, py = _rays(views // 2 * 2, channels)
    ref = _chord(sx, sy, px, py, x0, x1, y0, y1)
    tol = (1e-10 if walk == vct.WALK_EXACT else 1e-7) * pix
    org = _origin_rays(channels, ref.shape)
    assert np.abs(L - ref)[~org].max() <= tol, np.abs(L - ref)[~org].max() / pix
    hit = (ref > 0) & ~org
    assert hit.sum() >= views // 2 * 2  # every view has rays through the pixel
    assert np.abs(L[hit].sum() - ref[hit].sum()) <= 1e-6 * ref[hit].sum()
