"""The oracle's reference walk against closed-form chords on the CPU (the
same cases as tests/test_gpu_analytic.py): a uniform square inside an empty
ring and a single-pixel impulse give the rays' chords to FP64 rounding,
except the rays through the grid origin, where the reference's sign test
divides 0 by 0."""
import numpy as np
import pytest

import oracle as O
from test_gpu_analytic import CASES, _chord, _origin_rays, _rays


@pytest.mark.parametrize("N,pix,views,channels", CASES)
def test_oracle_walk_gives_chords(N, pix, views, channels):
    g = O.geom(views=views, channels=channels, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(views)
    nxm = N // 2
    sx, sy, px, py = _rays(views // 2 * 2, channels)
    ring = max(12, int(np.ceil(1.2 / pix)) + 2)
    col, row = N // 2 + 3, N // 2 - 5
    for lo_c, hi_c, lo_r, hi_r, scale in ((ring, N - ring, ring, N - ring, None), (col, col + 1, row, row + 1, pix)):
        rho = np.zeros((1, N, N))
        rho[0, lo_r:hi_r, lo_c:hi_c] = 1.0
        L = O.walk_project(g, c, s, rho)[: views // 2 * 2, :channels, 0]
        ref = _chord(sx, sy, px, py, (lo_c - nxm) * pix, (hi_c - nxm) * pix, (nxm - hi_r) * pix, (nxm - lo_r) * pix)
        org = _origin_rays(channels, ref.shape)
        assert np.abs(L - ref)[~org].max() <= 1e-12 * (scale or ref.max())
        if org.any() and scale is None:  # the 0/0 rays cross the square and differ
            assert np.abs(L - ref)[org].max() > 1e-3 * ref.max()
