"""lengthproj_TOMO on the GPU, through the C ABI, against the reference's own
outputs (tests/golden/lengthproj.npz): helical cases and the 512^2 x 800-view
case, npf within 1e-5 relative per pixel (every term is positive); and
against the oracle with a couch that does not move (views from 0)."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import golden
from golden_cases import LP_C1, LP_C1_STEP, LP_CASES, lp_proj

pytestmark = pytest.mark.gpu

NPF_RTOL = 1e-5


def _rel(a, ref):
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    inside = ref != 0
    assert np.array_equal(a != 0, inside)
    return float(np.max(np.abs(a[inside] - ref[inside]) / np.abs(ref[inside])))


@pytest.mark.parametrize("k", range(len(LP_CASES)))
def test_lengthproj_matches_reference(cuda_device, k):
    N, V, pix, z, cs, seed = LP_CASES[k]
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=pix)) as ctx:
        npf = ctx.lengthproj(lp_proj(V, seed), z, cs)
    assert _rel(npf, golden("lengthproj.npz")[f"npf_{k}"]) < NPF_RTOL


def test_lengthproj_c1_matches_reference(cuda_device):
    N, V, pix, z, cs, seed = LP_C1
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=pix)) as ctx:
        npf = ctx.lengthproj(lp_proj(V, seed), z, cs)
    assert _rel(npf[::LP_C1_STEP], golden("lengthproj.npz")["c1_npf_rows"]) < NPF_RTOL


def test_lengthproj_static_couch_vs_oracle(cuda_device):
    N, V, pix = 96, 60, 0.2
    g = O.geom(views=V, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    proj = lp_proj(V, 11)
    ref = O.lengthproj(g, c, s, proj, 0.0, 0.0)
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=pix)) as ctx:
        npf = ctx.lengthproj(proj, 0.0, 0.0)
    assert _rel(npf, ref) < NPF_RTOL
