"""lengthproj_TOMO: the oracle's restatement against the reference's own
function (fixtures made by it, tests/golden/make_golden.py), bit for bit,
including the 512^2 x 800-view case and the pixel column whose source-to-
pixel line has a 0/0 slope (the reference adds nothing there)."""
import numpy as np
import pytest

import oracle as O
from conftest import golden, have_reference_sources
from golden_cases import LP_C1, LP_C1_STEP, LP_CASES, lp_proj


@pytest.mark.parametrize("k", range(len(LP_CASES)))
def test_oracle_lengthproj_matches_reference_fixture(k):
    N, V, pix, z, cs, seed = LP_CASES[k]
    g = O.geom(views=V, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    npf = O.lengthproj(g, c, s, lp_proj(V, seed), z, cs)
    assert np.array_equal(npf, golden("lengthproj.npz")[f"npf_{k}"])


def test_oracle_lengthproj_c1_rows():
    N, V, pix, z, cs, seed = LP_C1
    g = O.geom(views=V, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    npf = O.lengthproj(g, c, s, lp_proj(V, seed), z, cs)
    assert np.array_equal(npf[::LP_C1_STEP], golden("lengthproj.npz")["c1_npf_rows"])


@pytest.mark.skipif(not (have_reference_sources() and O.ref_available()), reason="reference harness not built")
def test_oracle_lengthproj_matches_live_reference():
    N, V, pix, z, cs = 96, 60, 0.2, 4.1, 1.1
    g = O.geom(views=V, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    proj = lp_proj(V, 9)
    ref, _ = O.ref_lengthproj(N, pix, proj, V, c, s, z, cs)
    assert np.array_equal(O.lengthproj(g, c, s, proj, z, cs), ref)
