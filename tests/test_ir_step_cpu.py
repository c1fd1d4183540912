"""The reference's iterative step: the oracle's lengthproj_TOMO_2 and
IR_ImageTOMO against the reference's own functions (fixtures made by them,
tests/golden/ir_step.npz), bit for bit."""
import numpy as np
import pytest

import oracle as O
from conftest import golden
from golden_cases import IR_CASES, LP2_CASES, ir_inputs, lp2_inputs


@pytest.mark.parametrize("k", range(len(LP2_CASES)))
def test_lengthproj2_matches_reference(k):
    N, V, pix, z, cs, ite, th, seed = LP2_CASES[k]
    g = O.geom(views=V, recon_size=N, pixel_cm=pix)
    c, s = O.trig_tables(V)
    _, p = lp2_inputs(V, seed)
    assert np.array_equal(O.lengthproj2(g, c, s, p, ite, th, z, cs), golden("ir_step.npz")[f"lp2_{k}"])


@pytest.mark.parametrize("k", range(len(IR_CASES)))
def test_ir_update_matches_reference(k):
    N, ite, th, wb, wtv, wpr, seed = IR_CASES[k]
    before, npf, npf_re, prior, after = ir_inputs(N, seed)
    out = O.ir_update(before, npf, npf_re, wb, wtv, wpr, ite, th, prior, after)
    assert np.array_equal(out, golden("ir_step.npz")[f"ir_{k}"])
