"""Beam-hardening correction: the oracle's restatement against the
reference program's own output (tests/golden/beam_hardening.npz), bit for
bit, including the minima it prints."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import golden, have_reference_sources
from golden_cases import BH_PARAMS, BH_ROW_STEP, bh_sino


@pytest.mark.parametrize("k", range(len(BH_PARAMS)))
def test_oracle_matches_reference_fixture(k):
    a, b = BH_PARAMS[k]
    cor, mins = O.beam_hardening(bh_sino(), a, b)
    d = golden("beam_hardening.npz")
    assert np.array_equal(cor[::BH_ROW_STEP], d[f"rows_{k}"])
    assert "%lf %lf" % mins == str(d[f"line_{k}"])


@pytest.mark.skipif(not (have_reference_sources() and os.path.exists(os.path.join(os.path.dirname(O.__file__), "_ref", "bhc"))),
                    reason="reference not built")
def test_oracle_matches_live_reference():
    p = np.random.default_rng(4).uniform(1e-4, 1.0, (800, 609)).astype(np.float32)
    ref, line = O.ref_beam_hardening(p, 0.03, 2.5)
    cor, mins = O.beam_hardening(p, 0.03, 2.5)
    assert np.array_equal(cor, ref) and "%lf %lf" % mins == line
