"""Seeded synthetic inputs: deterministic, in range, readable by the oracle's
restatement of the reference's spectrum parser."""
import numpy as np

import oracle as O
from virtualct_b200 import phantoms


def test_ellipse_phantom_deterministic_and_bounded():
    a = phantoms.ellipse_phantom(3, 128)
    b = phantoms.ellipse_phantom(3, 128)
    c = phantoms.ellipse_phantom(4, 128)
    assert a.dtype == np.int16 and a.shape == (6, 128, 128)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    dens = a.astype(np.float64).sum(0) / 1000
    assert dens.max() <= 1.9 + 1e-9 and dens[dens > 0].min() >= 0.29
    assert not a[:, :8].any() and not a[:, :, -8:].any()  # empty border ring


def test_gammex_phantom_eight_elements():
    m = phantoms.gammex_cylinder_phantom(1, 512)
    assert m.shape == (8, 512, 512)
    dens = m.astype(np.float64).sum(0) / 1000
    assert abs(dens[256, 256] - 1.018) < 0.01 or dens[256, 256] > 0.25
    assert dens[0, 0] == 0


def test_spectrum_txt_round_trip(tmp_path):
    rows = phantoms.kramers_spectrum(80)
    p = tmp_path / "s.txt"
    phantoms.write_spectrum_txt(p, rows)
    pdf, e = O.spectrum(str(p))
    assert len(pdf) == 70
    assert abs(float(pdf.sum()) - 1.0) < 1e-5
    assert np.allclose(e, 0.5 * (rows[:, 0] + rows[:, 1]), rtol=1e-6)
    rows6 = phantoms.mv_spectrum()
    assert rows6.shape == (60, 3) and np.all(rows6[:, 2] >= 0)
