"""Input cases of the lengthproj fixture (tests/golden/make_golden.py): the
tests regenerate the seeded sinograms instead of storing them."""
import numpy as np

# (N, views, pixel cm, z cm, couch cm/rotation, seed); the first view lies
# inside the trig tables in every case.
LP_CASES = [(64, 40, 0.1, 1.0, 0.8, 1), (63, 36, 0.4, 2.0, 1.2, 2), (128, 80, 0.1, 0.5, 0.4, 3),
            (33, 44, 0.5, 7.3, 0.9, 4)]
LP_C1 = (512, 800, 0.1, 3.0, 0.8, 5)
LP_C1_STEP = 16


def lp_proj(views, seed, width=609):
    return np.random.default_rng(seed).uniform(0.1, 1.0, (views // 2 * 2, width)).astype(np.float32)


# Beam-hardening correction: a seeded 800 x 609 transmission sinogram, the
# (alpha, beta) pairs of the reference program's usage line (kV, MV), and
# the rows the fixture keeps.
BH_PARAMS = [(0.01, 2.00), (0.01, 3.70)]
BH_ROW_STEP = 32


def bh_sino(seed=1):
    return np.random.default_rng(seed).uniform(1e-3, 1.0, (800, 609)).astype(np.float32)
