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


# The iterative step: lengthproj_TOMO_2 cases (N, views, pixel cm, z cm, couch
# cm/rotation, ite, thinout, seed) and IR_ImageTOMO cases (N, ite, thinout,
# wbefore, w_tv, w_prior, seed) on seeded inputs.
LP2_CASES = [(64, 40, 0.1, 1.0, 0.8, 1, 10, 21), (63, 36, 0.4, 2.0, 1.2, 3, 4, 22), (128, 80, 0.1, 0.5, 0.4, 1, 1, 23)]
IR_CASES = [(64, 1, 10, 0.0106, 1e-4, 0.0, 31), (63, 301, 4, 0.0106, 1e-4, 0.3, 32), (96, 2, 1, 0.02, 0.05, 0.0, 33)]


def lp2_inputs(views, seed, width=609):
    rng = np.random.default_rng(seed)
    p0 = rng.uniform(0.1, 1.0, (views // 2 * 2, width)).astype(np.float32)
    p = rng.uniform(0.1, 1.0, (views // 2 * 2, width)).astype(np.float32)
    return p0, p


def ir_inputs(N, seed):
    rng = np.random.default_rng(seed)
    before = rng.uniform(0.0, 0.2, (N, N)).astype(np.float32)
    npf = rng.uniform(0.0, 5.0, (N, N)).astype(np.float32)
    npf_re = rng.uniform(0.0, 5.0, (N, N)).astype(np.float32)
    prior = rng.uniform(0.0, 0.2, (N, N)).astype(np.float32)
    after = rng.uniform(-1.0, 1.0, (N, N)).astype(np.float32)  # kept outside the mask
    return before, npf, npf_re, prior, after
