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


# Measured-data ingestion (loadProjectionData): seeded air scans and measured
# sinograms in the reference's raw layout (609 raw channels, 27 skipped, 800
# air rows, 5 averaged air blocks after the first).  Each case: energy label,
# used width, views per rotation after thinning, sino_fact, rotations,
# sampling rate (Hz; 5 rows per view from 200 on), bytes kept of the measured
# file (None: all), zeroed air channels, the IN upper bound of
# measured / (2 * air) (above 1 takes the reference's stop), seed.
MEAS_RAW = dict(ch=609, skip=27, air_rows=800, air_blocks=5)
MEAS_CASES = {
    "pr_2rot": ("PR", 527, 800, 1, 2, 80.0, None, False, 0.95, 41),
    "pr_thin2": ("PR", 527, 400, 2, 1, 80.0, None, False, 0.95, 42),
    "pr_short": ("PR", 582, 800, 1, 2, 80.0, 800 * 609 * 4 + 1234567, False, 0.95, 43),
    "in_2rot": ("IN", 527, 800, 1, 2, 80.0, None, False, 0.95, 44),
    "in_240hz": ("IN", 527, 480, 1, 2, 240.0, None, False, 0.95, 45),
    "in_air_zero": ("IN", 527, 800, 1, 1, 80.0, None, True, 0.95, 46),
    "in_short": ("IN", 609, 400, 1, 3, 40.0, 609 * 4 * 400 + 10, False, 0.95, 47),
}
MEAS_STOP = ("IN", 527, 800, 1, 2, 80.0, None, False, 1.2, 48)


def write_measured(d, case, proj="proj.raw", air="air.raw"):
    """Writes the air scan and the measured sinogram of `case` into d."""
    import os

    cls, width, views, nskip, rotations, rate, keep, air_zero, hi, seed = case
    rng = np.random.default_rng(seed)
    ch, rows, nb = MEAS_RAW["ch"], MEAS_RAW["air_rows"], MEAS_RAW["air_blocks"]
    a = rng.uniform(1000.0, 2000.0, (1 + nb, rows, ch)).astype(np.float32)
    if air_zero:
        a[:, 0, 100:110] = 0.0
    a.tofile(os.path.join(d, air))
    mean = a[1:].mean(0)
    if cls == "PR":
        p = mean[None] * rng.uniform(0.01, 1.0, (rotations, rows, ch))
    else:
        rpv = 5 if rate >= 200 else 1
        p = 2.0 * mean[0][None, None] * rng.uniform(0.05, hi, (rotations * views * rpv, 1, ch))
    b = p.astype(np.float32).tobytes()
    with open(os.path.join(d, proj), "wb") as f:
        f.write(b if keep is None else b[:keep])


def write_measured_txt(d, case, name="mb.txt", spectrum="spec.txt", N=64, pixel_cm=0.8, couch_speed=0.8, z0=0.4):
    """The MBFPA txt naming the files of write_measured.  The couch moves
    0.8 cm per rotation and the slice sits at z = 0.4 cm, where
    lengthproj_TOMO's first view, (int)(z / (couch / views) - views / 2), is 0
    (with a still couch that expression divides 0 by 0)."""
    import os

    from virtualct_b200 import phantoms

    cls, width, views, nskip, rotations, rate, keep, air_zero, hi, seed = case
    period = 10.0
    phantoms.write_mb_txt(os.path.join(d, name), spectrum=spectrum, width=width, views=views * nskip, N=N,
                          pixel_cm=pixel_cm, cls=cls, sino="proj.raw", air="air.raw", rotations=rotations,
                          rate=rate, sino_fact=nskip, period=period, couch_speed=couch_speed, z0=z0)


# The drop-in on measured data, end to end against the reference's own
# program: IN mode at the full 609 channels (PR would read past the raw row),
# 400 views per rotation, 2 rotations, a 64^2 grid at 0.4 cm, a 2-bin
# spectrum, six-element maps, couch 0.8 cm per rotation, slice at z 0.4 cm.
# (At 0.8 cm some rays cross 129 cells; the reference's per-ray segment
# table holds 2 N = 128 and its writes run past the buffer.)
MEAS_E2E = ("IN", 609, 400, 1, 2, 40.0, None, False, 0.95, 49)
MEAS_E2E_N = 64
MEAS_E2E_PIX = 0.4


def write_e2e_inputs(d):
    import os

    from virtualct_b200 import phantoms

    write_measured(d, MEAS_E2E)
    write_measured_txt(d, MEAS_E2E, N=MEAS_E2E_N, pixel_cm=MEAS_E2E_PIX)
    phantoms.write_spectrum_txt(os.path.join(d, "spec.txt"), phantoms.kramers_spectrum(120, 60.0, 30.0))
    phantoms.ellipse_phantom(50, MEAS_E2E_N, border_px=2).tofile(os.path.join(d, "Weight_input_ICRU110.raw"))
