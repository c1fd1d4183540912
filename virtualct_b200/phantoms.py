"""Seeded synthetic inputs in the reference's own file formats.

* element maps: int16 [M][N][N], value = element partial density x 1000 g/cm^3
  (the layout of Weight_input_ICRU110.raw, read at MB/main.cpp:421-429);
* spectra: one header line then "E_lo E_hi weight" rows in MeV
  (MB/Spectrum/PhaseSpace_photon_120kV_0cm.txt, parsed at
  MB/prior_weight_production.cpp:196-207);
* input txts for the drop-in executables (the reference's positional format).

Tissue mass fractions are the Gammex insert compositions of
MB/phantom_creation_Gammex.cpp:113-212 (water from its :214-218 row); for the
six-element human set (H, C, N, O, P, Ca) Mg and Si are dropped and the rest
renormalised.  No dataset is involved: every phantom is drawn from a seed.
"""
from __future__ import annotations

import numpy as np

ELEMENTS8 = ("H", "C", "N", "O", "P", "Ca", "Mg", "Si")

# Mass fractions in percent, element order H, C, N, O, P, Ca, Mg, Si.
TISSUES = {
    "water": (100 * 2 * 1.00798 / (2 * 1.00798 + 15.9994), 0, 0, 100 * 15.9994 / (2 * 1.00798 + 15.9994), 0, 0, 0, 0),
    "LN300": (8.46, 59.38, 1.96, 18.14, 0.0, 0.0, 11.19, 0.78),
    "LN450": (8.47, 59.57, 1.97, 18.11, 0.0, 0.0, 11.21, 0.58),
    "AP6": (9.06, 72.30, 2.25, 16.27, 0.0, 0.0, 0, 0),
    "BR12": (8.59, 70.11, 2.33, 17.90, 0.0, 0.95, 0, 0),
    "solid_water": (8.02, 67.23, 2.41, 19.91, 0.0, 2.31, 0, 0),
    "brain": (10.83, 72.54, 1.69, 14.86, 0.0, 0.0, 0, 0),
    "LV1": (8.06, 67.01, 2.47, 20.01, 0.0, 2.31, 0, 0),
    "IB3": (6.67, 55.64, 1.96, 23.52, 3.23, 8.86, 0, 0),
    "B200": (6.65, 55.52, 1.98, 23.64, 3.24, 8.87, 0, 0),
    "CB2_30": (6.68, 53.48, 2.12, 25.61, 0.0, 12.01, 0, 0),
    "CB2_50": (4.77, 41.63, 1.52, 32.00, 0.0, 20.02, 0, 0),
    "SB3": (3.41, 31.41, 1.84, 36.50, 0.0, 26.81, 0, 0),
}


def fractions(tissue: str, elements=ELEMENTS8[:6]) -> np.ndarray:
    """Mass fractions of `tissue` over `elements`, renormalised to sum 1."""
    full = np.array(TISSUES[tissue], np.float64)
    idx = [ELEMENTS8.index(e) for e in elements]
    w = full[idx]
    return w / w.sum()


def _paint(maps: np.ndarray, mask: np.ndarray, rho: float, w: np.ndarray) -> None:
    for m in range(maps.shape[0]):
        maps[m][mask] = rho * w[m]


def _finish(dens: np.ndarray) -> np.ndarray:
    # (int) truncation of density*1000 as the Gammex generator writes it.
    return np.trunc(dens * 1000.0).astype(np.int16)


def ellipse_phantom(seed: int, N: int = 512, elements=ELEMENTS8[:6], n_lung: int = 2, n_bone: int = 3,
                    border_px: int = 8) -> np.ndarray:
    """Water body (1.0 g/cc) with lung ellipses (0.3 g/cc) and bone ellipses
    (1.2-1.9 g/cc), int16 [M][N][N].  The outer `border_px` ring stays empty."""
    rng = np.random.default_rng(seed)
    M = len(elements)
    dens = np.zeros((M, N, N), np.float64)
    c = (N - 1) / 2.0
    yy, xx = np.mgrid[0:N, 0:N].astype(np.float64)
    R = c - border_px
    # body
    a = R * rng.uniform(0.80, 0.98)
    b = R * rng.uniform(0.60, 0.85)
    th = rng.uniform(-0.3, 0.3)
    body = _ellipse(xx, yy, c, c, a, b, th)
    _paint(dens, body, 1.0, fractions("water", elements))
    # lungs
    for k in range(n_lung):
        side = -1 if k % 2 == 0 else 1
        cx = c + side * a * rng.uniform(0.35, 0.5)
        cy = c + b * rng.uniform(-0.2, 0.2)
        m = _ellipse(xx, yy, cx, cy, a * rng.uniform(0.18, 0.28), b * rng.uniform(0.35, 0.5),
                     rng.uniform(-0.5, 0.5)) & body
        _paint(dens, m, 0.3, fractions(rng.choice(["LN300", "LN450"]), elements))
    # bones
    for k in range(n_bone):
        r_ = rng.uniform(0.0, 0.6)
        phi = rng.uniform(0, 2 * np.pi)
        cx = c + a * r_ * np.cos(phi)
        cy = c + b * r_ * np.sin(phi)
        m = _ellipse(xx, yy, cx, cy, R * rng.uniform(0.04, 0.12), R * rng.uniform(0.04, 0.12),
                     rng.uniform(0, np.pi)) & body
        _paint(dens, m, rng.uniform(1.2, 1.9), fractions(rng.choice(["SB3", "CB2_50", "IB3"]), elements))
    return _finish(dens)


def _ellipse(xx, yy, cx, cy, a, b, th):
    ct, st = np.cos(th), np.sin(th)
    u = (xx - cx) * ct + (yy - cy) * st
    v = -(xx - cx) * st + (yy - cy) * ct
    return (u / a) ** 2 + (v / b) ** 2 <= 1.0


def gammex_cylinder_phantom(seed: int, N: int = 512, pixel_cm: float = 0.1, elements=ELEMENTS8) -> np.ndarray:
    """33 cm solid-water cylinder with 16 cylindrical inserts (diameter 2.8 cm)
    on two rings of radius 5.5 cm and 10.5 cm (the layout of
    MB/phantom_creation_Gammex.cpp:246-319), each insert a seeded random
    Gammex tissue scaled to a density in [0.3, 1.9] g/cc."""
    rng = np.random.default_rng(seed)
    M = len(elements)
    dens = np.zeros((M, N, N), np.float64)
    c = N / 2.0
    yy, xx = np.mgrid[0:N, 0:N].astype(np.float64)
    x = (xx - c) * pixel_cm
    y = (c - yy) * pixel_cm
    body = np.sqrt(x * x + y * y) <= 16.5
    _paint(dens, body, 1.018, fractions("solid_water", elements))
    names = [t for t in TISSUES if t != "water"]
    for ring_r, phase in ((5.5, 0.0), (10.5, np.pi / 8)):
        for k in range(8):
            th = phase + k * np.pi / 4
            cx, cy = ring_r * np.sin(th), ring_r * np.cos(th)
            m = np.sqrt((x - cx) ** 2 + (y - cy) ** 2) <= 1.4
            _paint(dens, m, rng.uniform(0.3, 1.9), fractions(rng.choice(names), elements))
    return _finish(dens)


# ------------------------------------------------------------------ spectra
def kramers_spectrum(kvp: float, e_min_kev: float = 10.0, bin_kev: float = 1.0) -> np.ndarray:
    """Kramers' law phi(E) ~ (kVp - E)/E on [e_min, kVp] in bin_kev bins.
    Returns rows (E_lo, E_hi, weight) in MeV."""
    edges = np.arange(e_min_kev, kvp + 1e-9, bin_kev)
    lo, hi = edges[:-1], edges[1:]
    e = 0.5 * (lo + hi)
    w = np.clip((kvp - e) / e, 0, None)
    return np.stack([lo / 1000.0, hi / 1000.0, w / w.sum()], axis=1)


def mv_spectrum(e_max_mev: float = 6.0, e_min_mev: float = 0.1, nbins: int = 60) -> np.ndarray:
    """Synthetic thick-target bremsstrahlung shape for a linac beam: Kramers'
    (E0 - E)/E hardened by exp(-0.3/E) for target/flattening-filter
    absorption; `nbins` equal bins on [e_min, e_max] MeV."""
    edges = np.linspace(e_min_mev, e_max_mev, nbins + 1)
    lo, hi = edges[:-1], edges[1:]
    e = 0.5 * (lo + hi)
    w = np.clip((e_max_mev - e) / e, 0, None) * np.exp(-0.3 / e)
    return np.stack([lo, hi, w / w.sum()], axis=1)


def write_spectrum_txt(path, rows: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("1\n")
        for lo, hi, w in rows:
            f.write(f"{lo:.6f} {hi:.6f} {w:.9g}\n")


# --------------------------------------------------------------- input txts
_MB_FIELDS = [
    ("Energy Label (IN (for treatment beam) or PR (for CT))", "{cls}"),
    ("Prior image ON/OFF (0: no prior, 1: planCT, 2: MVCT)", "0"),
    ("sinogram width ", "{width}"),
    ("sinogram height ", "{height}"),
    ("Data type", "float"),
    ("projection image file header bytes ", "0"),
    ("sinogram image data for input ", "{sino}"),
    ("Air scan image data for input // parameters are fixed", "{air}"),
    ("Gantry rotation period [s]", "{period}"),
    ("Data sampling rate [Hz]", "{rate}"),
    ("Starting view angle [degree]", "{start_angle}"),
    ("Couch speed [cm/rotation]", "{couch_speed}"),
    ("Start couch position [cm]", "{couch_start}"),
    ("reconstruction size (square format) ", "{N}"),
    ("reconstruction pixel size [cm]", "{pixel}"),
    ("reconstruction target class string ", "*"),
    ("reconstruction start z [cm]", "{z0}"),
    ("reconstruction z step [cm]", "0.1"),
    ("reconstruction slices ", "1"),
    ("Factor for output CT value ", "{xfactor}"),
    ("reconstruction file name (prior image)", "*"),
    ("number of reconstructed slices (prior image)", "1"),
    ("Prior image shift ", "0.0 0.0 0.0"),
    ("ScanListZvalue", "0.0"),
    ("Thin out for OSEM (NOT used)", "10"),
    ("Constants for regularization terms' weight // TV, Prior, Other (NOT used)", "0.0001 0.0 0.0"),
    ("Gradient Decent constant (NOT used)", "0.01"),
    ("Number of iteration (NOT used)", "500"),
    ("Sinogram factor (NOT used)", "{sino_fact}"),
    ("Spectrum data name", "{spectrum}"),
    ("Photon noise in detector", "{noise}"),
]

_FBP_FIELDS = [
    ("Energy Label (IN : 6MV, PR : 3.5MV)", "{cls}"),
    ("Filter Label (1 : Ram-Lak, 2 : Shepp Logan)", "{filter}"),
    ("sinogram width ", "{width}"),
    ("sinogram height ", "{height}"),
    ("Data type", "float"),
    ("projection image file header bytes ", "0"),
    ("sinogram image data for input ", "{sino}"),
    ("Air scan image data for input // parameters are fixed", "*"),
    ("Gantry rotation period [s]", "{period}"),
    ("Data sampling rate [Hz]", "{rate}"),
    ("Starting view angle [degree]", "{start_angle}"),
    ("Couch speed [cm/rotation] // 0.4=fine, 0.8=normal, 1.2=coarse", "0.0"),
    ("Start couch position [cm]", "0.0"),
    ("reconstruction size (square format) ", "{N}"),
    ("reconstruction pixel size [cm]", "{pixel}"),
    ("reconstruction target class string (used for gating, etc.) ", "*"),
    ("reconstruction start z [cm]", "0.0"),
    ("reconstruction z step [cm]", "0.2"),
    ("reconstruction slices ", "1"),
    ("Factor for output CT value ", "{xfactor}"),
    ("reconstructed data file for output ", "{out}"),
]

_HEADER = ["/" * 56, "// ", "//    Input file (positional format: do not remove header, blank and comment lines)",
           "// ", "//    written by virtualct_b200.phantoms", "/" * 56]


def _write_txt(path, fields, values) -> None:
    lines = list(_HEADER)
    for comment, val in fields:
        lines += ["", "// " + comment, val.format(**values)]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_mb_txt(path, *, spectrum: str, width: int = 609, views: int = 800, N: int = 512, pixel_cm: float = 0.1,
                 noise: float = 0.0, xfactor: int = 1, start_angle: float = 0.0, period: float = 10.0,
                 cls: str = "PR", sino: str = "*", air: str = "*", rotations: int = 1, rate: float | None = None,
                 sino_fact: int = 1, couch_speed: float = 0.0, couch_start: float = 0.0, z0: float = 0.0) -> None:
    """The 31-field MBFPA txt.  The sampling rate defaults to views / period;
    the txt's sinogram height is period * rate raw rows per rotation (5 per
    view at 200 Hz and above), times `rotations`, from which the reader
    derives the rotation count."""
    rate = views / period if rate is None else rate
    height = int(round(period * rate)) * rotations
    _write_txt(path, _MB_FIELDS, dict(cls=cls, width=width, height=height, sino=sino, air=air,
                                      period=f"{period:g}", rate=f"{rate:g}", start_angle=f"{start_angle:g}",
                                      couch_speed=f"{couch_speed:g}", couch_start=f"{couch_start:g}", z0=f"{z0:g}",
                                      N=N, pixel=f"{pixel_cm:g}", xfactor=xfactor, sino_fact=sino_fact,
                                      spectrum=spectrum, noise=f"{noise:.10g}"))


def write_fbp_txt(path, *, sino: str, out: str, filter: int = 1, width: int = 609, views: int = 800, N: int = 512,
                  pixel_cm: float = 0.1, xfactor: int = 1, start_angle: float = 0.0, period: float = 10.0,
                  cls: str = "PR") -> None:
    rate = views / period
    _write_txt(path, _FBP_FIELDS, dict(cls=cls, filter=filter, width=width, height=views, sino=sino,
                                       period=f"{period:g}", rate=f"{rate:g}", start_angle=f"{start_angle:g}", N=N,
                                       pixel=f"{pixel_cm:g}", xfactor=xfactor, out=out))


# ------------------------------------------------------- batched workloads
def kramers_tables(kvp: float, elements=ELEMENTS8[:6], e_min_kev: float = 10.0, bin_kev: float = 1.0):
    """mu [M][NE] and pdf [NE] of a Kramers spectrum through the reference's
    attenuation model (the spectrum goes through its txt format)."""
    import os
    import tempfile

    from . import attenuation_coefficient

    fd, path = tempfile.mkstemp(suffix=".txt", prefix=f"kramers{int(kvp)}_")
    os.close(fd)
    try:
        write_spectrum_txt(path, kramers_spectrum(kvp, e_min_kev, bin_kev))
        return attenuation_coefficient(path, elements)
    finally:
        os.unlink(path)


def batch_specs(n: int, seed: int = 0, grids=(256, 384, 512), kvps=(80, 100, 120, 140), rate=(36, 90),
                channels=(512, 800)):
    """The uneven batch: per slice a seeded ellipse phantom, grid N from
    `grids` (0.1 cm pixels), kVp from `kvps`, views = 10 * DataSamplingRate
    with the rate uniform in `rate`, channels uniform in `channels`."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        out.append({
            "seed": seed * 100003 + i,
            "N": int(rng.choice(grids)),
            "kvp": int(rng.choice(kvps)),
            "views": 10 * int(rng.integers(rate[0], rate[1] + 1)),
            "channels": int(rng.integers(channels[0], channels[1] + 1)),
        })
    return out
