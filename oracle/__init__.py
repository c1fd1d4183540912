"""TEST INFRASTRUCTURE -- the CPU checker for the CUDA path, never product code.

ctypes bindings for

* ``liboracle.so``: this project's plain-C restatement of the reference's MBFPA
  forward projector, noise model and FBP (``vct_oracle.c``; each function cites
  the reference lines it follows);
* ``_ref/libvct_ref_mb.so`` / ``_ref/libvct_ref_fbp.so``: the reference's own
  kernels, compiled from its sources by ``oracle/Makefile`` (present wherever
  the reference sources were available at build time).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (cpu_baseline leg
and ``--impl reference``) import this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF_MB = None
_REF_FBP = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class OrcGeom(C.Structure):
    """Mirror of ``orc_geom`` (vct_oracle.h)."""

    _fields_ = [
        ("start_channel", C.c_int),
        ("end_channel", C.c_int),
        ("iso_channel", C.c_double),
        ("max_alpha", C.c_double),
        ("max_beta", C.c_double),
        ("sid", C.c_double),
        ("det_radius", C.c_double),
        ("det_src_iso", C.c_double),
        ("views", C.c_int),
        ("width", C.c_int),
        ("recon_size", C.c_int),
        ("pixel_cm", C.c_double),
        ("xfactor", C.c_int),
    ]


def geom(views=800, channels=609, recon_size=512, pixel_cm=0.1, xfactor=1, **kw) -> OrcGeom:
    """Reference geometry (physParamsTOMO.h defaults) with the txt fields set.

    ``channels`` sets End_Channel with the reference's own derived quantities:
    isocenter = channels/2.0 (304.5 for 609); Max_alpha/Max_beta stay fixed.
    """
    g = OrcGeom()
    lib().orc_geom_default(C.byref(g))
    g.views = views
    g.width = channels
    g.end_channel = g.start_channel + channels
    g.iso_channel = channels / 2.0
    g.recon_size = recon_size
    g.pixel_cm = pixel_cm
    g.xfactor = xfactor
    for k, v in kw.items():
        setattr(g, k, v)
    return g


def reference_root():
    """Where the reference's sources are: $REF if set, else the default the
    build recipe (oracle/Makefile) holds.  Only test and fixture code reads
    them; the GPU tests and the bench never do."""
    ref = os.environ.get("REF")
    if ref:
        return ref
    import subprocess

    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True, timeout=30)
    except (OSError, subprocess.TimeoutExpired):
        return ""
    return r.stdout.strip() if r.returncode == 0 else ""


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (run `make -C oracle oracle`)")
        L = C.CDLL(path)
        L.orc_geom_default.argtypes = [C.POINTER(OrcGeom)]
        L.orc_trig_tables.argtypes = [C.c_int, C.c_double, _dp, _dp]
        L.orc_spectrum.argtypes = [C.c_char_p, C.c_int, _fp, _dp, C.c_int]
        L.orc_spectrum.restype = C.c_int
        L.orc_attenuation.argtypes = [_dp, C.c_int, _dp, _dp, C.c_int, _fp]
        L.orc_walk.argtypes = [C.POINTER(OrcGeom), C.c_double, C.c_double, C.c_int, _dp, _ip, _dp, C.c_int]
        L.orc_walk.restype = C.c_int
        L.orc_forward_exact.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _fp, C.c_int, _fp, _fp, C.c_int, _fp,
                                        C.c_void_p, C.c_int]
        L.orc_forward_fp64.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _fp, C.c_int, _fp, _fp, C.c_int, _dp,
                                       C.c_void_p, C.c_int]
        L.orc_forward_fp64_maps.argtypes = [C.POINTER(OrcGeom), _dp, _dp,
                                            np.ctypeslib.ndpointer(dtype=np.int16, flags="C_CONTIGUOUS"), C.c_int,
                                            _fp, _fp, C.c_int, _dp, C.c_void_p, C.c_int]
        L.orc_siddon.argtypes = [C.POINTER(OrcGeom), C.c_double, C.c_double, C.c_int, _dp, _ip, C.c_int]
        L.orc_siddon.restype = C.c_int
        L.orc_walk_project.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.orc_walk_backproject.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.orc_beam_hardening.argtypes = [_fp, C.c_longlong, C.c_double, C.c_double, _dp]
        L.orc_lengthproj.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _fp, C.c_double, C.c_double, _fp]
        L.orc_lengthproj2.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _fp, C.c_double, C.c_double, C.c_int, C.c_int,
                                      _fp]
        L.orc_ir_update.argtypes = [C.c_int, _fp, C.c_void_p, _fp, _fp, C.c_double, C.c_double, C.c_double, C.c_int,
                                    C.c_int, _fp]
        L.orc_walk_project_rays.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _dp, C.c_int, _ip, C.c_int, _dp, C.c_int]
        L.orc_siddon_project.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _dp, C.c_int, _dp, C.c_int]
        L.orc_load_measured.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _fp, _u8p,
                                        C.POINTER(C.c_double)]
        L.orc_load_measured.restype = C.c_int
        L.orc_helical.argtypes = [_fp, C.c_int, C.c_int, C.c_int, _fp]
        L.orc_normalize_noise.argtypes = [_fp, C.c_int, C.c_double, C.c_uint, C.c_int]
        L.orc_normalize_noise.restype = C.c_double
        L.orc_fbp_constmap.argtypes = [C.POINTER(OrcGeom), C.c_int, _dp]
        L.orc_fbp_filter.argtypes = [C.POINTER(OrcGeom), _fp, _dp, C.c_int, _fp]
        L.orc_fbp_backproject.argtypes = [C.POINTER(OrcGeom), _fp, _dp, _dp, _fp]
        L.orc_fbp_transpose.argtypes = [C.POINTER(OrcGeom), _dp, _dp, _dp, _dp, _dp]
        L.orc_fbp_fp64.argtypes = [C.POINTER(OrcGeom), _fp, _dp, _dp, _dp, _dp]
        L.orc_mask.argtypes = [C.c_int, _u8p]
        _LIB = L
    return _LIB


# ---------------------------------------------------------------- restatement
ELEMENTS_ZA = {
    # (Z, A) as MB/prior_weight_production.cpp:250-255 (H, C, N, O, P, Ca); Mg and
    # Si follow the same A ~ 2Z convention for the 8-element Gammex phantom.
    "H": (1, 1), "C": (6, 12), "N": (7, 14), "O": (8, 16), "P": (15, 31), "Ca": (20, 40),
    "Mg": (12, 24), "Si": (14, 28),
}


def trig_tables(views, start_deg=0.0):
    c = np.zeros(views, np.float64)
    s = np.zeros(views, np.float64)
    lib().orc_trig_tables(views, start_deg, c, s)
    return c, s


def spectrum(path, nthin=1):
    pdf = np.zeros(1024, np.float32)
    e = np.zeros(1024, np.float64)
    n = lib().orc_spectrum(str(path).encode(), nthin, pdf, e, 1024)
    if n < 0:
        raise FileNotFoundError(path)
    return pdf[:n].copy(), e[:n].copy()


def attenuation(energy_mev, elements=("H", "C", "N", "O", "P", "Ca")):
    Z = np.array([ELEMENTS_ZA[e][0] for e in elements], np.float64)
    A = np.array([ELEMENTS_ZA[e][1] for e in elements], np.float64)
    e = np.ascontiguousarray(energy_mev, np.float64)
    mu = np.zeros(len(elements) * len(e), np.float32)
    lib().orc_attenuation(e, len(e), Z, A, len(elements), mu)
    return mu.reshape(len(elements), len(e))


def walk(g, cosb, sinb, jj):
    cap = 4 * g.recon_size + 64
    ln = np.zeros(cap, np.float64)
    px = np.zeros(cap, np.int32)
    r = np.zeros(cap, np.float64)
    n = lib().orc_walk(C.byref(g), cosb, sinb, jj, ln, px, r, cap)
    if n < 0:
        raise RuntimeError("segment capacity exceeded")
    return ln[:n].copy(), px[:n].copy(), r[:n].copy()


def rho_from_maps(maps_i16):
    """(float)short/1000 as MB/main.cpp:103."""
    return (maps_i16.astype(np.float32) / np.float32(1000)).astype(np.float32)


def forward_exact(g, cos_t, sin_t, rho, mu, pdf, nthreads=0, want_nseg=False):
    M = rho.shape[0]
    NE = len(pdf)
    out = np.zeros((g.views, g.width), np.float32)
    nseg = np.zeros((g.views, g.width), np.int32) if want_nseg else None
    lib().orc_forward_exact(C.byref(g), cos_t, sin_t, np.ascontiguousarray(rho, np.float32), M,
                            np.ascontiguousarray(mu, np.float32), np.ascontiguousarray(pdf, np.float32), NE,
                            out, nseg.ctypes.data if want_nseg else None, nthreads)
    return (out, nseg) if want_nseg else out


def forward_fp64(g, cos_t, sin_t, rho, mu, pdf, nthreads=0, want_lint=False):
    M = rho.shape[0]
    NE = len(pdf)
    out = np.zeros((g.views, g.width), np.float64)
    lint = np.zeros((g.views, g.width, M), np.float64) if want_lint else None
    lib().orc_forward_fp64(C.byref(g), cos_t, sin_t, np.ascontiguousarray(rho, np.float32), M,
                           np.ascontiguousarray(mu, np.float32), np.ascontiguousarray(pdf, np.float32), NE,
                           out, lint.ctypes.data if want_lint else None, nthreads)
    return (out, lint) if want_lint else out


def forward_fp64_maps(g, cos_t, sin_t, maps, mu, pdf, nthreads=0, want_lint=False):
    """FP64 forward with exact s/1000 densities (the device path's density semantics)."""
    maps = np.ascontiguousarray(maps, np.int16)
    M = maps.shape[0]
    NE = len(pdf)
    out = np.zeros((g.views, g.width), np.float64)
    lint = np.zeros((g.views, g.width, M), np.float64) if want_lint else None
    lib().orc_forward_fp64_maps(C.byref(g), cos_t, sin_t, maps, M, np.ascontiguousarray(mu, np.float32),
                                np.ascontiguousarray(pdf, np.float32), NE, out,
                                lint.ctypes.data if want_lint else None, nthreads)
    return (out, lint) if want_lint else out


def siddon(g, cosb, sinb, jj):
    cap = 4 * g.recon_size + 64
    ln = np.zeros(cap, np.float64)
    px = np.zeros(cap, np.int32)
    n = lib().orc_siddon(C.byref(g), cosb, sinb, jj, ln, px, cap)
    return ln[:n].copy(), px[:n].copy()


def walk_project(g, cos_t, sin_t, rho):
    """A rho: the reference walk's line integrals of FP64 densities rho
    (double [M][N][N], g/cm^3) -> double [views][width][M] (cm * g/cm^3)."""
    rho = np.ascontiguousarray(rho, np.float64)
    M = rho.shape[0]
    out = np.zeros((g.views, g.width, M), np.float64)
    lib().orc_walk_project(C.byref(g), cos_t, sin_t, rho, M, out, 0)
    return out


def walk_backproject(g, cos_t, sin_t, w):
    """A^T w for per-ray, per-element weights w (double [views][width][M])."""
    w = np.ascontiguousarray(w, np.float64)
    M = w.shape[2]
    N = g.recon_size
    out = np.zeros((M, N, N), np.float64)
    lib().orc_walk_backproject(C.byref(g), cos_t, sin_t, w, M, out, 0)
    return out


def walk_project_rays(g, cos_t, sin_t, rho, rays):
    """A rho on the rays listed (view * width + channel) -> [len(rays)][M]."""
    rho = np.ascontiguousarray(rho, np.float64)
    rays = np.ascontiguousarray(rays, np.int32)
    M = rho.shape[0]
    out = np.zeros((len(rays), M), np.float64)
    lib().orc_walk_project_rays(C.byref(g), cos_t, sin_t, rho, M, rays, len(rays), out, 0)
    return out


def rays_near_pixel(g, cos_t, sin_t, col, row, margin_px=3.0):
    """Every ray (view * width + channel) whose line passes within margin_px
    pixels of the centre of pixel (col, row): a superset of the rays whose
    walk can put a segment on that pixel (its lumped and folded border pieces
    lie within one pixel of the ray)."""
    N, s = g.recon_size, g.pixel_cm
    n = int(N * 0.5)
    cx, cy = (col - n + 0.5) * s, (n - row - 0.5) * s
    half = (g.end_channel - g.start_channel - 1) // 2
    jj = np.arange(g.start_channel, g.end_channel)
    theta = (g.iso_channel - jj) * g.max_alpha / half
    px0 = g.det_radius * np.sin(theta)
    py0 = -g.det_radius * np.cos(theta) + g.det_src_iso
    out = []
    for v in range(g.views // 2 * 2):
        cb, sb = cos_t[v], sin_t[v]
        sx, sy = g.sid * sb, g.sid * cb
        px, py = px0 * cb + py0 * sb, -px0 * sb + py0 * cb
        dx, dy = px - sx, py - sy
        d = np.abs(dx * (cy - sy) - dy * (cx - sx)) / np.hypot(dx, dy)
        out.extend((v * g.width + jj[d <= margin_px * s]).tolist())
    return np.asarray(out, np.int32)


def loss_terms(L, mu, pdf, meas_r, wts_r, xfactor, ynorm):
    """Per-ray loss 1/2 w (ln(y/ynorm) - ln p)^2 (0 where p <= 0)."""
    y, _ = spectral(L, mu, pdf, xfactor)
    p = np.asarray(meas_r, np.float64)
    w = p if wts_r is None else np.asarray(wts_r, np.float64)
    ok = p > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(ok, np.log(y / ynorm) - np.log(np.where(ok, p, 1.0)), 0.0)
    return np.where(ok, 0.5 * w * r * r, 0.0)


def fd_pixel(g, cos_t, sin_t, rho, m, col, row, h, mu, pdf, meas, weights=None):
    """Central difference (l(rho + h e) - l(rho - h e)) / 2h of the FP64 walk
    loss for element m at pixel (col, row); rays that cannot touch the pixel
    cancel exactly and are left out of both sums."""
    rays = rays_near_pixel(g, cos_t, sin_t, col, row)
    ynorm = float(np.asarray(pdf, np.float32).astype(np.float64).sum())
    mr = np.asarray(meas, np.float32).reshape(-1)[rays]
    wr = None if weights is None else np.asarray(weights, np.float32).reshape(-1)[rays]
    tot = []
    for sgn in (1.0, -1.0):
        r2 = np.array(rho, np.float64, copy=True)
        r2[m, row, col] += sgn * h
        L = walk_project_rays(g, cos_t, sin_t, r2, rays)
        tot.append(loss_terms(L, mu, pdf, mr, wr, g.xfactor, ynorm).sum())
    return (tot[0] - tot[1]) / (2.0 * h)


def spectral(L, mu, pdf, xfactor=1.0):
    """Polyenergetic intensity y = sum_E pdf exp(-sum_m mu_mE L_m / xfactor) and
    its derivative dy/dL_m = -D_m, both FP64; L: [..., M], mu: [M][NE]."""
    mu = np.asarray(mu, np.float64) / float(xfactor)
    pdf = np.asarray(pdf, np.float64)
    e = pdf * np.exp(-(L @ mu))            # [..., NE]
    y = e.sum(-1)
    D = e @ mu.T                           # [..., M]
    return y, D


def loss_grad(g, cos_t, sin_t, rho, mu, pdf, meas, weights=None, want_grad=True):
    """FP64 weighted log least squares of the walk model (the loss of
    MB/main.cpp:125-126 with y/sum(pdf) in place of the max-normalised
    reprojection): l = 1/2 sum_i w_i (ln(y_i/ynorm) - ln p_i)^2 over rays with
    p_i > 0, w_i = p_i unless weights are given; returns (l, dl/drho)."""
    L = walk_project(g, cos_t, sin_t, rho)
    pdf = np.asarray(pdf, np.float64)
    ynorm = float(np.asarray(pdf, np.float32).astype(np.float64).sum())
    y, D = spectral(L, mu, pdf, g.xfactor)
    p = np.asarray(meas, np.float64)
    wt = p if weights is None else np.asarray(weights, np.float64)
    valid = np.zeros(p.shape, bool)
    nv = g.views // 2 * 2
    valid[:nv, g.start_channel:g.end_channel] = True
    valid &= p > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(valid, np.log(y / ynorm) - np.log(np.where(valid, p, 1.0)), 0.0)
    loss = 0.5 * float(np.sum(np.where(valid, wt * r * r, 0.0)))
    if not want_grad:
        return loss
    w = np.where(valid[..., None], -(wt * r / y)[..., None] * D, 0.0)
    return loss, walk_backproject(g, cos_t, sin_t, w)


def siddon_project(g, cos_t, sin_t, x):
    x = np.ascontiguousarray(x, np.float64)
    M = x.shape[0]
    out = np.zeros((g.views, g.width, M), np.float64)
    lib().orc_siddon_project(C.byref(g), cos_t, sin_t, x, M, out, 0)
    return out


def normalize_noise(sino, sigma, seed=1, order=0):
    a = np.ascontiguousarray(sino, np.float32).copy()
    pmin = lib().orc_normalize_noise(a.reshape(-1), a.size, sigma, seed, order)
    return a, pmin


def fbp_constmap(g, filt):
    Cn = g.end_channel - g.start_channel
    h = np.zeros(Cn * Cn, np.float64)
    lib().orc_fbp_constmap(C.byref(g), filt, h)
    return h.reshape(Cn, Cn)


def fbp_filter(g, sino, h, in_mode=0):
    Cn = g.end_channel - g.start_channel
    out = np.zeros((g.views, Cn), np.float32)
    lib().orc_fbp_filter(C.byref(g), np.ascontiguousarray(sino, np.float32), np.ascontiguousarray(h), in_mode,
                         out)
    return out


def fbp_backproject(g, fltd, cos_t, sin_t):
    img = np.zeros((g.recon_size, g.recon_size), np.float32)
    lib().orc_fbp_backproject(C.byref(g), np.ascontiguousarray(fltd, np.float32), cos_t, sin_t, img)
    return img


def fbp(g, sino, filt, cos_t, sin_t, in_mode=0):
    h = fbp_constmap(g, filt)
    q = fbp_filter(g, sino, h, in_mode)
    return fbp_backproject(g, q, cos_t, sin_t), q


def fbp_fp64(g, sino, filt, cos_t, sin_t):
    """The FBP with every sum in double (the FP64 denominator): [N][N]."""
    h = fbp_constmap(g, filt)
    img = np.zeros((g.recon_size, g.recon_size), np.float64)
    lib().orc_fbp_fp64(C.byref(g), np.ascontiguousarray(sino, np.float32), np.ascontiguousarray(h), cos_t, sin_t,
                       img)
    return img


def fbp_transpose(g, u, filt, cos_t, sin_t):
    """FP64 W^T F^T B^T u: the transpose of the FBP in lam = -ln p."""
    h = fbp_constmap(g, filt)
    u = np.ascontiguousarray(u, np.float64)
    out = np.zeros((g.views, g.width), np.float64)
    lib().orc_fbp_transpose(C.byref(g), h, cos_t, sin_t, u, out)
    return out


def ref_lengthproj(N, pixel_cm, proj, V, cos_t, sin_t, z, couch_speed):
    """The reference's own lengthproj_TOMO (oracle/_ref); 609 channels."""
    proj = np.ascontiguousarray(proj, np.float32)
    out = np.zeros((N, N), np.float32)
    secs = C.c_double()
    rc = ref_mb().vctref_lengthproj(N, pixel_cm, proj, proj.shape[1], V, np.ascontiguousarray(cos_t),
                                    np.ascontiguousarray(sin_t), float(z), float(couch_speed), out, C.byref(secs))
    if rc:
        raise RuntimeError(f"vctref_lengthproj failed ({rc})")
    return out, secs.value


def beam_hardening(p, alpha, beta):
    """Beam-hardening correction of transmissions p (float32); returns the
    corrected copy and the (before, after) minima."""
    out = np.array(p, np.float32, copy=True)
    mins = np.zeros(2, np.float64)
    lib().orc_beam_hardening(out.reshape(-1), out.size, float(alpha), float(beta), mins)
    return out, (float(mins[0]), float(mins[1]))


def ref_beam_hardening(p, alpha, beta):
    """The reference's own program (oracle/_ref/bhc) on an 800 x 609
    reprojection_float.raw in a scratch directory: (corrected, printed line)."""
    import subprocess
    import tempfile

    exe = os.path.join(HERE, "_ref", "bhc")
    with tempfile.TemporaryDirectory() as d:
        np.ascontiguousarray(p, np.float32).tofile(os.path.join(d, "reprojection_float.raw"))
        r = subprocess.run([exe, repr(float(alpha)), repr(float(beta))], cwd=d, capture_output=True, text=True,
                           check=True)
        out = np.fromfile(os.path.join(d, "reprojection_float_cor.raw"), np.float32).reshape(np.shape(p))
    return out, r.stdout.strip()


def lengthproj2(g, cos_t, sin_t, proj, ite, thinout, z=0.0, couch_speed=0.0):
    """lengthproj_TOMO_2 restated (side tables recomputed, rounded to float)."""
    proj = np.ascontiguousarray(proj, np.float32)
    out = np.zeros((g.recon_size, g.recon_size), np.float32)
    lib().orc_lengthproj2(C.byref(g), cos_t, sin_t, proj, float(z), float(couch_speed), int(ite), int(thinout), out)
    return out


def ref_lengthproj2(N, pixel_cm, proj0, proj, V, cos_t, sin_t, z, couch_speed, ite, thinout):
    """The reference: lengthproj_TOMO on proj0 (fills its side tables), then
    lengthproj_TOMO_2 on proj for iteration ite."""
    proj0 = np.ascontiguousarray(proj0, np.float32)
    proj = np.ascontiguousarray(proj, np.float32)
    out = np.zeros((N, N), np.float32)
    rc = ref_mb().vctref_lengthproj2(N, pixel_cm, proj0, proj, proj.shape[1], V, np.ascontiguousarray(cos_t),
                                     np.ascontiguousarray(sin_t), float(z), float(couch_speed), int(ite), int(thinout),
                                     out)
    if rc:
        raise RuntimeError(f"vctref_lengthproj2 failed ({rc})")
    return out


def ir_update(before, npf, npf_re, wbefore, w_tv, w_prior=0.0, ite=1, thinout=1, prior=None, after=None):
    before = np.ascontiguousarray(before, np.float32)
    N = before.shape[0]
    out = np.array(before if after is None else after, np.float32, copy=True)
    pr = None if prior is None else np.ascontiguousarray(prior, np.float32)
    lib().orc_ir_update(N, before, None if pr is None else pr.ctypes.data, np.ascontiguousarray(npf, np.float32),
                        np.ascontiguousarray(npf_re, np.float32), float(wbefore), float(w_tv), float(w_prior),
                        int(ite), int(thinout), out)
    return out


def ref_ir_update(before, npf, npf_re, wbefore, w_tv, w_prior=0.0, ite=1, thinout=1, prior=None, after=None):
    before = np.ascontiguousarray(before, np.float32)
    N = before.shape[0]
    out = np.array(before if after is None else after, np.float32, copy=True)
    pr = np.zeros_like(before) if prior is None else np.ascontiguousarray(prior, np.float32)
    rc = ref_mb().vctref_ir_update(N, before, pr, np.ascontiguousarray(npf, np.float32),
                                   np.ascontiguousarray(npf_re, np.float32), float(wbefore), float(w_tv),
                                   float(w_prior), int(ite), int(thinout), out)
    if rc:
        raise RuntimeError(f"vctref_ir_update failed ({rc})")
    return out


def lengthproj(g, cos_t, sin_t, proj, z=0.0, couch_speed=0.0):
    """lengthproj_TOMO restated: npf [N][N] from proj [views used][width]."""
    proj = np.ascontiguousarray(proj, np.float32)
    out = np.zeros((g.recon_size, g.recon_size), np.float32)
    lib().orc_lengthproj(C.byref(g), cos_t, sin_t, proj, float(z), float(couch_speed), out)
    return out


def mask(N):
    m = np.zeros(N * N, np.uint8)
    lib().orc_mask(N, m)
    return m.reshape(N, N)


# ------------------------------------------------------ the reference itself
def ref_available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f)) for f in ("libvct_ref_mb.so", "libvct_ref_fbp.so"))


# The raw layout constants of MB/physParamsTOMO.h:32-33,43-46,64-65.
RAW_LAYOUT = dict(ch=609, skip=27, air_rows=800, air_blocks=5, start_ch=0, end_ch=609)


def load_measured(proj_file, air_file, in_mode, width, views, nskip, rotations, rate_orig, layout=None):
    """orc_load_measured: (code, volume [rotations][views][width], mask, max)."""
    lay = dict(RAW_LAYOUT, **(layout or {}))
    vol = np.zeros((max(rotations, 0), views, width), np.float32)
    mask = np.zeros(vol.shape, np.uint8)
    mx = C.c_double(0.0)
    rpv = 5 if rate_orig >= 200 else 1
    rc = lib().orc_load_measured(str(proj_file).encode(), str(air_file).encode(), int(in_mode), width, views, nskip,
                                 rotations, rpv, lay["ch"], lay["skip"], lay["air_rows"], lay["air_blocks"],
                                 lay["start_ch"], lay["end_ch"], vol, mask, C.byref(mx))
    return rc, vol, mask, mx.value


def helical(vol):
    """orc_helical: the z-interpolated [views][width] sinogram."""
    vol = np.ascontiguousarray(vol, np.float32)
    R, V, W = vol.shape
    out = np.zeros((V, W), np.float32)
    lib().orc_helical(vol, R, V, W, out)
    return out


def ref_load_measured(proj_file, air_file, in_pr, width, height_raw, nskip, rotations, rate_orig):
    """The reference's loadProjectionData (run in the current directory, where
    it writes projections.raw): (return value, volume, mask)."""
    views = height_raw // nskip
    vol = np.zeros((max(rotations, 0), views, width), np.float32)
    mask = np.zeros(vol.shape, np.uint8)
    rc = ref_mb().vctref_load_measured(str(proj_file).encode(), str(air_file).encode(), in_pr.encode(), width,
                                       height_raw, nskip, rotations, float(rate_orig), vol, mask)
    return rc, vol, mask


def ref_mb():
    global _REF_MB
    if _REF_MB is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "libvct_ref_mb.so"))
        L.vctref_attenuation.argtypes = [C.c_char_p, C.c_int, _fp, _fp, C.POINTER(C.c_int)]
        L.vctref_attenuation.restype = C.c_int
        L.vctref_set_threads.argtypes = [C.c_int]
        L.vctref_set_threads.restype = C.c_int
        L.vctref_lengthproj.argtypes = [C.c_int, C.c_double, _fp, C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double,
                                        _fp, C.POINTER(C.c_double)]
        L.vctref_lengthproj.restype = C.c_int
        L.vctref_lengthproj2.argtypes = [C.c_int, C.c_double, _fp, _fp, C.c_int, C.c_int, _dp, _dp, C.c_double,
                                         C.c_double, C.c_int, C.c_int, _fp]
        L.vctref_ir_update.argtypes = [C.c_int, _fp, _fp, _fp, _fp, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_int, _fp]
        L.vctref_reprojection_bins.argtypes = [C.c_int, C.c_double, _fp, C.c_int, C.c_int, _dp, _dp, C.c_int,
                                               _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.POINTER(C.c_double)]
        L.vctref_reprojection_bins.restype = C.c_int
        L.vctref_load_measured.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_double, _fp, _u8p]
        L.vctref_load_measured.restype = C.c_int
        _REF_MB = L
    return _REF_MB


def ref_fbp_lib():
    global _REF_FBP
    if _REF_FBP is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "libvct_ref_fbp.so"))
        L.vctref_fbp.argtypes = [C.c_int, C.c_int, C.c_int, _fp, C.c_int, C.c_double, C.c_int, _dp, _dp, _fp,
                                 C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.vctref_fbp.restype = C.c_int
        _REF_FBP = L
    return _REF_FBP


def ref_attenuation(path, num_material=6):
    att = np.zeros(1024 * num_material, np.float32)
    pdf = np.zeros(1024, np.float32)
    ne = C.c_int(0)
    rc = ref_mb().vctref_attenuation(str(path).encode(), num_material, att, pdf, C.byref(ne))
    if rc != 0:
        raise RuntimeError("reference attenuation_coefficient failed")
    n = ne.value
    return pdf[:n].copy(), att[: num_material * n].reshape(num_material, n).copy()


def ref_reprojection(N, pixel_cm, rho, views, width, cos_t, sin_t, xfactor, mu, pdf, ke0=0, ke1=None,
                     threads=0, want_last=False):
    """Runs the reference's reprojection_TOMO for bins [ke0, ke1) and sums them
    in float (MB/main.cpp:492-506).  Returns (full, seconds[, last_bin])."""
    NE = len(pdf)
    ke1 = NE if ke1 is None else ke1
    if threads:
        ref_mb().vctref_set_threads(threads)
    full = np.zeros((views, width), np.float32)
    last = np.zeros((views, width), np.float32) if want_last else None
    secs = C.c_double(0)
    mu_flat = np.ascontiguousarray(mu, np.float32).reshape(-1)
    rc = ref_mb().vctref_reprojection_bins(N, pixel_cm, np.ascontiguousarray(rho, np.float32), views, width,
                                           cos_t, sin_t, xfactor, mu_flat, np.ascontiguousarray(pdf, np.float32),
                                           NE, ke0, ke1, full.ctypes.data,
                                           last.ctypes.data if want_last else None, None, C.byref(secs))
    if rc != 0:
        raise RuntimeError(f"reference reprojection failed ({rc})")
    return (full, secs.value, last) if want_last else (full, secs.value)


def ref_fbp(filt, sino, N, pixel_cm, xfactor, cos_t, sin_t):
    """The reference's filterSinogram + reconstructImage. Returns (img, fltd, t_filter, t_bp)."""
    V, W = sino.shape
    img = np.zeros((N, N), np.float32)
    fl = np.zeros((V, W), np.float32)
    tf, tb = C.c_double(0), C.c_double(0)
    rc = ref_fbp_lib().vctref_fbp(filt, V, W, np.ascontiguousarray(sino, np.float32), N, pixel_cm, xfactor, cos_t,
                                  sin_t, img, fl.ctypes.data, C.byref(tf), C.byref(tb))
    if rc != 0:
        raise RuntimeError(f"reference fbp failed ({rc})")
    return img, fl, tf.value, tb.value
