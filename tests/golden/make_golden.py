"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has the reference sources ($REF, else the default
written in oracle/Makefile) and `make -C oracle` done:

    python tests/golden/make_golden.py

Every array below is produced by the reference's own code, compiled from its
sources by oracle/Makefile (oracle/_ref/libvct_ref_*.so), except where noted
as the pinned oracle (used only where the reference would need one run per
energy bin for hours).  The GPU tests read these files; they never read REF.

Fixtures
  mu_tables.npz   attenuation_coefficient tables (pdf, mu) of the two shipped
                  spectra and of the synthetic 120 kVp Kramers spectrum.
  mb_small.npz    reprojection_TOMO summed over all bins (MB/main.cpp:492-506)
                  for a seeded 64^2 ellipse phantom, 40 and 41 views.
  fbp_small.npz   filterSinogram + reconstructImage of a 40-view sinogram onto
                  64^2, Ram-Lak and Shepp-Logan.
  c1_subset.npz   full-size single slice (512^2, 800 x 609, 6 elements, 110-bin Kramers
                  spectrum, seeded ellipse phantom seed 0): every 20th view of
                  the reference's un-normalised spectral sum and the FP64
                  oracle's, its global max and min, the total segment count,
                  and every 16th row of the reference's Ram-Lak FBP of the
                  max-normalised, noise-free sinogram and of the FBP with
                  every sum in FP64.
  icru_shipped.npz  the reference's shipped inputs: the ICRU-110 phantom
                  (Weight_input_ICRU110.raw, 6 x 512^2 int16) with the shipped
                  100-bin 120 kV and 650-bin 6 MV spectra, noise-free: every
                  20th view of reprojection_TOMO's spectral sum over all bins
                  (the reference run on those 40 views) and of the FP64
                  oracle's; the 120 kV sum's global max and min (pinned
                  oracle, bit-identical to the reference); and every 8th row
                  of the shipped noisy sinogram (reprojection_float.raw,
                  sigma 5.37e-5).
  fbp_human.npz   the shipped FBP case: the input sinogram
                  (Release_FBP_CPU/reprojection_float.raw, 800 x 609) and every
                  8th row of the shipped Shepp-Logan image
                  (FBP_virtual_projection_512x512_human.raw) and of the FBP
                  with every sum in FP64.
  c2_subset.npz   the 6 MV configuration at full size: 512^2, 8 elements, the
                  seeded 33 cm cylinder with 16 inserts, the synthetic 60-bin
                  6 MV spectrum (mu and pdf of the attenuation model),
                  800 x 609: every 20th view of the pinned oracle's spectral
                  sum in reference order and of the FP64 sum, its max and
                  min, and every 16th row of the Shepp-Logan FBP of the
                  normalised sinogram (reference arithmetic) and in FP64.
  beam_hardening.npz  the beam-hardening correction program's output
                  (reprojection_float_cor.raw, every 32nd row) and printed
                  minima on a seeded 800 x 609 sinogram, kV and MV parameters.
  ir_step.npz     the iterative step's lengthproj_TOMO_2 (side tables from
                  lengthproj_TOMO on a first sinogram) and IR_ImageTOMO on
                  seeded inputs (tests/golden_cases.py).
  lengthproj.npz  lengthproj_TOMO on seeded sinograms (uniform(0.1, 1) from
                  numpy's default_rng(seed), regenerated by the tests): small
                  helical cases in full, and the 512^2 x 800-view case as
                  every 16th row of npf.
  measured.npz    loadProjectionData on seeded measured sinograms and air
                  scans (tests/golden_cases.py MEAS_CASES, regenerated by the
                  tests): return value and SHA-256 of the volume and mask per
                  case, a sample of each volume, and the line the reference
                  prints when an IN-mode value exceeds 1 (MEAS_STOP).
  measured_e2e.npz  the reference's MBFPA program on measured IN-mode input
                  (MEAS_E2E): projections.raw (SHA-256 and nonzero indices),
                  npf_float.raw, the iterative step's two ReconImageRaw
                  files, every 10th view of reprojection_float.raw and the
                  printed maximum.

    python tests/golden/make_golden.py [fixture ...]   (default: all)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from virtualct_b200 import phantoms  # noqa: E402

REF = O.reference_root()
MB = os.path.join(REF, "Release_MBFPA_CPU_human")
FBP_DIR = os.path.join(REF, "Release_FBP_CPU")
OUT = os.path.dirname(os.path.abspath(__file__))

C1_SEED = 0
C1_FBP_ROW_STEP = 16
C1_SUBSET_STEP = 20
SHIP_ROW_STEP = 20      # forward rows of the shipped-input fixture
SHIP_NOISY_STEP = 8     # rows of the shipped noisy sinogram
FBP_HUMAN_ROW_STEP = 8  # image rows of the shipped FBP case
C2_SEED = 3


def kramers_file(tmp, kvp=120):
    p = os.path.join(tmp, f"kramers_{kvp}.txt")
    phantoms.write_spectrum_txt(p, phantoms.kramers_spectrum(kvp))
    return p


def mu_tables(tmp):
    out = {}
    for name, path in (("kv120", os.path.join(MB, "Spectrum/PhaseSpace_photon_120kV_0cm.txt")),
                       ("mv6", os.path.join(MB, "Spectrum/PhaseSpace_photon_6MV_0cm.txt")),
                       ("kramers120", kramers_file(tmp))):
        pdf, mu = O.ref_attenuation(path)
        out[f"{name}_pdf"] = pdf
        out[f"{name}_mu"] = mu
    np.savez_compressed(os.path.join(OUT, "mu_tables.npz"), **out)
    # The Kramers text file itself, so the GPU box can parse the same bytes.
    with open(kramers_file(tmp)) as f:
        txt = f.read()
    with open(os.path.join(OUT, "kramers_120kvp.txt"), "w") as f:
        f.write(txt)
    return out


def mb_small(tabs):
    N, pix = 64, 0.4
    maps = phantoms.ellipse_phantom(7, N, border_px=2)
    rho = O.rho_from_maps(maps)
    pdf, mu = tabs["kv120_pdf"], tabs["kv120_mu"]
    out = {"maps": maps, "N": N, "pixel_cm": pix}
    for V in (40, 41):
        c, s = O.trig_tables(V)
        full, _ = O.ref_reprojection(N, pix, rho, V, 609, c, s, 1, mu, pdf)
        out[f"full_v{V}"] = full
    np.savez_compressed(os.path.join(OUT, "mb_small.npz"), **out)


def fbp_small():
    d = np.load(os.path.join(OUT, "mb_small.npz"))
    full = d["full_v40"]
    sino = (full / full.max()).astype(np.float32)
    c, s = O.trig_tables(40)
    out = {"sino": sino}
    for filt in (1, 2):
        img, fl, _, _ = O.ref_fbp(filt, sino, 64, 0.4, 1, c, s)
        out[f"img_f{filt}"] = img
        out[f"fltd_f{filt}"] = fl
    np.savez_compressed(os.path.join(OUT, "fbp_small.npz"), **out)


def c1_subset(tabs):
    maps = phantoms.ellipse_phantom(C1_SEED, 512)
    rho = O.rho_from_maps(maps)
    pdf, mu = tabs["kramers120_pdf"], tabs["kramers120_mu"]
    c, s = O.trig_tables(800)
    g = O.geom()
    # Pinned oracle in reference order (bit-identical to reprojection_TOMO on
    # the shipped golden); cross-checked against the reference on two bins.
    full, nseg = O.forward_exact(g, c, s, rho, mu, pdf, want_nseg=True)
    ref2, _ = O.ref_reprojection(512, 0.1, rho, 800, 609, c, s, 1, mu, pdf, ke0=50, ke1=52)
    ora2 = O.forward_exact(g, c, s, rho, np.ascontiguousarray(mu[:, 50:52]), pdf[50:52].copy())
    assert np.array_equal(ora2, ref2), "oracle and reference disagree on bins 50-51"
    rows = np.arange(0, 800, C1_SUBSET_STEP)
    f64 = O.forward_fp64(g, c, s, rho, mu, pdf)
    # the reference's FBP (Ram-Lak) of the max-normalised, noise-free sinogram
    # (MB/main.cpp:511-522 in float, then FBP/main.cpp:137-167)
    norm = (full / full.max()).astype(np.float32)
    img, _, _, _ = O.ref_fbp(1, norm, 512, 0.1, 1, c, s)
    img64 = O.fbp_fp64(g, norm, 1, c, s)
    np.savez_compressed(os.path.join(OUT, "c1_subset.npz"), rows=rows, full_rows=full[rows],
                        fp64_rows=f64[rows], fbp_ramlak_rows=img[::C1_FBP_ROW_STEP],
                        fbp_ramlak_fp64_rows=img64[::C1_FBP_ROW_STEP],
                        max=np.float32(full.max()), min=np.float32(full.min()),
                        segments=np.int64(nseg.sum()), seed=C1_SEED,
                        maps_sha=np.frombuffer(__import__("hashlib").sha256(maps.tobytes()).digest(), np.uint8))


def icru_shipped(tabs):
    maps = np.fromfile(os.path.join(MB, "Weight_input_ICRU110.raw"), np.int16).reshape(6, 512, 512)
    rho = O.rho_from_maps(maps)
    c, s = O.trig_tables(800)
    rows = np.arange(0, 800, SHIP_ROW_STEP)
    cs, ss = np.ascontiguousarray(c[rows]), np.ascontiguousarray(s[rows])
    gsub = O.geom(views=len(rows))
    out = {"maps": maps, "rows": rows}
    for name in ("kv120", "mv6"):
        pdf, mu = tabs[f"{name}_pdf"], tabs[f"{name}_mu"]
        # reprojection_TOMO over every bin on the 40 views (each view's rays
        # are walked as in the full run: the walk reads only its cos/sin)
        ref, _ = O.ref_reprojection(512, 0.1, rho, len(rows), 609, cs, ss, 1, mu, pdf)
        out[f"{name}_rows"] = ref
        out[f"{name}_fp64_rows"] = O.forward_fp64(gsub, cs, ss, rho, mu, pdf)
        out[f"{name}_pdf"], out[f"{name}_mu"] = pdf, mu
    # the full 120 kV sum's extremes (the pinned oracle reproduces the shipped
    # noisy output from it bit for bit)
    full = O.forward_exact(O.geom(), c, s, rho, tabs["kv120_mu"], tabs["kv120_pdf"])
    out["kv120_max"], out["kv120_min"] = np.float32(full.max()), np.float32(full.min())
    gold = np.fromfile(os.path.join(MB, "reprojection_float.raw"), np.float32).reshape(800, 609)
    out["noisy_rows"] = np.arange(0, 800, SHIP_NOISY_STEP)
    out["noisy"] = gold[::SHIP_NOISY_STEP]
    out["sigma"] = np.float64(0.0000537)
    np.savez_compressed(os.path.join(OUT, "icru_shipped.npz"), **out)


def fbp_human():
    sino = np.fromfile(os.path.join(FBP_DIR, "reprojection_float.raw"), np.float32).reshape(800, 609)
    gold = np.fromfile(os.path.join(FBP_DIR, "FBP_virtual_projection_512x512_human.raw"), np.float32)
    gold = gold.reshape(512, 512)
    g = O.geom()
    c, s = O.trig_tables(800)
    img, _, _, _ = O.ref_fbp(2, sino, 512, 0.1, 1, c, s)
    assert np.array_equal(img, gold), "the reference built here does not reproduce the shipped FBP image"
    f64 = O.fbp_fp64(g, sino, 2, c, s)
    np.savez_compressed(os.path.join(OUT, "fbp_human.npz"), sino=sino, rows=np.arange(0, 512, FBP_HUMAN_ROW_STEP),
                        golden_rows=gold[::FBP_HUMAN_ROW_STEP], fp64_rows=f64[::FBP_HUMAN_ROW_STEP], filter=2)


def c2_tables():
    """mu [8][60] and pdf [60] of the synthetic 6 MV spectrum (through its
    txt form) for H C N O P Ca Mg Si, by the oracle's attenuation model."""
    with tempfile.TemporaryDirectory() as tmp:
        p = os.path.join(tmp, "mv6_60.txt")
        phantoms.write_spectrum_txt(p, phantoms.mv_spectrum())
        pdf, e = O.spectrum(p)
    return O.attenuation(e, phantoms.ELEMENTS8), pdf


def c2_subset():
    maps = phantoms.gammex_cylinder_phantom(C2_SEED, 512)
    rho = O.rho_from_maps(maps)
    mu, pdf = c2_tables()
    c, s = O.trig_tables(800)
    g = O.geom()
    full = O.forward_exact(g, c, s, rho, mu, pdf)
    f64 = O.forward_fp64(g, c, s, rho, mu, pdf)
    rows = np.arange(0, 800, C1_SUBSET_STEP)
    norm = (full / full.max()).astype(np.float32)
    img, _ = O.fbp(g, norm, 2, c, s)
    img64 = O.fbp_fp64(g, norm, 2, c, s)
    np.savez_compressed(os.path.join(OUT, "c2_subset.npz"), rows=rows, full_rows=full[rows], fp64_rows=f64[rows],
                        max=np.float32(full.max()), min=np.float32(full.min()), mu=mu, pdf=pdf, seed=C2_SEED,
                        fbp_sl_rows=img[::C1_FBP_ROW_STEP], fbp_sl_fp64_rows=img64[::C1_FBP_ROW_STEP],
                        maps_sha=_sha(maps))


sys.path.insert(0, os.path.join(ROOT, "tests"))
from golden_cases import (BH_PARAMS, BH_ROW_STEP, IR_CASES, LP2_CASES, LP_C1, LP_C1_STEP, LP_CASES,  # noqa: E402
                          MEAS_CASES, MEAS_E2E_N, MEAS_STOP, bh_sino, ir_inputs, lp2_inputs, lp_proj,
                          write_e2e_inputs, write_measured)


def lengthproj():
    out = {}
    for k, (N, V, pix, z, cs, seed) in enumerate(LP_CASES + [LP_C1]):
        c, s = O.trig_tables(V)
        npf, _ = O.ref_lengthproj(N, pix, lp_proj(V, seed), V, c, s, z, cs)
        if (N, V, pix, z, cs, seed) == LP_C1:
            out["c1_rows"] = np.arange(0, N, LP_C1_STEP)
            out["c1_npf_rows"] = npf[::LP_C1_STEP]
        else:
            out[f"npf_{k}"] = npf
    np.savez_compressed(os.path.join(OUT, "lengthproj.npz"), **out)


def beam_hardening():
    out = {}
    for k, (a, b) in enumerate(BH_PARAMS):
        cor, line = O.ref_beam_hardening(bh_sino(), a, b)
        out[f"rows_{k}"] = cor[::BH_ROW_STEP]
        out[f"line_{k}"] = np.array(line)
    np.savez_compressed(os.path.join(OUT, "beam_hardening.npz"), **out)


def ir_step():
    out = {}
    for k, (N, V, pix, z, cs, ite, th, seed) in enumerate(LP2_CASES):
        c, s = O.trig_tables(V)
        p0, p = lp2_inputs(V, seed)
        out[f"lp2_{k}"] = O.ref_lengthproj2(N, pix, p0, p, V, c, s, z, cs, ite, th)
    for k, (N, ite, th, wb, wtv, wpr, seed) in enumerate(IR_CASES):
        before, npf, npf_re, prior, after = ir_inputs(N, seed)
        out[f"ir_{k}"] = O.ref_ir_update(before, npf, npf_re, wb, wtv, wpr, ite, th, prior, after)
    np.savez_compressed(os.path.join(OUT, "ir_step.npz"), **out)


def _sha(a):
    import hashlib

    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


def measured():
    """loadProjectionData of the reference (the harness in a scratch
    directory) on every MEAS_CASES input: its return value and the SHA-256 of
    the volume and mask it leaves; and, from a child process (the reference
    exits there), the line it prints when an IN-mode value exceeds 1."""
    import subprocess

    out = {}
    cwd = os.getcwd()
    for name, case in MEAS_CASES.items():
        cls, width, views, nskip, rotations, rate = case[:6]
        with tempfile.TemporaryDirectory() as d:
            write_measured(d, case)
            os.chdir(d)
            try:
                rc, vol, mask = O.ref_load_measured("proj.raw", "air.raw", cls, width, views * nskip, nskip,
                                                    rotations, rate)
            finally:
                os.chdir(cwd)
        out[f"{name}_rc"] = np.int32(rc)
        out[f"{name}_vol_sha"] = _sha(vol)
        out[f"{name}_mask_sha"] = _sha(mask)
        out[f"{name}_vol_sample"] = vol[:, ::37, ::41]
    cls, width, views, nskip, rotations, rate = MEAS_STOP[:6]
    with tempfile.TemporaryDirectory() as d:
        write_measured(d, MEAS_STOP)
        code = ("import sys; sys.path.insert(0, %r); import oracle as O; "
                "O.ref_load_measured('proj.raw', 'air.raw', %r, %d, %d, %d, %d, %r)"
                % (ROOT, cls, width, views * nskip, nskip, rotations, rate))
        r = subprocess.run([sys.executable, "-c", code], cwd=d, capture_output=True, text=True, timeout=300)
    line = [x for x in r.stderr.splitlines() if "STOP" in x]
    assert r.returncode == 0 and len(line) == 1, r.stderr[-500:]
    out["stop_line"] = np.array(line[0].strip())
    np.savez_compressed(os.path.join(OUT, "measured.npz"), **out)


def measured_e2e():
    """The reference's MBFPA program (oracle/_ref/mb_mvct) on measured input
    (golden_cases.MEAS_E2E): projections.raw, npf_float.raw, the iterative
    step's ReconImageRaw outputs and the reprojection."""
    import subprocess

    exe = os.path.join(ROOT, "oracle", "_ref", "mb_mvct")
    N = MEAS_E2E_N
    with tempfile.TemporaryDirectory() as d:
        write_e2e_inputs(d)
        r = subprocess.run([exe, "mb.txt"], cwd=d, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-500:]
        proj = np.fromfile(os.path.join(d, "projections.raw"), np.float32)
        np.savez_compressed(
            os.path.join(OUT, "measured_e2e.npz"),
            projections_sha=_sha(proj), projections_nonzero=np.flatnonzero(proj).astype(np.int32),
            npf=np.fromfile(os.path.join(d, "npf_float.raw"), np.float32).reshape(N, N),
            ite1=np.fromfile(os.path.join(d, "ReconImageRaw", "Reconstruction_ite0001_z0000.raw"),
                             np.float32).reshape(N, N),
            recon16=np.fromfile(os.path.join(d, "ReconImageRaw", f"Reconstruction_512x512x1.raw"), np.int16),
            reprojection_rows=np.fromfile(os.path.join(d, "reprojection_float.raw"), np.float32).reshape(-1, 609)[::10],
            max_line=np.array([x for x in r.stderr.splitlines() if x.startswith("Maximum projection")][0].strip()))


def main():
    if not O.ref_available():
        raise SystemExit("reference harness not built: make -C oracle ref")
    want = set(sys.argv[1:]) or {"mu_tables", "mb_small", "fbp_small", "c1_subset", "lengthproj", "beam_hardening",
                                   "ir_step", "measured", "measured_e2e", "icru_shipped", "fbp_human", "c2_subset"}
    tabs = None
    if want & {"mu_tables", "mb_small", "c1_subset", "icru_shipped"}:
        with tempfile.TemporaryDirectory() as tmp:
            tabs = mu_tables(tmp)
    if "mb_small" in want:
        mb_small(tabs)
    if "fbp_small" in want:
        fbp_small()
    if "c1_subset" in want:
        c1_subset(tabs)
    if "lengthproj" in want:
        lengthproj()
    if "beam_hardening" in want:
        beam_hardening()
    if "ir_step" in want:
        ir_step()
    if "measured" in want:
        measured()
    if "measured_e2e" in want:
        measured_e2e()
    if "icru_shipped" in want:
        icru_shipped(tabs)
    if "fbp_human" in want:
        fbp_human()
    if "c2_subset" in want:
        c2_subset()
    for f in sorted(os.listdir(OUT)):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
