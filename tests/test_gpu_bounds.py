"""The index-checked build (libvct_bounds.so, -DVCT_BOUNDS=1) on the GPU:
every kernel family runs on geometries chosen to reach its edges -- coarse and
fine pixels, odd grids, even channel counts (rays through the origin), view
counts with and without the quarter-turn symmetry, moving-couch windows of
lengthproj, measured PR/IN data and the helical interpolation -- and no
index check may fail.  A failed check skips its access and is counted, so the
run cannot fault; it runs in a child process that loads the checked library
(VCT_LIB=bounds)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import json, os, sys, tempfile
import numpy as np
import torch
sys.path.insert(0, ROOT); sys.path.insert(0, os.path.join(ROOT, "tests"))
import virtualct_b200 as vct
from virtualct_b200 import phantoms
import golden_cases as G

assert vct.LIB_PATH.endswith("libvct_bounds.so"), vct.LIB_PATH
vct.bounds_violations()  # clears
runs = []
mu, pdf = phantoms.kramers_tables(120)
for N, pix, views, ch in [(256, 0.1, 200, 609), (127, 0.4, 90, 512), (64, 0.8, 40, 610), (96, 0.5, 122, 800)]:
    geo = vct.Geometry.with_channels(ch, views=views, recon_size=N, pixel_cm=pix)
    maps = phantoms.ellipse_phantom(N + views, N, border_px=0)
    with vct.Context(geo) as ctx:
        ctx.set_maps(maps)
        ctx.set_spectrum(mu, pdf)
        for walk in (vct.WALK_FAST, vct.WALK_EXACT):
            ctx.set_walk_mode(walk)
            sino = ctx.mbfpa(5.37e-5, 3)
        img = ctx.fbp(sino, filter=2)
        lam = ctx.fbp_transpose(img, filter=1)
        try:
            loss, grad = ctx.forward_adjoint(sino)
        except vct.VctError as e:  # pixels too coarse for the gather's channel window
            assert e.code == vct.VCT_E_UNSUPPORTED
            loss = 0.0
        for z, couch in ((0.0, 0.0), (3.7, 0.8), (-2.1, 1.2), (40.0, 0.4)):
            ctx.lengthproj(sino[: views // 2 * 2], z=z, couch_speed=couch)
        runs.append([N, pix, views, ch, bool(np.isfinite(loss))])
with tempfile.TemporaryDirectory() as d:
    cwd = os.getcwd()
    os.chdir(d)
    try:
        for case in list(G.MEAS_CASES.values()):
            G.write_measured(d, case)
            G.write_measured_txt(d, case)
            cfg = vct.MbConfig.load("mb.txt")
            vol, mask, rot, mx = vct.load_measured(cfg)
            vct.helical_sinogram(vol)
    finally:
        os.chdir(cwd)
specs = phantoms.batch_specs(6, seed=3)
jobs = []
for sp in specs:
    g = vct.Geometry.with_channels(sp["channels"], views=sp["views"], recon_size=sp["N"], pixel_cm=0.1)
    m = torch.from_numpy(phantoms.ellipse_phantom(sp["seed"], sp["N"])).cuda()
    tab = phantoms.kramers_tables(sp["kvp"])
    sino = torch.empty((g.views, g.width), dtype=torch.float32, device="cuda")
    img = torch.empty((g.recon_size, g.recon_size), dtype=torch.float32, device="cuda")
    jobs.append(vct.Job(g, m, tab[0], tab[1], sino=sino, img=img, sigma=5.37e-5))
b = vct.Batch(jobs, tune=False)
b.run()
b.synchronize()
b.close()
hits, where = vct.bounds_violations()
print(json.dumps({"hits": hits, "where": where, "runs": runs}))
"""


def test_no_index_check_fails(cuda_device, tmp_path):
    lib = os.path.join(ROOT, "virtualct_b200", "lib", "libvct_bounds.so")
    if not os.path.exists(lib):
        pytest.fail("libvct_bounds.so not built (python -m virtualct_b200.build)")
    env = dict(os.environ, VCT_LIB="bounds")
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CHILD], env=env, capture_output=True, text=True,
                       timeout=900, cwd=tmp_path)
    assert r.returncode == 0, r.stderr[-3000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert len(out["runs"]) == 4 and all(run[-1] for run in out["runs"])
    assert out["hits"] == 0, out
