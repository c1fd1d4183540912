"""The reference's iterative step on the GPU, through the C ABI:
lengthproj_TOMO_2 and IR_ImageTOMO against the reference's own outputs
(tests/golden/ir_step.npz), calc_squdiff_quad against a float64 sum, and
vct_ir_step composed of them."""
import numpy as np
import pytest

import oracle as O
import virtualct_b200 as vct
from conftest import golden
from golden_cases import IR_CASES, LP2_CASES, ir_inputs, lp2_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", range(len(LP2_CASES)))
def test_lengthproj2_matches_reference(cuda_device, k):
    N, V, pix, z, cs, ite, th, seed = LP2_CASES[k]
    _, p = lp2_inputs(V, seed)
    with vct.Context(vct.Geometry(views=V, recon_size=N, pixel_cm=pix)) as ctx:
        npf = ctx.lengthproj2(p, ite, th, z, cs).astype(np.float64)
    ref = golden("ir_step.npz")[f"lp2_{k}"].astype(np.float64)
    inside = ref != 0
    assert np.array_equal(npf != 0, inside)
    assert np.max(np.abs(npf[inside] - ref[inside]) / np.abs(ref[inside])) < 1e-5


@pytest.mark.parametrize("k", range(len(IR_CASES)))
def test_ir_update_matches_reference(cuda_device, k):
    import torch

    N, ite, th, wb, wtv, wpr, seed = IR_CASES[k]
    before, npf, npf_re, prior, after = ir_inputs(N, seed)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out = t(after)
    with vct.Context(vct.Geometry(views=40, recon_size=N, pixel_cm=0.1)) as ctx:
        ctx.ir_update_dev(t(before), t(npf), t(npf_re), out, wb, wtv, wpr, ite, th, prior=t(prior))
        ctx.synchronize()
    # IEEE operations in the reference's order (no contraction): bit for bit
    assert np.array_equal(out.cpu().numpy(), golden("ir_step.npz")[f"ir_{k}"])


@pytest.mark.parametrize("ite,thinout,num_ite", [(1, 10, 500), (3, 4, 3), (2, 1, 2)])
def test_squdiff(cuda_device, ite, thinout, num_ite):
    import torch

    V, W = 80, 609
    rng = np.random.default_rng(ite * 7 + thinout)
    p = rng.uniform(0.1, 1.0, (V, W)).astype(np.float32)
    r = rng.uniform(0.1, 1.0, (V, W)).astype(np.float32)
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    with vct.Context(vct.Geometry(views=V, recon_size=64, pixel_cm=0.1)) as ctx:
        ctx.squdiff_dev(torch.from_numpy(p).cuda(), torch.from_numpy(r).cuda(), out, ite, thinout, num_ite)
        ctx.synchronize()
    rows = np.arange((ite - 1) % thinout, V, thinout)[: V // thinout]
    d = (p[rows] - r[rows]).astype(np.float64)
    obj = float((d * d).sum())
    quad = float((0.5 * p[rows] * np.log((p[rows] / r[rows]).astype(np.float64)) ** 2).sum()) if ite == num_ite else 0.0
    got = out.cpu().numpy()
    assert got[0] == pytest.approx(obj, rel=1e-12)
    assert got[1] == pytest.approx(quad, rel=1e-12, abs=1e-300)
