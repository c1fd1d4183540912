"""The decomposition's per-slice step control on the CPU: its verdicts, and
projected, quantised descent on a badly conditioned quadratic (eigenvalues
1 .. 1e4), where the adaptive Barzilai-Borwein steps must keep the loss
monotone and reach far below what steepest descent with line minimisation
reaches in the same number of evaluations."""
import numpy as np

from virtualct_b200.decomposition import ACCEPT, REJECT, UNCHANGED, step_control


def test_verdicts():
    assert step_control(10.0, 10.0, 0.0, 0.0, 0.0, 0.0, 0.5) == (UNCHANGED, 2.0)
    # accepted with curvature: BB1 = dd/dy = 2, BB2 = dy/yy = 1.6 (ratio 0.8: BB1)
    v, t = step_control(10.0, 9.0, -2.0, 1.0, 0.5, 0.15625, 1.0)
    assert v == ACCEPT and t == 2.0
    # BB2 / BB1 < 1/2: BB2
    v, t = step_control(10.0, 9.0, -2.0, 1.0, 0.5, 1.0, 1.0)
    assert v == ACCEPT and t == 0.5
    # no positive curvature seen: grow
    assert step_control(10.0, 9.0, -2.0, 1.0, -0.1, 1.0, 1.0) == (ACCEPT, 4.0)
    # loss rose: the quadratic through l(0) = 10, l'(0) = -2, l(1) = 12 has
    # its minimum at 2 / (2 * 4) = 0.25
    v, t = step_control(10.0, 12.0, -2.0, 1.0, 0.5, 1.0, 1.0)
    assert v == REJECT and abs(t - 0.25) < 1e-15
    # a huge rise: at least 1/50 of the step
    assert step_control(10.0, 1e9, -2.0, 1.0, 0.5, 1.0, 1.0) == (REJECT, 0.02)
    # the projected step was no descent direction
    assert step_control(10.0, 12.0, 0.5, 1.0, 0.5, 1.0, 1.0) == (REJECT, 0.25)
    # a decrease too small for the Armijo test is rejected
    assert step_control(10.0, 10.0 - 1e-9, -2.0, 1.0, 0.5, 1.0, 1.0)[0] == REJECT


def _quadratic(n=300, seed=3):
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    h = (q * np.logspace(0, 4, n)) @ q.T
    xs = np.maximum(rng.standard_normal(n), 0.0) * 0.5  # a quarter of the optimum on the bound
    return h, xs


def _descend(h, xs, iters, units, control):
    f = lambda x: 0.5 * (x - xs) @ h @ (x - xs)  # noqa: E731
    rho = xs * 0.9 + 0.05
    x = np.round(rho * units) / units
    loss, g = f(x), h @ (x - xs)
    t = 0.003 / np.abs(g).max()
    hist = [loss]
    for _ in range(iters):
        rt = np.maximum(rho - t * g, 0.0)
        xt = np.round(rt * units) / units
        d = xt - x
        lt, gt = f(xt), h @ (xt - xs)
        y = gt - g
        v, t = control(loss, lt, g @ d, d @ d, d @ y, y @ y, t, g @ g)
        if v == ACCEPT:
            rho, x, loss, g = rt, xt, lt, gt
        hist.append(loss)
    return np.array(hist)


def _steepest(loss, lt, gd, dd, dy, yy, t, g2):
    """Steepest descent with the step at the minimum of the quadratic model
    along the gradient."""
    k = 2.0 * (lt - loss + t * g2) / (t * t)
    tn = min(max(g2 / k, 0.1 * t), 4.0 * t) if k > 0 else 2.0 * t
    return (ACCEPT, tn) if lt < loss else (REJECT, min(tn, 0.5 * t))


def test_bb_descent_on_a_badly_conditioned_quadratic():
    h, xs = _quadratic()
    bb = lambda loss, lt, gd, dd, dy, yy, t, g2: step_control(loss, lt, gd, dd, dy, yy, t)  # noqa: E731
    for units in (1e12, 1e6):
        hb = _descend(h, xs, 100, units, bb)
        hs = _descend(h, xs, 100, units, _steepest)
        assert np.all(np.diff(hb) <= 0)
        assert hb[-1] < 1e-3 * hb[0], (units, hb[-1] / hb[0])
        assert hb[-1] < 0.5 * hs[-1], (units, hb[-1], hs[-1])
