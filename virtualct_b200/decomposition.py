"""Material decomposition by projected gradient descent on the element
density maps, driven by the adjoint of the forward projector (no counterpart
in the reference, whose iterative step is a multiplicative ratio update).

Each slice has one measured sinogram per spectrum (dual energy: two).  One
iteration takes, per slice, a trial step from the last accepted point along
the sum of its spectra's gradients (vct_descent_step_dev),

    rho <- max(0, rho - step_s * sum_E dl_E/drho),   maps <- round(rho * units)

then evaluates the loss and gradient of every (slice, spectrum) pair at the
trial points -- all pairs in ONE adjoint batch replay, the path lengths
recomputed by the walk, never stored.  The loss is a function of the
quantised point x = maps / units, so the step actually taken is
d = x_trial - x.  step_control() decides per slice:

  * accept when l(x + d) <= l(x) + 1e-4 g.d (Armijo); the next step is the
    adaptive Barzilai-Borwein step of Zhou, Gao and Dai ("Gradient methods
    with adaptive step-sizes", Comput. Optim. Appl. 35, 2006): with
    y = g(x + d) - g(x), BB1 = d.d / d.y and BB2 = d.y / y.y, take BB2 when
    BB2 / BB1 < 1/2, else BB1.  Plain steepest descent with line
    minimisation zig-zags on this badly conditioned loss (spatial frequencies
    times nearly collinear element spectra); BB steps do not.
  * reject otherwise: return to x and shrink the step to the minimum of the
    quadratic through l(x), g.d and l(x + d), kept within [1/50, 1/2] of it.
  * a trial that changed no map (the step is below the density quantum)
    carries no information: keep x, and grow the step 4x.

So every slice's loss falls monotonically.  The device holds rho (float) and
the maps (int16 at `units` per g/cm^3, 16384 by default: steps of 6e-5
g/cm^3); the host reads S x E losses and S x 4 dot products per iteration.
"""
from __future__ import annotations

import numpy as np

from . import Batch, Context, Geometry, Job, descent_step_dev, descent_step_scaled_dev


class Decomposition:
    def __init__(self, geometry: Geometry, spectra, measured, rho0, *, units: float = 16384.0,
                 step: float | None = None, max_change: float = 0.003, precondition: bool = True,
                 tune: bool = True, device: int = 0):
        """geometry: one Geometry for every slice; spectra: [(mu [M][NE], pdf
        [NE]), ...] one per energy; measured: [slice][energy] CUDA tensors
        [views][width] (max-normalised transmissions); rho0: CUDA float tensor
        [S][M][N][N] (g/cm^3), updated in place.  precondition: scale the
        gradient by the inverse of sqs_diagonal().  The first step moves the
        density with the largest (scaled) gradient by max_change g/cm^3
        unless `step` gives it."""
        import torch

        self.geometry, self.units = geometry, float(units)
        S, M = int(rho0.shape[0]), int(rho0.shape[1])
        E = len(spectra)
        if len(measured) != S or any(len(m) != E for m in measured):
            raise ValueError("measured must be [slices][energies]")
        self.S, self.M, self.E = S, M, E
        self.rho = rho0
        self.maps = torch.round(rho0 * self.units).clamp(0, 32767).to(torch.int16).contiguous()
        N = geometry.recon_size
        self.grads = torch.zeros((S, E, M, N, N), dtype=torch.float32, device=rho0.device)
        self.loss = torch.zeros((S, E), dtype=torch.float64, device=rho0.device)
        jobs = []
        for s in range(S):
            for e, (mu, pdf) in enumerate(spectra):
                jobs.append(Job(geometry, self.maps[s], mu, pdf, meas=measured[s][e], grad=self.grads[s, e],
                                loss=self.loss[s, e:e + 1], density_units=self.units))
        self.batch = Batch(jobs, M=M, device=device, tune=tune)
        # Every step of an iteration -- descent kernels, the batch replay,
        # the reductions the step control reads -- runs on this one stream
        # (or the caller's), so each sees the previous one's results.
        self.stream = torch.cuda.Stream(device=rho0.device)
        self.rho_prev = torch.empty_like(rho0)
        self.maps_prev = torch.empty_like(self.maps)
        self.g = torch.zeros((S, M, N, N), dtype=torch.float32, device=rho0.device)  # at the accepted point
        self.pdiag = self.pscale = None
        if precondition:
            self.pdiag = sqs_diagonal(geometry, spectra, M, device)
            self.pscale = torch.where(self.pdiag > 0, 1.0 / self.pdiag, torch.zeros_like(self.pdiag))
        self.step_size = np.full(S, np.nan if step is None else float(step))
        self.max_change = max_change
        self.cur_loss = None
        self.history: list[float] = []
        self.accepted = 0
        self.rejected = 0
        self.unchanged = 0

    def _on(self, stream_ptr):
        """The stream to run on (the caller's, else the decomposition's own),
        ordered after the work the current stream has queued."""
        import torch

        st = self.stream if stream_ptr is None else torch.cuda.ExternalStream(stream_ptr, device=self.rho.device)
        st.wait_stream(torch.cuda.current_stream(self.rho.device))
        return st

    def _joined(self, st) -> None:
        import torch

        torch.cuda.current_stream(self.rho.device).wait_stream(st)

    def gradients(self, stream_ptr: int | None = None) -> None:
        """Loss and gradient of every (slice, energy) pair at the current maps
        (enqueued; the current stream waits for it)."""
        st = self._on(stream_ptr)
        self.batch.run(st.cuda_stream)
        self._joined(st)

    def _step(self, s: int, step: float, stream_ptr) -> None:
        if self.pscale is None:
            descent_step_dev(self.rho[s], self.g[s], None, step, self.units, self.maps[s], stream_ptr)
        else:
            descent_step_scaled_dev(self.rho[s], self.g[s], self.pscale, step, self.units, self.maps[s], stream_ptr)

    def _requantize(self, s: int, stream_ptr) -> None:
        descent_step_dev(self.rho[s], self.g[s], None, 0.0, self.units, self.maps[s], stream_ptr)

    def iterate(self, n: int = 1, stream_ptr: int | None = None) -> None:
        """n iterations (n loss + gradient evaluations of the whole batch)."""
        import torch

        st = self._on(stream_ptr)
        with torch.cuda.stream(st):
            self._iterate(n, st.cuda_stream)
        self._joined(st)

    def _iterate(self, n: int, stream_ptr: int) -> None:
        import torch

        if self.cur_loss is None:
            self._requantize_all(stream_ptr)
            self.batch.run(stream_ptr)
            self.cur_loss = self.loss.sum(1).cpu().numpy()
            torch.sum(self.grads, 1, out=self.g)
            gp = self.g if self.pscale is None else self.g * self.pscale
            gmax = gp.abs().amax(dim=(1, 2, 3)).cpu().numpy()
            del gp
            fresh = np.isnan(self.step_size)
            self.step_size[fresh] = np.where(gmax[fresh] > 0, self.max_change / np.maximum(gmax[fresh], 1e-30), 0.0)
            self.history.append(float(self.cur_loss.sum()))
            n -= 1
        S = self.S
        stats = torch.empty((S, 4), dtype=torch.float64, device=self.rho.device)
        inv_units = 1.0 / self.units
        for _ in range(max(n, 0)):
            self.rho_prev.copy_(self.rho)
            self.maps_prev.copy_(self.maps)
            for s in range(S):
                self._step(s, float(self.step_size[s]), stream_ptr)
            self.batch.run(stream_ptr)
            for s in range(S):
                d = (self.maps[s].float() - self.maps_prev[s].float()).mul_(inv_units).view(-1)
                y = torch.sum(self.grads[s], 0).sub_(self.g[s]).view(-1)
                gs = self.g[s].view(-1)
                stats[s, 0] = torch.dot(gs, d)
                stats[s, 2] = torch.dot(d, y)
                if self.pdiag is None:
                    stats[s, 1] = torch.dot(d, d)
                    stats[s, 3] = torch.dot(y, y)
                else:  # the BB quotients in the metric of the preconditioner
                    stats[s, 1] = torch.dot(d, d * self.pdiag.view(-1))
                    stats[s, 3] = torch.dot(y, y * self.pscale.view(-1))
            new = self.loss.sum(1).cpu().numpy()
            st = stats.cpu().numpy()
            for s in range(S):
                verdict, t_next = step_control(float(self.cur_loss[s]), float(new[s]), *st[s],
                                               float(self.step_size[s]))
                if verdict == ACCEPT:
                    self.cur_loss[s] = new[s]
                    torch.sum(self.grads[s], 0, out=self.g[s])
                    self.accepted += 1
                else:
                    self.rho[s].copy_(self.rho_prev[s])
                    self.maps[s].copy_(self.maps_prev[s])
                    if verdict == REJECT:
                        self.rejected += 1
                    else:
                        self.unchanged += 1
                self.step_size[s] = t_next
            self.history.append(float(self.cur_loss.sum()))

    def _requantize_all(self, stream_ptr) -> None:
        for s in range(self.S):
            self._requantize(s, stream_ptr)

    # checkpoint / resume ------------------------------------------------------
    def save(self, directory) -> None:
        """Densities of every slice as float32 [M][N][N] raw files
        (rho_sNNNN.raw, the reference's raw layout) and the descent state
        (state.json).  The gradient at the accepted point is not stored: the
        kernels are deterministic, so load() recomputes it bit for bit."""
        import json
        import os

        import torch

        torch.cuda.synchronize(self.rho.device)
        os.makedirs(directory, exist_ok=True)
        for s in range(self.S):
            self.rho[s].cpu().numpy().astype(np.float32).tofile(os.path.join(directory, f"rho_s{s:04d}.raw"))
        state = {"slices": self.S, "elements": self.M, "units": self.units,
                 "step_size": [float(x) for x in self.step_size],
                 "cur_loss": None if self.cur_loss is None else [float(x) for x in self.cur_loss],
                 "history": self.history, "accepted": self.accepted, "rejected": self.rejected,
                 "unchanged": self.unchanged}
        with open(os.path.join(directory, "state.json"), "w") as f:
            json.dump(state, f)

    def load(self, directory, stream_ptr: int | None = None) -> None:
        """Continue from save(): the next iterate() takes the step the saved
        run would have taken."""
        import torch

        st = self._on(stream_ptr)
        with torch.cuda.stream(st):
            self._load(directory, st.cuda_stream)
        self._joined(st)

    def _load(self, directory, stream_ptr: int) -> None:
        import json
        import os

        import torch

        with open(os.path.join(directory, "state.json")) as f:
            state = json.load(f)
        if state["slices"] != self.S or state["elements"] != self.M or state["units"] != self.units:
            raise ValueError("checkpoint does not match this decomposition")
        N = self.geometry.recon_size
        for s in range(self.S):
            a = np.fromfile(os.path.join(directory, f"rho_s{s:04d}.raw"), np.float32).reshape(self.M, N, N)
            self.rho[s].copy_(torch.from_numpy(a))
        self._requantize_all(stream_ptr)
        self.step_size = np.array(state["step_size"], np.float64)
        self.history = list(state["history"])
        self.accepted, self.rejected, self.unchanged = state["accepted"], state["rejected"], state["unchanged"]
        if state["cur_loss"] is None:
            self.cur_loss = None
            return
        self.cur_loss = np.array(state["cur_loss"], np.float64)
        self.batch.run(stream_ptr)
        torch.sum(self.grads, 1, out=self.g)

    def total_loss(self) -> float:
        """Total loss at the accepted points."""
        return float(self.cur_loss.sum()) if self.cur_loss is not None else float("nan")

    def close(self) -> None:
        self.batch.close()


ACCEPT, REJECT, UNCHANGED = 0, 1, 2


def step_control(loss: float, trial_loss: float, gd: float, dd: float, dy: float, yy: float,
                 step: float) -> tuple[int, float]:
    """One slice's verdict on a trial step and its next step size.

    loss, trial_loss: the loss at x and at x + d; gd = g(x).d, dd = d.D.d,
    dy = d.y, yy = y.D^-1.y with y = g(x + d) - g(x) and D the
    preconditioner's diagonal (the identity without one); step: the step
    size that made d.  Returns (ACCEPT | REJECT | UNCHANGED, next step)."""
    if dd == 0.0:
        return UNCHANGED, 4.0 * step
    if trial_loss < loss and trial_loss <= loss + 1e-4 * gd:
        if dy <= 0.0:  # no positive curvature seen along d
            return ACCEPT, 4.0 * step
        bb1 = dd / dy
        bb2 = dy / yy if yy > 0.0 else bb1
        t = bb2 if bb2 < 0.5 * bb1 else bb1
        return ACCEPT, min(max(t, 0.01 * step), 100.0 * step)
    if gd >= 0.0:  # the projected, quantised step is no descent direction
        return REJECT, 0.25 * step
    k = 2.0 * (trial_loss - loss - gd)  # curvature of the quadratic in the step fraction
    frac = -gd / k if k > 0.0 else 0.5
    return REJECT, min(max(frac, 0.02), 0.5) * step


def sqs_diagonal(geometry: Geometry, spectra, M: int, device: int = 0):
    """Diagonal of a separable quadratic surrogate of the loss's Hessian,
    [M][N][N] on the device:

        D[m][j] = sum_E mu_m(E) sum_n mu_n(E) / xfactor^2 * sum_i a_ij L_i

    with mu_m(E) the element's spectrum-mean mass attenuation, a_ij ray i's
    length in pixel j and L_i = sum_k a_ik its whole path in the grid (the
    walk's lumped first segment included).  sum_i a_ij L_i is one forward of
    a unit-density map and one adjoint (vct_line_integrals_dev,
    vct_adjoint_rays_dev).  With J the Jacobian of the log intensities,
    J^T J <= diag(D) when mu is the effective attenuation.  The bound is
    loose (it assumes every pixel of a ray moves together), so it serves as
    a diagonal scaling under the step control, not as a step: what it fixes
    is that the lumped border cells, whose curvature dwarfs the interior's,
    no longer set the step for every pixel."""
    import torch

    N = geometry.recon_size
    rays = (geometry.views // 2 * 2, geometry.channels, 1)
    dev = torch.device("cuda", device)
    st = torch.cuda.Stream(device=dev)
    st.wait_stream(torch.cuda.current_stream(dev))
    with Context(geometry, device=device) as ctx, torch.cuda.stream(st):
        ctx.set_stream(st.cuda_stream)
        ctx.set_maps(np.full((1, N, N), 1000, np.int16))  # 1 g/cm^3
        ctx.set_spectrum(np.ones((1, 1), np.float32), np.ones(1, np.float32))
        L = torch.zeros(rays, dtype=torch.float64, device=dev)
        ctx.line_integrals_dev(L)
        c = torch.zeros((1, N, N), dtype=torch.float32, device=dev)
        ctx.adjoint_rays_dev(L.float(), c)
        ctx.synchronize()
    coef = np.zeros(M)
    for mu, pdf in spectra:
        mu = np.asarray(mu, np.float64)[:M]
        pdf = np.asarray(pdf, np.float64)
        mean = (mu * pdf).sum(1) / pdf.sum()
        coef += mean * mean.sum()
    coef /= float(geometry.xfactor) ** 2
    return torch.from_numpy(coef.astype(np.float32)).to(c.device).view(M, 1, 1) * c


def rays_bins_per_iteration(geometry: Geometry, spectra, slices: int) -> int:
    """Rays x energy bins of one iteration (every slice, every spectrum)."""
    rays = geometry.views // 2 * 2 * geometry.channels
    return int(slices * rays * sum(len(np.asarray(p)) for _, p in spectra))
