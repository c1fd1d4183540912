"""Material decomposition by projected gradient descent on the element
density maps, driven by the adjoint of the forward projector (no counterpart
in the reference, whose iterative step is a multiplicative ratio update).

Each slice has one measured sinogram per spectrum (dual energy: two).  One
iteration takes, per slice, a trial step from the last accepted point along
the sum of its spectra's gradients (vct_descent_step_dev),

    rho <- max(0, rho - step_s * sum_E dl_E/drho),   maps <- round(rho * units)

then evaluates the loss and gradient of every (slice, spectrum) pair at the
trial points -- all pairs in ONE adjoint batch replay, the path lengths
recomputed by the walk, never stored.  A slice whose loss fell keeps the
trial point, otherwise it returns to its previous point, so every slice's
loss falls monotonically.  The next step comes from a quadratic model of the
loss along the gradient: with slope -|g|^2 at 0 and the loss l(t) seen at
the trial step t, the curvature is k = 2 (l(t) - l(0) + t |g|^2) / t^2 and
the model's minimum is at |g|^2 / k (kept within [t/10, 4t]).  The
device holds rho (float) and the maps (int16 at `units` per g/cm^3, 16384 by
default: steps of 6e-5 g/cm^3); the host reads S x E losses per iteration.
"""
from __future__ import annotations

import numpy as np

from . import Batch, Geometry, Job, descent_step_dev


class Decomposition:
    def __init__(self, geometry: Geometry, spectra, measured, rho0, *, units: float = 16384.0,
                 step: float | None = None, max_change: float = 0.003, tune: bool = True, device: int = 0):
        """geometry: one Geometry for every slice; spectra: [(mu [M][NE], pdf
        [NE]), ...] one per energy; measured: [slice][energy] CUDA tensors
        [views][width] (max-normalised transmissions); rho0: CUDA float tensor
        [S][M][N][N] (g/cm^3), updated in place.  step: fixed step (g/cm^3 per
        gradient unit); None picks max_change / max|gradient| of the first
        evaluation."""
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
        self.rho_prev = torch.empty_like(rho0)
        self.g = torch.zeros((S, M, N, N), dtype=torch.float32, device=rho0.device)  # at the accepted point
        self.gnorm2 = np.zeros(S)
        self.step_size = np.full(S, np.nan if step is None else float(step))
        self.max_change = max_change
        self.cur_loss = None
        self.history: list[float] = []
        self.accepted = 0
        self.rejected = 0

    def gradients(self, stream_ptr: int | None = None) -> None:
        """Loss and gradient of every (slice, energy) pair at the current maps."""
        self.batch.run(stream_ptr)

    def _requantize(self, s: int, stream_ptr) -> None:
        descent_step_dev(self.rho[s], self.g[s], None, 0.0, self.units, self.maps[s], stream_ptr)

    def iterate(self, n: int = 1, stream_ptr: int | None = None) -> None:
        """n iterations (n loss + gradient evaluations of the whole batch)."""
        import torch

        if self.cur_loss is None:
            self._requantize_all(stream_ptr)
            self.gradients(stream_ptr)
            torch.cuda.synchronize()
            self.cur_loss = self.loss.sum(1).cpu().numpy()
            torch.sum(self.grads, 1, out=self.g)
            gmax = self.g.abs().amax(dim=(1, 2, 3)).cpu().numpy()
            self.gnorm2 = self.g.double().pow(2).sum(dim=(1, 2, 3)).cpu().numpy()
            fresh = np.isnan(self.step_size)
            self.step_size[fresh] = np.where(gmax[fresh] > 0, self.max_change / np.maximum(gmax[fresh], 1e-30), 0.0)
            self.history.append(float(self.cur_loss.sum()))
            n -= 1
        for _ in range(max(n, 0)):
            self.rho_prev.copy_(self.rho)
            for s in range(self.S):
                descent_step_dev(self.rho[s], self.g[s], None, float(self.step_size[s]), self.units, self.maps[s],
                                 stream_ptr)
            self.gradients(stream_ptr)
            torch.cuda.synchronize()
            new = self.loss.sum(1).cpu().numpy()
            for s in range(self.S):
                t = float(self.step_size[s])
                g2 = float(self.gnorm2[s])
                k = 2.0 * (new[s] - self.cur_loss[s] + t * g2) / (t * t) if t > 0 else 0.0
                t_next = min(max(g2 / k, 0.1 * t), 4.0 * t) if k > 0 else 2.0 * t
                if new[s] < self.cur_loss[s]:
                    self.cur_loss[s] = new[s]
                    torch.sum(self.grads[s], 0, out=self.g[s])
                    self.gnorm2[s] = float(self.g[s].double().pow(2).sum())
                    self.accepted += 1
                else:
                    self.rho[s].copy_(self.rho_prev[s])
                    self._requantize(s, stream_ptr)
                    t_next = min(t_next, 0.5 * t)
                    self.rejected += 1
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
        kernels are deterministic, so load() recomputes it bit for bit (its
        squared norm is stored, as the reduction order that made it varies)."""
        import json
        import os

        import torch

        torch.cuda.synchronize()
        os.makedirs(directory, exist_ok=True)
        for s in range(self.S):
            self.rho[s].cpu().numpy().astype(np.float32).tofile(os.path.join(directory, f"rho_s{s:04d}.raw"))
        state = {"slices": self.S, "elements": self.M, "units": self.units,
                 "step_size": [float(x) for x in self.step_size],
                 "cur_loss": None if self.cur_loss is None else [float(x) for x in self.cur_loss],
                 "gnorm2": [float(x) for x in self.gnorm2],
                 "history": self.history, "accepted": self.accepted, "rejected": self.rejected}
        with open(os.path.join(directory, "state.json"), "w") as f:
            json.dump(state, f)

    def load(self, directory, stream_ptr: int | None = None) -> None:
        """Continue from save(): the next iterate() takes the step the saved
        run would have taken."""
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
        self.accepted, self.rejected = state["accepted"], state["rejected"]
        if state["cur_loss"] is None:
            self.cur_loss = None
            return
        self.cur_loss = np.array(state["cur_loss"], np.float64)
        self.gnorm2 = np.array(state["gnorm2"], np.float64)
        self.gradients(stream_ptr)
        torch.cuda.synchronize()
        torch.sum(self.grads, 1, out=self.g)

    def total_loss(self) -> float:
        """Total loss at the accepted points."""
        return float(self.cur_loss.sum()) if self.cur_loss is not None else float("nan")

    def close(self) -> None:
        self.batch.close()


def rays_bins_per_iteration(geometry: Geometry, spectra, slices: int) -> int:
    """Rays x energy bins of one iteration (every slice, every spectrum)."""
    rays = geometry.views // 2 * 2 * geometry.channels
    return int(slices * rays * sum(len(np.asarray(p)) for _, p in spectra))
