"""Benchmark: MBFPA rays*bins/s and FBP slices/s on the plain single-slice
configuration (512 x 512 grid, 6 element maps of a seeded ellipse phantom,
800 views x 609 channels, 120 kVp Kramers spectrum in 110 1-keV bins, Gaussian
noise, Ram-Lak FBP to 512 x 512).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = the MBFPA hot path for one slice (forward walk + spectral sum for
all 110 bins, max-normalisation, Philox noise) with the slice's inputs
resident in HBM; L2 is flushed (256 MB write) between timed steps and each
step is bracketed by CUDA events on the launching stream.  FBP is timed the
same way in its own loop.  Under torchrun every rank projects its own slice
(phantom seed = rank): weak scaling, no data-path collective; the elapsed time
is the max over ranks.

--impl reference times the reference's own CPU code, reprojection_TOMO and
filterSinogram + reconstructImage compiled from its sources into oracle/_ref/
(rank 0 only; other ranks exit 0).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

V, C, N, PIX = 800, 609, 512, 0.1
SIGMA = 0.0000537  # txt field "Photon noise in detector" of the shipped 120 kV input
SPECTRUM = os.path.join(ROOT, "tests", "golden", "kramers_120kvp.txt")
METRIC = "MBFPA rays*bins/s (FBP slices/s alongside)"
CONFIG_NAME = "plain MBFPA+FBP single slice: 512^2, 6 elements, 800 views x 609 channels, 120 kVp Kramers 110 bins"


def load_inputs(seed: int):
    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    mu, pdf = vct.attenuation_coefficient(SPECTRUM)
    maps = phantoms.ellipse_phantom(seed, N)
    return maps, mu, pdf


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu_id}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 5:  # wait for the first sample
                time.sleep(0.02)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------- our arm
def run_ours(args, rank, world, dist):
    import torch

    import virtualct_b200 as vct

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    maps, mu, pdf = load_inputs(seed=rank)
    NE = len(pdf)
    geo = vct.Geometry()
    ctx = vct.Context(geo, device=dev)
    ctx.set_stream(stream.cuda_stream)
    d_maps = torch.from_numpy(maps).to("cuda")
    ctx.set_maps(d_maps)
    ctx.set_spectrum(mu, pdf)
    d_sino = torch.empty((V, C), dtype=torch.float32, device="cuda")
    d_img = torch.empty((N, N), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        """Per-step CUDA events around fn() with an L2 flush before each step."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / 1e3  # seconds

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    step = lambda: ctx.mbfpa_dev(SIGMA, 1 + rank, d_sino)  # noqa: E731
    fbp_step = lambda: ctx.fbp_dev(d_sino, d_img, 1)  # noqa: E731

    uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    clk = ClockSampler(uuid).__enter__()
    for _ in range(args.warmup):
        step()
        fbp_step()
    barrier()
    launches0 = ctx.kernel_launches
    t_mb = timed(step, args.steps)
    launches_mb = ctx.kernel_launches - launches0
    barrier()
    t_mb = max_over_ranks(t_mb)
    segments_visited = ctx.last_segment_count  # fast walk: includes zero-weight pieces

    barrier()
    t_fbp = max_over_ranks(timed(fbp_step, args.steps))

    # Dominant kernel alone (forward walk + spectral epilogue): per-launch
    # device time for the roofline, same flush discipline.
    barrier()
    t_fwd = max_over_ranks(timed(lambda: ctx.forward_dev(d_sino), args.steps)) / args.steps
    clk.__exit__(None, None, None)
    # Algorithmic work unit: the reference walk's in-grid segments, counted by
    # one forward in exact-walk mode (outside every timed region).
    ctx.set_walk_mode(vct.WALK_EXACT)
    ctx.forward_dev(d_sino)
    segments = ctx.last_segment_count
    ctx.set_walk_mode(vct.WALK_FAST)

    # End to end through the public API with host buffers: per step the maps
    # go host->device from pinned memory and the noisy sinogram comes back.
    h_maps = torch.from_numpy(maps).pin_memory()
    h_out = torch.empty((V, C), dtype=torch.float32).pin_memory()
    h_maps_np, h_out_np = h_maps.numpy(), h_out.numpy()

    def e2e_step():
        ctx.set_maps(h_maps_np)
        vct.lib().vct_mbfpa(ctx.handle, SIGMA, 1 + rank, h_out_np.ctypes.data, None)

    for _ in range(2):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(max(e0.elapsed_time(e1) / 1e3, 0.0) or (time.perf_counter() - t0))
    t_e2e_wall = max_over_ranks(time.perf_counter() - t0)

    if rank != 0:
        return None
    units = V * C * NE  # rays * bins per slice
    value = units * world * args.steps / t_mb
    peaks = vct.probe_peaks(dev)
    meas_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    measured = json.load(open(meas_path)) if os.path.exists(meas_path) else {}
    M = maps.shape[0]
    # Algorithmic bytes of one forward launch: every walk segment gathers the
    # M int16 densities of its pixel, plus the float output per ray.
    alg_bytes = segments * M * 2 + V * C * 4
    achieved = alg_bytes / t_fwd / 1e9
    fp64_flops = segments * 2 * M + V * C * NE * (2 * M + 1)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "rays*bins/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_mb / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 walk + f64 spectral sum (f32 I/O)",
        "data": "synthetic: seeded ellipse phantom (seed = rank), 120 kVp Kramers spectrum",
        "config": {"workload": CONFIG_NAME, "views": V, "channels": C, "grid": N, "pixel_cm": PIX,
                   "elements": M, "energy_bins": NE, "noise_sigma": SIGMA, "slices_per_gpu": 1,
                   "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                   "l2": "flushed (256 MB write) before every timed step"},
        "fbp": {"metric": "FBP slices/s", "value": world * args.steps / t_fbp, "unit": "slices/s",
                "ms_per_slice": t_fbp / args.steps * 1e3, "filter": "Ram-Lak"},
        "pipeline_ms_per_slice": (t_mb + t_fbp) / args.steps * 1e3,
        "e2e": {"value": units * world * args.steps / t_e2e, "unit": "rays*bins/s",
                "h2d_bytes_per_step": int(maps.nbytes), "d2h_bytes_per_step": int(V * C * 4),
                "wall_s": t_e2e_wall, "api": "vct_set_maps + vct_mbfpa (host buffers)"},
        "gpu_launches": int(launches_mb),
        "roofline": {
            "kernel": "forward_kernel (walk + spectral epilogue)",
            "bound": "l2",
            "achieved": achieved,
            "peak": peaks["l2_read_gbs"],
            "unit": "GB/s",
            "frac": achieved / peaks["l2_read_gbs"],
            "traffic": None,
            "peak_source": "measured live: vct_probe_peaks L2 read (ld.global.cg, 16 MB resident)",
            "algorithmic_bytes_per_launch": int(alg_bytes),
            "segments_per_launch": int(segments),
            "segments_visited_per_launch": int(segments_visited),
            "launch_ms": t_fwd * 1e3,
            "hbm_peak_gbs": measured.get("hbm_gbs"),
            "fp64": {"achieved_tflops": fp64_flops / t_fwd / 1e12, "peak_tflops": peaks["fp64_tflops"],
                     "frac": fp64_flops / t_fwd / 1e12 / peaks["fp64_tflops"]},
            "fp32_peak_tflops": peaks["fp32_tflops"],
        },
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(maps, mu, pdf)
    return line


def cpu_baseline(maps, mu, pdf):
    """The reference's reprojection_TOMO (oracle/_ref, built from its sources)
    on all host cores for a bounded sample: 2 of the 110 energy bins over the
    full 800 x 609 sinogram."""
    import oracle as O

    cores = os.cpu_count() or 1
    rho = O.rho_from_maps(maps)
    c, s = O.trig_tables(V)
    if O.ref_available():
        O.ref_reprojection(N, PIX, rho, V, C, c, s, 1, mu, pdf, ke0=0, ke1=1, threads=cores)  # cold tables
        _, secs = O.ref_reprojection(N, PIX, rho, V, C, c, s, 1, mu, pdf, ke0=50, ke1=52, threads=cores)
        return {"value": V * C * 2 / secs, "unit": "rays*bins/s", "cores": cores, "kind": "reference",
                "sample": "reprojection_TOMO for 2 energy bins x 800 views x 609 channels", "seconds": secs}
    g = O.geom()
    t0 = time.perf_counter()
    O.forward_exact(g, c, s, rho, np.ascontiguousarray(mu[:, 50:52]), pdf[50:52].copy(), nthreads=cores)
    secs = time.perf_counter() - t0
    return {"value": V * C * 2 / secs, "unit": "rays*bins/s", "cores": cores, "kind": "port",
            "sample": "oracle forward (reference order) for 2 energy bins x 800 views x 609 channels",
            "seconds": secs}


# ----------------------------------------------------------- reference arm
def run_reference(args, rank):
    if rank != 0:
        return None
    import oracle as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"}
    cores = os.cpu_count() or 1
    maps, mu, pdf = load_inputs(seed=0)
    NE = len(pdf)
    rho = O.rho_from_maps(maps)
    c, s = O.trig_tables(V)
    # One step = reprojection_TOMO (the reference walks every ray once per
    # energy bin, MB/main.cpp:492-506) for one bin over one block of 40 of the
    # 800 views, cycling through blocks and bins; the per-ray work is that of
    # the full sinogram.
    VB = 40

    def ref_step(k):
        b, ke = k % (V // VB), (50 + k) % NE
        cs, sn = np.ascontiguousarray(c[b * VB:(b + 1) * VB]), np.ascontiguousarray(s[b * VB:(b + 1) * VB])
        _, secs = O.ref_reprojection(N, PIX, rho, VB, C, cs, sn, 1, mu, pdf, ke0=ke, ke1=ke + 1, threads=cores)
        return secs

    for w in range(max(args.warmup, 1)):
        ref_step(w)
    total = sum(ref_step(k) for k in range(args.steps))
    value = VB * C * args.steps / total
    # FBP as shipped: single-threaded filterSinogram + reconstructImage, once.
    full, _ = O.ref_reprojection(N, PIX, rho, V, C, c, s, 1, mu, pdf, ke0=0, ke1=1, threads=cores)
    sino = (full / full.max()).astype(np.float32)
    _, _, tf, tb = O.ref_fbp(1, sino, N, PIX, 1, c, s)
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "rays*bins/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3,
        "ms_per_slice_all_bins": total / args.steps * (V // VB) * NE * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 walk, f32 densities (reference CPU code)",
        "data": "synthetic: seeded ellipse phantom (seed 0), 120 kVp Kramers spectrum",
        "config": {"workload": CONFIG_NAME, "views": V, "channels": C, "grid": N, "elements": 6, "energy_bins": NE},
        "fbp": {"metric": "FBP slices/s", "value": 1.0 / (tf + tb), "unit": "slices/s",
                "filter_s": tf, "backprojection_s": tb, "threads": 1},
        "cpu_baseline": {"value": value, "unit": "rays*bins/s", "cores": cores, "kind": "reference",
                         "sample": "reprojection_TOMO, one energy bin x 40 views x 609 channels per step"},
        "e2e": {"value": value, "unit": "rays*bins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "ours" and world > 1:
        import datetime

        import torch
        import torch.distributed as tdist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        line = run_reference(args, rank) if args.impl == "reference" else run_ours(args, rank, world, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
