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
# From one ncu capture of forward_kernel<6, COMPENSATED> on this workload
# (C1, 512^2, 800 x 609, 110 bins; `ncu --set full --clock-control none -k
# regex:forward_kernel -s 3 -c 1` of `python bench.py --steps 2 --warmup 3
# --no-cpu-baseline --no-extras`): DRAM bytes read + written per launch (the two
# map copies once; the gathers hit L1/L2) and warp instructions executed per
# launch.  Not measured by the run that prints them.
FWD_CAPTURE = {"dram_bytes": 8582400, "warp_instructions": 2.932e8,
               "source": "ncu capture of forward_kernel<6,0> (integer fixed-point event loop, 6 gathers in flight, "
                         "5 blocks per SM), commit 48c9d28"}
CONFIG_NAME = "plain MBFPA+FBP single slice: 512^2, 6 elements, 800 views x 609 channels, 120 kVp Kramers 110 bins"
# mask pixels of the 512^2 reconstruction circle (FBP/misc.cpp:9-37)
MASK_PX = 205012
# FP32 operations per backprojection update (rotation 6, L^2 4, fan angle 3,
# channel 2, interpolation 3, weight and sum 4; plus one arctangent and one
# reciprocal), FBP/reconstructImageTOMO.cpp:67-93
BP_FLOP_PER_UPDATE = 22


def load_inputs(seed: int):
    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    mu, pdf = vct.attenuation_coefficient(SPECTRUM)
    maps = phantoms.ellipse_phantom(seed, N)
    return maps, mu, pdf


def phantoms_module():
    """virtualct_b200/phantoms.py (numpy only) loaded on its own, so that the
    reference arm never loads the package or its library."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("vct_phantoms_standalone",
                                                  os.path.join(ROOT, "virtualct_b200", "phantoms.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def probe_peaks(device: int) -> dict:
    """Live roofline denominators from lib/libvct_peaks.so (bench-only probes,
    not the product library): L2 read bandwidth, FP64 and FP32 FMA rate."""
    import ctypes

    L = ctypes.CDLL(os.path.join(ROOT, "virtualct_b200", "lib", "libvct_peaks.so"))
    L.vct_probe_peaks.argtypes = [ctypes.c_int] + [ctypes.POINTER(ctypes.c_double)] * 3
    L.vct_peaks_error.restype = ctypes.c_char_p
    l2, f64, f32 = ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
    rc = L.vct_probe_peaks(device, ctypes.byref(l2), ctypes.byref(f64), ctypes.byref(f32))
    if rc != 0:
        raise RuntimeError(f"vct_probe_peaks: {L.vct_peaks_error().decode()}")
    return {"l2_read_gbs": l2.value, "fp64_tflops": f64.value, "fp32_tflops": f32.value}


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
def reduce_max(x: float, dist, device) -> float:
    """Largest x over the ranks (every rank gets it); x itself without a
    process group.  The elapsed times of a multi-rank run are taken this way."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def stage_medians(ctx, fn, reps):
    """Per-stage device times of fn() (vct_set_stage_timing: CUDA events on the
    context's stream around each kernel stage), median over reps calls made
    after the timed regions."""
    ctx.set_stage_timing(True)
    runs = []
    for _ in range(reps):
        fn()
        runs.append(ctx.stage_times())
    ctx.set_stage_timing(False)
    names = [n for n, _ in runs[-1]]
    return {n: statistics.median(r[i][1] for r in runs if len(r) > i) for i, n in enumerate(names)}


def issue_roofline(warp_inst, t_launch, clocks, dev):
    """Instruction-issue axis of a kernel: warp instructions per launch (from
    an ncu capture) over the launch time, against one warp instruction per
    clock per SM sub-partition (4 per SM) at the median SM clock sampled under
    load."""
    import torch

    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    peak = 4.0 * sms * mhz * 1e6
    achieved = warp_inst / t_launch
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "warp_instructions_per_launch": warp_inst, "sm_mhz": mhz,
            "source": "warp instructions: " + FWD_CAPTURE["source"]}


def fbp_roofline(stages, views, channels, mask_px, peaks):
    """Rooflines of the FBP's two compute kernels from their live stage times:
    the filter against the FP32 FMA peak (2 V C^2 FLOP, the reference's dense
    609-tap convolution per sample) and the backprojection against the same
    peak at BP_FLOP_PER_UPDATE per (mask pixel, view) update."""
    used = views // 2 * 2
    out = {"stages_ms": stages}
    t_f = stages.get("fbp_weight_filter_kernel")
    t_b = stages.get("fbp_backproject")
    if t_f:
        fl = 2.0 * views * channels * channels
        out["filter"] = {"kernel": "fbp_weight_filter_kernel (the weight -ln p * coeff fused into the row load)",
                         "bound": "fp32", "achieved": fl / t_f / 1e9, "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                         "frac": fl / t_f / 1e9 / peaks["fp32_tflops"], "flop_per_launch": fl, "launch_ms": t_f}
    if t_b:
        upd = float(mask_px) * used
        fl = upd * BP_FLOP_PER_UPDATE
        out["backprojection"] = {"bound": "fp32", "achieved": fl / t_b / 1e9, "peak": peaks["fp32_tflops"],
                                 "unit": "TFLOP/s", "frac": fl / t_b / 1e9 / peaks["fp32_tflops"],
                                 "updates_per_launch": upd, "updates_per_s": upd / t_b * 1e3,
                                 "flop_per_update": BP_FLOP_PER_UPDATE, "launch_ms": t_b}
    return out


def replica_inputs(rank: int):
    """Each rank projects its own slice: the phantom seed is the rank."""
    return load_inputs(seed=rank)


def run_ours(args, rank, world, dist):
    import torch

    import virtualct_b200 as vct

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    maps, mu, pdf = replica_inputs(rank)
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
        return reduce_max(x, dist, "cuda")

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
    fbp_stages = stage_medians(ctx, fbp_step, max(args.warmup, 5))

    # Dominant kernel alone (forward walk + spectral epilogue): per-launch
    # device time for the roofline, same flush discipline.
    barrier()
    t_fwd = max_over_ranks(timed(lambda: ctx.forward_dev(d_sino), args.steps)) / args.steps
    # Algorithmic work unit: the reference walk's in-grid segments, counted by
    # one forward in exact-walk mode (outside every timed region).
    ctx.set_walk_mode(vct.WALK_EXACT)
    ctx.forward_dev(d_sino)
    segments = ctx.last_segment_count
    ctx.set_walk_mode(vct.WALK_FAST)
    extras = {}
    if rank == 0:
        extras["parity"] = parity_vs_reference(ctx, d_sino, d_img)
    want = set() if args.no_extras or world > 1 else set(args.extras.split(","))
    if "c2" in want:
        extras["c2"] = bench_c2(stream, timed, args.steps, args.warmup)
    if "adjoint" in want:
        extras["adjoint"] = bench_adjoint(ctx, d_maps, mu, pdf, stream, timed, args.steps, args.warmup, segments,
                                          dev)
    if "lengthproj" in want:
        extras["lengthproj"] = bench_lengthproj(ctx, stream, timed, args.steps, args.warmup)
    if "fbp_transpose" in want:
        extras["fbp_transpose"] = bench_fbp_transpose(ctx, stream, timed, args.steps, args.warmup, dev)
    if "batched" in want:
        extras["batched"] = bench_batched(stream, args.warmup, n=args.batch_slices)
    if "scale" in want:
        extras["scale"] = bench_scale(stream, args.scale_slices, args.scale_iters)
    if "batched_adjoint" in want:
        extras["batched_adjoint"] = bench_batched_adjoint(stream, args.warmup, n=max(args.batch_slices // 4, 1))
    clk.__exit__(None, None, None)

    # End to end through the public API with host buffers: every step's maps
    # go host->device from pinned memory and every noisy sinogram comes back
    # to pinned memory; vct_mbfpa_many pipelines those copies behind the
    # projections (copy streams, double buffers).
    import ctypes

    M_maps = int(maps.shape[0])
    h_maps = torch.from_numpy(maps).pin_memory()
    h_outs = [torch.empty((V, C), dtype=torch.float32).pin_memory() for _ in range(2)]

    def e2e_run(k):
        pin = (ctypes.c_void_p * k)(*([h_maps.data_ptr()] * k))
        pout = (ctypes.c_void_p * k)(*[h_outs[i % 2].data_ptr() for i in range(k)])
        vct._check(vct.lib().vct_mbfpa_many(ctx.handle, k, pin, M_maps, SIGMA, 1 + rank, pout, None),
                   "vct_mbfpa_many")

    e2e_run(max(args.warmup, 2))
    barrier()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    e2e_run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = max_over_ranks(max(e0.elapsed_time(e1) / 1e3, 0.0) or (time.perf_counter() - t0))
    t_e2e_wall = max_over_ranks(time.perf_counter() - t0)

    if rank != 0:
        return None
    units = V * C * NE  # rays * bins per slice
    value = units * world * args.steps / t_mb
    peaks = probe_peaks(dev)
    clocks = clk.summary()
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
                "ms_per_slice": t_fbp / args.steps * 1e3, "filter": "Ram-Lak",
                "roofline": fbp_roofline(fbp_stages, V, C, MASK_PX, peaks)},
        "pipeline_ms_per_slice": (t_mb + t_fbp) / args.steps * 1e3,
        "e2e": {"value": units * world * args.steps / t_e2e, "unit": "rays*bins/s",
                "h2d_bytes_per_step": int(maps.nbytes), "d2h_bytes_per_step": int(V * C * 4),
                "wall_s": t_e2e_wall,
                "api": "vct_mbfpa_many (pinned host buffers; uploads and downloads pipelined behind the projections)"},
        "gpu_launches": int(launches_mb),
        "roofline": {
            "kernel": "forward_kernel (walk + spectral epilogue)",
            "bound": "l2",
            "achieved": achieved,
            "peak": peaks["l2_read_gbs"],
            "unit": "GB/s",
            "frac": achieved / peaks["l2_read_gbs"],
            "traffic": FWD_CAPTURE["dram_bytes"],
            "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch, " + FWD_CAPTURE["source"],
            "peak_source": "measured live: libvct_peaks L2 read probe (ld.global.cg, 16 MB resident)",
            "issue": issue_roofline(FWD_CAPTURE["warp_instructions"], t_fwd, clocks, dev),
            "algorithmic_bytes_per_launch": int(alg_bytes),
            "segments_per_launch": int(segments),
            "segments_visited_per_launch": int(segments_visited),
            "launch_ms": t_fwd * 1e3,
            "hbm_peak_gbs": measured.get("hbm_gbs"),
            "fp64": {"achieved_tflops": fp64_flops / t_fwd / 1e12, "peak_tflops": peaks["fp64_tflops"],
                     "frac": fp64_flops / t_fwd / 1e12 / peaks["fp64_tflops"]},
            "fp32_peak_tflops": peaks["fp32_tflops"],
        },
        "clocks": clocks,
    }
    line.update(extras)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(maps, mu, pdf)
    return line


# ------------------------------------------------------------------ parity
def parity_vs_reference(ctx, d_sino, d_img):
    """Errors of this rank-0 slice (phantom seed 0, the bench spectrum) against
    tests/golden/c1_subset.npz: the un-normalised forward on every 20th view
    against the reference's spectral sum (reprojection_TOMO over 110 bins in
    its order) and against the FP64 sum; and the Ram-Lak FBP of the
    max-normalised, noise-free sinogram against the reference's FBP on every
    16th image row."""
    import torch

    path = os.path.join(ROOT, "tests", "golden", "c1_subset.npz")
    if not os.path.exists(path):
        return {"unavailable": "c1_subset fixture missing"}
    d = np.load(path)
    if int(d["seed"]) != 0:
        return {"unavailable": "c1_subset fixture is not the seed-0 slice"}
    rows = d["rows"]
    ctx.forward_dev(d_sino)
    torch.cuda.synchronize()
    out = d_sino.cpu().numpy()[rows].astype(np.float64)
    ref, f64 = d["full_rows"].astype(np.float64), d["fp64_rows"]
    ok = ref > 0
    ctx.mbfpa_dev(0.0, 1, d_sino)  # sigma 0: max-normalisation only
    ctx.fbp_dev(d_sino, d_img, 1)
    torch.cuda.synchronize()
    step = N // d["fbp_ramlak_rows"].shape[0]
    img = d_img.cpu().numpy()[::step].astype(np.float64)
    fref = d["fbp_ramlak_rows"].astype(np.float64)
    f64img = d["fbp_ramlak_fp64_rows"].astype(np.float64)
    out_line = {
        "forward_vs_reference_max_rel": float(np.max(np.abs(out[ok] - ref[ok]) / ref[ok])),
        "forward_vs_fp64_max_rel": float(np.max(np.abs(out - f64) / f64)),
        "reference_vs_fp64_max_rel": float(np.max(np.abs(ref - f64) / f64)),
        "forward_tolerance": 1e-5,
        "fbp_vs_reference_max_abs_over_max": _max_abs_over_max(img, fref),
        "fbp_vs_reference_l2_rel": _l2_rel(img, fref),
        "fbp_vs_fp64_max_abs_over_max": _max_abs_over_max(img, f64img),
        "fbp_vs_fp64_l2_rel": _l2_rel(img, f64img),
        "reference_fbp_vs_fp64_max_abs_over_max": _max_abs_over_max(fref, f64img),
        "fbp_tolerance": 1e-4,
        "what": "forward: un-normalised polyenergetic sinogram, every 20th view (40 x 609); fbp: Ram-Lak image of "
                "the noise-free normalised sinogram, every 16th row (32 x 512); references from the reference "
                "compiled from its sources and the FP64 oracle (FBP with every sum in FP64)",
    }
    out_line["shipped"] = parity_shipped()
    return out_line


def _max_abs_over_max(a, ref):
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    return float(np.abs(a - ref).max() / np.abs(ref).max())


def _l2_rel(a, ref):
    a, ref = np.asarray(a, np.float64), np.asarray(ref, np.float64)
    return float(np.linalg.norm(a - ref) / np.linalg.norm(ref))


def parity_shipped():
    """The device path on the reference's shipped inputs (fixtures from the
    reference compiled from its sources): the ICRU-110 phantom with the
    shipped 100-bin 120 kV and 650-bin 6 MV spectra (noise-free forward,
    every 20th view) and the shipped human FBP case (Shepp-Logan, every 8th
    row), each against the reference and the FP64 oracle."""
    import torch

    import virtualct_b200 as vct

    res = {}
    path = os.path.join(ROOT, "tests", "golden", "icru_shipped.npz")
    if os.path.exists(path):
        d = np.load(path)
        rows = d["rows"]
        with vct.Context(vct.Geometry()) as c2:
            c2.set_maps(d["maps"])
            for name in ("kv120", "mv6"):
                c2.set_spectrum(d[f"{name}_mu"], d[f"{name}_pdf"])
                out = c2.forward()[rows].astype(np.float64)
                ref, f64 = d[f"{name}_rows"].astype(np.float64), d[f"{name}_fp64_rows"]
                res[f"icru110_{name}"] = {
                    "bins": int(len(d[f"{name}_pdf"])),
                    "forward_vs_reference_max_rel": float(np.max(np.abs(out - ref) / ref)),
                    "forward_vs_fp64_max_rel": float(np.max(np.abs(out - f64) / f64)),
                    "reference_vs_fp64_max_rel": float(np.max(np.abs(ref - f64) / f64))}
    path = os.path.join(ROOT, "tests", "golden", "fbp_human.npz")
    if os.path.exists(path):
        d = np.load(path)
        with vct.Context(vct.Geometry()) as c2:
            img = c2.fbp(d["sino"], int(d["filter"]))[d["rows"]]
        res["human_fbp_shepp_logan"] = {
            "vs_reference_max_abs_over_max": _max_abs_over_max(img, d["golden_rows"]),
            "vs_reference_l2_rel": _l2_rel(img, d["golden_rows"]),
            "vs_fp64_max_abs_over_max": _max_abs_over_max(img, d["fp64_rows"]),
            "vs_fp64_l2_rel": _l2_rel(img, d["fp64_rows"]),
            "reference_vs_fp64_max_abs_over_max": _max_abs_over_max(d["golden_rows"], d["fp64_rows"])}
    torch.cuda.synchronize()
    return res


# ------------------------------------------------ adjoint and batched lines
def _event_ms(stream, fn, reps):
    """Best of `reps` CUDA-event timings of fn() on `stream` (after one run)."""
    import torch

    fn()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def bench_adjoint(ctx, d_maps, mu, pdf, stream, timed, steps, warmup, segments, dev):
    """Loss + gradient at 512^2, 6 elements, 120 kVp, 800 x 609 (the adjoint
    configuration): measured sinogram = the noisy MBFPA of the phantom, the
    gradient taken at densities x 0.97.  One step = vct_forward_adjoint_dev
    (walk + ray factors, exact-walk scatter when needed, pixel-driven A^T
    gather, fixed-order loss sum); A^T alone is timed with fixed ray factors."""
    import torch

    meas = torch.empty((V, C), dtype=torch.float32, device="cuda")
    ctx.mbfpa_dev(SIGMA, 7, meas)
    at = (d_maps.double() * 0.97).round().to(torch.int16)
    ctx.set_maps(at)
    grad = torch.empty((6, N, N), dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    fn = lambda: ctx.forward_adjoint_dev(meas, grad, loss=loss)  # noqa: E731
    for _ in range(warmup):
        fn()
    n0 = ctx.kernel_launches
    t = timed(fn, steps) / steps
    launches = (ctx.kernel_launches - n0) // steps
    gr = torch.randn((V, C, 6), dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    g_fn = lambda: ctx.adjoint_rays_dev(gr, grad)  # noqa: E731
    for _ in range(warmup):
        g_fn()
    t_g = timed(g_fn, steps) / steps
    stages = stage_medians(ctx, fn, max(warmup, 5))
    ctx.set_maps(d_maps)
    NE = len(pdf)
    peaks = probe_peaks(dev)
    # A^T moves the forward's data the other way: one ray factor per
    # (segment, element) meets one map cell.  Its unit is the forward's gather
    # bytes, S*M*2 + V*C*4 per launch.
    alg = segments * int(d_maps.shape[0]) * 2 + V * C * 4
    t_gk = stages.get("adj_gather_kernel")
    roof = {"stages_ms": stages}
    if t_gk:
        roof.update({"kernel": "adj_gather_kernel", "bound": "l2", "achieved": alg / t_gk / 1e6,
                     "peak": peaks["l2_read_gbs"], "unit": "GB/s", "frac": alg / t_gk / 1e6 / peaks["l2_read_gbs"],
                     "algorithmic_bytes_per_launch": int(alg), "launch_ms": t_gk,
                     "unit_note": "the forward's gather bytes S*M*2 + V*C*4 (S: the walk's segments)"})
    return {"workload": "loss + dl/drho: 512^2, 6 elements, 120 kVp 110 bins, 800 views x 609 channels",
            "ms_per_gradient": t * 1e3, "rays_bins_per_s": V * C * NE / t,
            "gather_ms": t_g * 1e3, "gather_pixel_views_per_s": N * N * V / t_g,
            "kernels_per_gradient": int(launches), "loss": float(loss.item()), "roofline": roof,
            "notes": "deterministic: pixel-driven A^T, no float atomics"}


def bench_c2(stream, timed, steps, warmup):
    """The 6 MV configuration: 512^2 at 0.1 cm, 8 elements (H C N O P Ca Mg
    Si), the seeded 33 cm cylinder with 16 inserts (tests/golden/c2_subset.npz's
    slice), the synthetic 60-bin 6 MV spectrum, 800 x 609: MBFPA (noise) and
    the Shepp-Logan FBP per slice, L2 flushed before every step; the forward
    kernel's gather-byte roofline; parity against the fixture."""
    import torch

    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    d = np.load(os.path.join(ROOT, "tests", "golden", "c2_subset.npz"))
    maps = phantoms.gammex_cylinder_phantom(int(d["seed"]), N)
    mu, pdf = d["mu"], d["pdf"]
    NE, M = len(pdf), maps.shape[0]
    sino = torch.empty((V, C), dtype=torch.float32, device="cuda")
    img = torch.empty((N, N), dtype=torch.float32, device="cuda")
    with vct.Context(vct.Geometry()) as c2:
        c2.set_stream(stream.cuda_stream)
        c2.set_maps(torch.from_numpy(maps).cuda())
        c2.set_spectrum(mu, pdf)
        step = lambda: c2.mbfpa_dev(SIGMA, 3, sino)  # noqa: E731
        fstep = lambda: c2.fbp_dev(sino, img, 2)  # noqa: E731
        for _ in range(warmup):
            step()
            fstep()
        t_mb = timed(step, steps) / steps
        t_fbp = timed(fstep, steps) / steps
        t_fwd = timed(lambda: c2.forward_dev(sino), steps) / steps
        out = torch.empty_like(sino)
        c2.forward_dev(out)
        c2.synchronize()
        rows = d["rows"]
        o = out.cpu().numpy()[rows].astype(np.float64)
        c2.set_walk_mode(vct.WALK_EXACT)
        c2.forward_dev(out)
        c2.synchronize()
        segments = c2.last_segment_count
        c2.set_walk_mode(vct.WALK_FAST)
    peaks = probe_peaks(torch.cuda.current_device())
    alg = segments * M * 2 + V * C * 4
    ref, f64 = d["full_rows"].astype(np.float64), d["fp64_rows"]
    return {"workload": "6 MV: 512^2, 8 elements, 16-insert cylinder (seed %d), 800 views x 609 channels, "
                        "synthetic 6 MV 60 bins; MBFPA + noise, Shepp-Logan FBP" % int(d["seed"]),
            "value": V * C * NE / t_mb, "unit": "rays*bins/s", "ms_per_slice": t_mb * 1e3,
            "fbp_slices_per_s": 1.0 / t_fbp, "fbp_ms_per_slice": t_fbp * 1e3,
            "roofline": {"kernel": "forward_kernel<8>", "bound": "l2", "achieved": alg / t_fwd / 1e9,
                         "peak": peaks["l2_read_gbs"], "unit": "GB/s", "frac": alg / t_fwd / 1e9 / peaks["l2_read_gbs"],
                         "algorithmic_bytes_per_launch": int(alg), "segments_per_launch": int(segments),
                         "launch_ms": t_fwd * 1e3},
            "parity": {"forward_vs_oracle_max_rel": float(np.max(np.abs(o - ref) / ref)),
                       "forward_vs_fp64_max_rel": float(np.max(np.abs(o - f64) / f64))},
            "l2": "flushed (256 MB write) before every timed step"}


def bench_lengthproj(ctx, stream, timed, steps, warmup):
    """lengthproj_TOMO of a 800 x 609 sinogram onto the 512^2 mask (helical
    couch 0.8 cm/rotation at z = 3 cm), FP64 geometry per pixel and view."""
    import torch

    proj = torch.rand((V, C), dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    npf = torch.empty((N, N), dtype=torch.float32, device="cuda")
    fn = lambda: ctx.lengthproj_dev(proj, npf, 3.0, 0.8)  # noqa: E731
    for _ in range(warmup):
        fn()
    t = timed(fn, steps) / steps
    mask_px = 205012
    return {"workload": "lengthproj_TOMO: 512^2 mask (205,012 pixels) x 800 views, 609 channels",
            "ms_per_slice": t * 1e3, "pixel_views_per_s": mask_px * V / t}


def bench_fbp_transpose(ctx, stream, timed, steps, warmup, dev):
    """The FBP transpose (backprojection gather, transposed filter and
    weight) of an image-space gradient at 512^2 -> 800 x 609."""
    import torch

    u = torch.randn((N, N), dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    out = torch.empty((V, C), dtype=torch.float32, device="cuda")
    fn = lambda: ctx.fbp_transpose_dev(u, out, 1)  # noqa: E731
    for _ in range(warmup):
        fn()
    t = timed(fn, steps) / steps
    stages = stage_medians(ctx, fn, max(warmup, 5))
    peaks = probe_peaks(dev)
    roof = {"stages_ms": stages}
    t_b = stages.get("fbp_backproject_t")
    if t_b:
        upd = float(MASK_PX) * (V // 2 * 2)
        fl = upd * BP_FLOP_PER_UPDATE
        roof.update({"kernel": "fbp_bp_t_scatter_kernel (+ max|u|, transpose, finish)", "bound": "fp32",
                     "achieved": fl / t_b / 1e9, "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                     "frac": fl / t_b / 1e9 / peaks["fp32_tflops"], "updates_per_launch": upd,
                     "updates_per_s": upd / t_b * 1e3, "flop_per_update": BP_FLOP_PER_UPDATE, "launch_ms": t_b})
    return {"workload": "W^T F^T B^T u: 512^2 image-space gradient -> 800 x 609 (Ram-Lak)",
            "ms_per_slice": t * 1e3, "slices_per_s": 1.0 / t, "roofline": roof}


def _batch_inputs(n, seed, kvps_tabs):
    import torch

    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    specs = phantoms.batch_specs(n, seed=seed)
    out = []
    for i, sp in enumerate(specs):
        g = vct.Geometry.with_channels(sp["channels"], views=sp["views"], recon_size=sp["N"], pixel_cm=PIX)
        m = torch.from_numpy(phantoms.ellipse_phantom(sp["seed"], sp["N"])).cuda()
        out.append((sp, g, m, kvps_tabs[sp["kvp"]]))
    return out


def bench_batched(stream, warmup, n=256):
    """The batched configuration: 256 seeded ellipse phantoms of uneven grids
    (256^2/384^2/512^2), kVp 80-140 (1 keV bins), 360-900 views, 512-800
    channels; MBFPA (noise) + Ram-Lak FBP of every slice.  Plain = one slice
    per call on one stream (vct_set_maps_dev + vct_mbfpa_dev + vct_fbp_dev);
    batched = one replay of the captured graph.  The batch's inputs and
    outputs (about 1 GB) exceed L2."""
    import torch

    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    tabs = {k: phantoms.kramers_tables(k) for k in (80, 100, 120, 140)}
    inp = _batch_inputs(n, 0, tabs)
    units = sum(sp["views"] // 2 * 2 * sp["channels"] * len(tab[1]) for sp, _, _, tab in inp)
    jobs, ctxs = [], []
    for i, (sp, g, m, tab) in enumerate(inp):
        jobs.append(vct.Job(g, m, *tab, sino=torch.empty((g.views, g.width), dtype=torch.float32, device="cuda"),
                            img=torch.empty((g.recon_size, g.recon_size), dtype=torch.float32, device="cuda"),
                            filter=1, sigma=SIGMA, seed=i))
        c = vct.Context(g)
        c.set_stream(stream.cuda_stream)
        c.set_spectrum(*tab)
        c.set_maps(m)
        ctxs.append(c)
    torch.cuda.synchronize()

    def plain():
        for c, j in zip(ctxs, jobs):
            c.set_maps(j.maps)
            c.mbfpa_dev(j.sigma, j.seed, j.sino)
            c.fbp_dev(j.sino, j.img, 1)

    t_plain = _event_ms(stream, plain, max(warmup, 3))
    t0 = time.perf_counter()
    b = vct.Batch(jobs, tune=True)
    t_create = time.perf_counter() - t0
    t_batch = _event_ms(stream, lambda: b.run(stream.cuda_stream), max(warmup, 3))
    cfg = b.config()
    b.close()

    # The same slices without the FBP: MBFPA alone, the work the plain
    # single-slice rays*bins/s figure measures.
    mjobs = [vct.Job(j.geometry, j.maps, j.mu, j.pdf, sino=j.sino, sigma=j.sigma, seed=j.seed) for j in jobs]

    def plain_mb():
        for c, j in zip(ctxs, mjobs):
            c.set_maps(j.maps)
            c.mbfpa_dev(j.sigma, j.seed, j.sino)

    t_plain_mb = _event_ms(stream, plain_mb, max(warmup, 3))
    bm = vct.Batch(mjobs, tune=True)
    t_batch_mb = _event_ms(stream, lambda: bm.run(stream.cuda_stream), max(warmup, 3))
    cfg_mb = bm.config()
    bm.close()
    for c in ctxs:
        c.close()
    return {"workload": f"{n} uneven slices: grids 256/384/512, kVp 80-140, 360-900 views, 512-800 channels, "
                        "MBFPA + noise + Ram-Lak FBP",
            "value": units / t_batch * 1e3, "unit": "rays*bins/s", "slices_per_s": n / t_batch * 1e3,
            "ms_per_batch": t_batch, "plain_value": units / t_plain * 1e3, "plain_ms_per_batch": t_plain,
            "speedup_vs_plain": t_plain / t_batch, "rays_bins_per_batch": units, "create_and_tune_s": t_create,
            "tuned": cfg, "l2": "inputs and outputs of one batch exceed L2",
            "mbfpa_only": {"value": units / t_batch_mb * 1e3, "unit": "rays*bins/s", "ms_per_batch": t_batch_mb,
                           "plain_value": units / t_plain_mb * 1e3, "plain_ms_per_batch": t_plain_mb,
                           "speedup_vs_plain": t_plain_mb / t_batch_mb, "tuned": cfg_mb,
                           "what": "the same slices without the FBP (MBFPA: forward, normalisation, noise)"}}


def bench_batched_adjoint(stream, warmup, n=64):
    """Forward + adjoint of 64 uneven slices (the batched generator, seed 1):
    plain = vct_forward_adjoint_dev slice by slice on one stream; batched =
    one replay of an adjoint batch."""
    import torch

    import virtualct_b200 as vct
    from virtualct_b200 import phantoms

    tabs = {k: phantoms.kramers_tables(k) for k in (80, 100, 120, 140)}
    inp = _batch_inputs(n, 1, tabs)
    units = sum(sp["views"] // 2 * 2 * sp["channels"] * len(tab[1]) for sp, _, _, tab in inp)
    jobs, ctxs = [], []
    for i, (sp, g, m, tab) in enumerate(inp):
        c = vct.Context(g)
        c.set_stream(stream.cuda_stream)
        c.set_spectrum(*tab)
        c.set_maps(m)
        meas = torch.empty((g.views, g.width), dtype=torch.float32, device="cuda")
        c.mbfpa_dev(SIGMA, 100 + i, meas)
        at = (m.double() * 0.95).round().to(torch.int16)
        c.set_maps(at)
        grad = torch.empty((6, g.recon_size, g.recon_size), dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        jobs.append(vct.Job(g, at, *tab, meas=meas, grad=grad, loss=loss))
        ctxs.append(c)
    torch.cuda.synchronize()

    def plain():
        for c, j in zip(ctxs, jobs):
            c.set_maps(j.maps)
            c.forward_adjoint_dev(j.meas, j.grad, loss=j.loss)

    t_plain = _event_ms(stream, plain, max(warmup, 3))
    b = vct.Batch(jobs, tune=True)
    t_batch = _event_ms(stream, lambda: b.run(stream.cuda_stream), max(warmup, 3))
    cfg = b.config()
    b.close()
    for c in ctxs:
        c.close()
    return {"workload": f"{n} uneven slices (batched generator, seed 1): loss + dl/drho per slice",
            "value": units / t_batch * 1e3, "unit": "rays*bins/s (forward + adjoint)",
            "slices_per_s": n / t_batch * 1e3, "ms_per_batch": t_batch, "plain_value": units / t_plain * 1e3,
            "plain_ms_per_batch": t_plain, "speedup_vs_plain": t_plain / t_batch, "tuned": cfg}


def bench_scale(stream, slices=64, iters=2):
    """The scale configuration: 1024^2 at 0.05 cm, 8 elements (H C N O P Ca
    Mg Si), 1440 views x 1600 channels, dual energy 80/140 kVp, `slices`
    seeded slices; projected gradient-descent material decomposition, each
    iteration the loss + gradient of every (slice, spectrum) pair in one
    adjoint batch (path lengths recomputed by the walk) and a descent step per
    slice.  Measured sinograms: the noisy MBFPA of each phantom; start: 0.9 x
    the phantom.  One untimed first evaluation, then `iters` iterations, each
    timed by CUDA events (the per-iteration host read of the losses is
    inside); the line reports their median."""
    import torch

    import virtualct_b200 as vct
    from virtualct_b200 import phantoms
    from virtualct_b200.decomposition import Decomposition, rays_bins_per_iteration

    el = phantoms.ELEMENTS8
    tabs = [phantoms.kramers_tables(k, el) for k in (80, 140)]
    geo = vct.Geometry.with_channels(1600, views=1440, recon_size=1024, pixel_cm=0.05)
    t0 = time.perf_counter()
    meas, rho0 = [], []
    with vct.Context(geo) as ctx:
        for s in range(slices):
            m = phantoms.ellipse_phantom(1000 + s, 1024, elements=el)
            ctx.set_maps(m)
            per = []
            for e, tab in enumerate(tabs):
                ctx.set_spectrum(*tab)
                out = torch.empty((geo.views, geo.width), dtype=torch.float32, device="cuda")
                ctx.mbfpa_dev(SIGMA, 2 * s + e, out)
                per.append(out)
            meas.append(per)
            rho0.append(torch.from_numpy(m.astype(np.float32) / 1000.0 * 0.9))
        ctx.synchronize()
    rho = torch.stack(rho0).cuda()
    dec = Decomposition(geo, tabs, meas, rho)
    dec.iterate(1)
    setup_s = time.perf_counter() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    each = []
    for _ in range(iters):
        torch.cuda.synchronize()
        e0.record()
        dec.iterate(1)
        e1.record()
        torch.cuda.synchronize()
        each.append(e0.elapsed_time(e1))
    # median: an iteration launches many small per-slice steps from the host,
    # so a busy host core can stretch one of them
    t = float(np.median(each))
    units = rays_bins_per_iteration(geo, tabs, slices)
    line = {"workload": f"{slices} slices, 1024^2 at 0.05 cm, 8 elements, 1440 views x 1600 channels, 80/140 kVp; "
                        "projected gradient descent, loss + gradient of every slice and spectrum per iteration",
            "ms_per_iteration": t, "value": units / t * 1e3, "unit": "rays*bins/s (forward + adjoint)",
            "iterations_timed": iters, "ms_each": each, "statistic": "median of the timed iterations", "projected_50_iterations_s": 50 * t / 1e3,
            "loss_first": dec.history[0], "loss_last": dec.history[-1], "accepted": dec.accepted,
            "rejected": dec.rejected, "unchanged": dec.unchanged,
            "step_rule": "SQS-diagonal-scaled projected gradient, adaptive Barzilai-Borwein steps, Armijo test",
            "setup_s": setup_s}
    dec.close()
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
        return {"value": V * C * 2 / secs, "unit": "rays*bins/s", "cores": cores, "cpu_model": cpu_model(),
                "kind": "reference", "sample": "reprojection_TOMO for 2 energy bins x 800 views x 609 channels",
                "seconds": secs}
    g = O.geom()
    t0 = time.perf_counter()
    O.forward_exact(g, c, s, rho, np.ascontiguousarray(mu[:, 50:52]), pdf[50:52].copy(), nthreads=cores)
    secs = time.perf_counter() - t0
    return {"value": V * C * 2 / secs, "unit": "rays*bins/s", "cores": cores, "cpu_model": cpu_model(), "kind": "port",
            "sample": "oracle forward (reference order) for 2 energy bins x 800 views x 609 channels",
            "seconds": secs}


# ----------------------------------------------------------- reference arm
def run_reference(args, rank):
    """The reference's own CPU code on the host cores, for this arm's config:
    reprojection_TOMO (MB/reprojection_TOMO.cpp:13, compiled from its sources
    into oracle/_ref/libvct_ref_mb.so with its own OpenMP) with the reference's
    own attenuation_coefficient (MB/prior_weight_production.cpp:180) for mu and
    pdf, and filterSinogram + reconstructImage as shipped (single thread).  The
    phantom comes from phantoms.py loaded on its own: nothing of the product
    library is loaded in this process."""
    if rank != 0:
        return None
    import oracle as O

    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent at build time)"}
    cores = os.cpu_count() or 1
    pdf, mu = O.ref_attenuation(SPECTRUM)
    maps = phantoms_module().ellipse_phantom(0, N)
    NE = len(pdf)
    rho = O.rho_from_maps(maps)
    c, s = O.trig_tables(V)

    # One step = one reprojection_TOMO call: one energy bin over the whole
    # 800 x 609 sinogram (the reference walks every ray once per bin,
    # MB/main.cpp:492-506), cycling through the bins; a slice is NE steps.
    def ref_step(k):
        ke = (50 + k) % NE
        _, secs = O.ref_reprojection(N, PIX, rho, V, C, c, s, 1, mu, pdf, ke0=ke, ke1=ke + 1, threads=cores)
        return secs

    for w in range(max(args.warmup, 1)):
        ref_step(w)
    total = sum(ref_step(k) for k in range(args.steps))
    value = V * C * args.steps / total
    # FBP as shipped: single-threaded filterSinogram + reconstructImage, once.
    full, _ = O.ref_reprojection(N, PIX, rho, V, C, c, s, 1, mu, pdf, ke0=0, ke1=1, threads=cores)
    sino = (full / full.max()).astype(np.float32)
    _, _, tf, tb = O.ref_fbp(1, sino, N, PIX, 1, c, s)
    sample = f"reprojection_TOMO, one energy bin x {V} views x {C} channels per step ({NE} steps per slice)"
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "rays*bins/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3,
        "ms_per_slice_all_bins": total / args.steps * NE * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 walk, f32 densities (reference CPU code)",
        "data": "synthetic: seeded ellipse phantom (seed 0), 120 kVp Kramers spectrum",
        "config": {"workload": CONFIG_NAME, "views": V, "channels": C, "grid": N, "elements": 6, "energy_bins": NE},
        "fbp": {"metric": "FBP slices/s", "value": 1.0 / (tf + tb), "unit": "slices/s",
                "filter_s": tf, "backprojection_s": tb, "threads": 1},
        "cpu_baseline": {"value": value, "unit": "rays*bins/s", "cores": cores, "cpu_model": cpu_model(),
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "rays*bins/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the adjoint and batched lines")
    ap.add_argument("--batch-slices", type=int, default=256,
                    help="slices of the batched line (the batched adjoint line takes a quarter)")
    ap.add_argument("--extras", default="c2,adjoint,lengthproj,fbp_transpose,batched,batched_adjoint,scale",
                    help="comma list of extra lines (1 GPU): c2, adjoint, lengthproj, fbp_transpose, batched, "
                         "batched_adjoint, scale")
    ap.add_argument("--scale-slices", type=int, default=64, help="slices of the scale line")
    ap.add_argument("--scale-iters", type=int, default=3,
                    help="timed descent iterations of the scale line (the configuration runs 50)")
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
