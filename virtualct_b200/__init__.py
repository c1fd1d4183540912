"""virtualct_b200 -- B200-native MBFPA forward projection and fan-beam FBP.

Python view of the C ABI in ``include/vct.h`` (``lib/libvct.so``).  All compute
runs in the CUDA kernels of ``csrc/``; there is no CPU fallback: if the library
is missing, importing the bindings raises.

    import virtualct_b200 as vct
    g = vct.Geometry()                       # physParamsTOMO.h defaults, 800 x 609, 512^2
    mu, pdf = vct.attenuation_coefficient("PhaseSpace_photon_120kV_0cm.txt")
    with vct.Context(g) as ctx:
        ctx.set_maps(maps_int16)             # [M][N][N], density x 1000
        ctx.set_spectrum(mu, pdf)
        sino = ctx.mbfpa(sigma=5.37e-5, seed=1)   # MB/main.cpp:492-530
        img = ctx.fbp(sino, filter=2)        # FBP/main.cpp:137-167
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, fields

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# VCT_LIB=bounds loads the index-checked build (lib/libvct_bounds.so).
LIB_PATH = os.path.join(PKG, "lib", "libvct_bounds.so" if os.environ.get("VCT_LIB") == "bounds" else "libvct.so")

VCT_OK = 0
VCT_E_ARG = -1
VCT_E_CUDA = -2
VCT_E_TIMEOUT = -3
VCT_E_NOMEM = -4
VCT_E_IO = -5
VCT_E_STATE = -6
VCT_E_UNSUPPORTED = -7
VCT_E_RANGE = -8
SUM_COMPENSATED = 0
SUM_REFERENCE = 1
WALK_FAST = 0
WALK_EXACT = 1
MAX_BINS = 1024

ELEMENT_Z = {"H": 1, "C": 6, "N": 7, "O": 8, "P": 15, "Ca": 20, "Mg": 12, "Si": 14}
HUMAN_ELEMENTS = ("H", "C", "N", "O", "P", "Ca")
GAMMEX_ELEMENTS = ("H", "C", "N", "O", "P", "Ca", "Mg", "Si")

# Every entry point include/vct.h and include/vct_io.h declare.
EXPORTED_SYMBOLS = (
    "vct_geometry_default", "vct_strerror", "vct_last_error", "vct_create", "vct_destroy", "vct_set_stream",
    "vct_synchronize", "vct_attenuation_coefficient", "vct_set_maps", "vct_set_maps_dev", "vct_set_spectrum",
    "vct_set_sum_mode", "vct_set_walk_mode", "vct_forward", "vct_forward_dev", "vct_line_integrals_dev", "vct_mbfpa", "vct_mbfpa_dev",
    "vct_normalize_noise_dev", "vct_mbfpa_many", "vct_forward_views_dev", "vct_normalize_noise_rows_dev",
    "vct_fbp_band_count", "vct_fbp_band_dev", "vct_fbp", "vct_fbp_dev", "vct_fbp_noalloc", "vct_fbp_filtered_dev",
    "vct_fbp_transpose", "vct_fbp_transpose_dev",
    "vct_set_density_scale", "vct_descent_step_dev", "vct_descent_step_scaled_dev", "vct_lengthproj", "vct_lengthproj_dev",
    "vct_beam_hardening", "vct_beam_hardening_dev", "vct_set_beam_hardening",
    "vct_lengthproj2", "vct_lengthproj2_dev", "vct_ir_update_dev", "vct_squdiff_dev", "vct_ir_step",
    "vct_forward_adjoint", "vct_forward_adjoint_dev", "vct_forward_vjp_dev", "vct_adjoint_rays_dev",
    "vct_batch_create", "vct_batch_run", "vct_batch_synchronize", "vct_batch_config", "vct_batch_destroy",
    "vct_forward_batched",
    "vct_last_segment_count", "vct_set_stage_timing", "vct_stage_times",
    "vct_kernel_launches", "vct_bounds_violations", "vct_version", "vct_philox4x32_10",
    "vct_load_mb_config", "vct_load_fbp_config", "vct_mb_geometry", "vct_fbp_geometry", "vct_read_raw",
    "vct_write_raw", "vct_raw_layout_default", "vct_load_measured", "vct_load_measured_dev",
    "vct_helical_sinogram", "vct_helical_sinogram_dev",
)


class VctError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {msg} (code {code})")
        self.code = code


class MbConfig(C.Structure):
    """vct_mb_config: the MBFPA input txt's fields (include/vct_io.h)."""
    _fields_ = [
        ("in_pr_class", C.c_char * 16), ("prior_image_onoff", C.c_int), ("proj_width", C.c_int),
        ("proj_height", C.c_int), ("proj_data_type", C.c_char * 16), ("proj_file_offset", C.c_int),
        ("proj_file", C.c_char * 256), ("air_scan_file", C.c_char * 256), ("gantry_rotation_period", C.c_double),
        ("data_sampling_rate", C.c_double), ("data_sampling_rate_orig", C.c_double),
        ("start_view_angle", C.c_double), ("couch_speed", C.c_double), ("start_couch_position", C.c_double),
        ("recon_size", C.c_int), ("recon_pix_size", C.c_double), ("recon_tgt_class", C.c_char * 16),
        ("recon_offset", C.c_double), ("recon_step", C.c_double), ("recon_slices", C.c_int), ("xfactor", C.c_int),
        ("recon_data_file", C.c_char * 256), ("fbp_slice", C.c_int), ("x_reg", C.c_double), ("y_reg", C.c_double),
        ("z_reg", C.c_double), ("scan_list_z", C.c_double), ("osemset", C.c_int), ("total_variation", C.c_double),
        ("prior_const", C.c_double), ("markov_const", C.c_double), ("gradient_decent_const", C.c_double),
        ("num_ite", C.c_int), ("sino_fact", C.c_int), ("spectrum_file", C.c_char * 256),
        ("photon_noise", C.c_double), ("total_proj_number", C.c_int),
    ]

    @classmethod
    def load(cls, path: str) -> "MbConfig":
        cfg = cls()
        _check(lib().vct_load_mb_config(str(path).encode(), C.byref(cfg)), "vct_load_mb_config")
        return cfg


class RawLayout(C.Structure):
    """vct_raw_layout: the raw detector layout of a measured sinogram."""
    _fields_ = [("raw_channels", C.c_int), ("skip_channels", C.c_int), ("air_rows", C.c_int),
                ("air_blocks", C.c_int), ("start_channel", C.c_int), ("end_channel", C.c_int)]

    @classmethod
    def default(cls, **kw) -> "RawLayout":
        lay = cls()
        lib().vct_raw_layout_default(C.byref(lay))
        for k, v in kw.items():
            setattr(lay, k, v)
        return lay


class _CGeometry(C.Structure):
    _fields_ = [
        ("sid_cm", C.c_double), ("det_radius_cm", C.c_double), ("det_src_iso_cm", C.c_double),
        ("start_channel", C.c_int), ("end_channel", C.c_int), ("iso_channel", C.c_double),
        ("max_alpha", C.c_double), ("max_beta", C.c_double), ("views", C.c_int), ("width", C.c_int),
        ("start_view_deg", C.c_double), ("recon_size", C.c_int), ("pixel_cm", C.c_double), ("xfactor", C.c_int),
    ]


class _CJob(C.Structure):
    _fields_ = [
        ("geo", _CGeometry), ("d_maps", C.c_void_p), ("mu", C.c_void_p), ("pdf", C.c_void_p), ("NE", C.c_int),
        ("sigma", C.c_double), ("seed", C.c_uint64), ("d_sino", C.c_void_p), ("d_img", C.c_void_p),
        ("filter", C.c_int), ("d_meas", C.c_void_p), ("d_weights", C.c_void_p), ("d_grad", C.c_void_p),
        ("d_loss", C.c_void_p), ("density_units", C.c_double),
    ]


@dataclass
class Geometry:
    """Runtime form of physParamsTOMO.h plus the txt fields of the hot path."""

    sid_cm: float = 85.0
    det_radius_cm: float = 142.6
    det_src_iso_cm: float = 85.0
    start_channel: int = 0
    end_channel: int = 609
    iso_channel: float = 304.5
    max_alpha: float = 0.326086956
    max_beta: float = 0.326086956
    views: int = 800
    width: int = 609
    start_view_deg: float = 0.0
    recon_size: int = 512
    pixel_cm: float = 0.1
    xfactor: int = 1

    @classmethod
    def with_channels(cls, channels: int, **kw) -> "Geometry":
        """Geometry with ``channels`` detector channels; the iso-channel follows
        the reference's convention (End_Channel/2.0, 304.5 for 609)."""
        return cls(end_channel=channels, width=channels, iso_channel=channels / 2.0, **kw)

    @property
    def channels(self) -> int:
        return self.end_channel - self.start_channel

    def to_c(self) -> _CGeometry:
        c = _CGeometry()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c


_lib = None


def lib():
    """The loaded libvct.so.  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libvct.so not built ({LIB_PATH}); run `python -m virtualct_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.vct_strerror.restype = C.c_char_p
    L.vct_strerror.argtypes = [C.c_int]
    L.vct_last_error.restype = C.c_char_p
    L.vct_geometry_default.argtypes = [C.POINTER(_CGeometry)]
    L.vct_create.argtypes = [C.POINTER(_CGeometry), C.c_int, C.POINTER(vp)]
    L.vct_destroy.argtypes = [vp]
    L.vct_destroy.restype = None
    L.vct_set_stream.argtypes = [vp, vp]
    L.vct_synchronize.argtypes = [vp]
    L.vct_attenuation_coefficient.argtypes = [C.c_char_p, C.c_int, vp, C.c_int, vp, vp, C.POINTER(C.c_int)]
    L.vct_set_maps.argtypes = [vp, vp, C.c_int]
    L.vct_set_maps_dev.argtypes = [vp, vp, C.c_int]
    L.vct_set_spectrum.argtypes = [vp, vp, vp, C.c_int, C.c_int]
    L.vct_set_sum_mode.argtypes = [vp, C.c_int]
    L.vct_set_walk_mode.argtypes = [vp, C.c_int]
    L.vct_forward.argtypes = [vp, vp]
    L.vct_forward_dev.argtypes = [vp, vp]
    L.vct_line_integrals_dev.argtypes = [vp, vp]
    L.vct_mbfpa.argtypes = [vp, C.c_double, C.c_uint64, vp, vp]
    L.vct_mbfpa_dev.argtypes = [vp, C.c_double, C.c_uint64, vp]
    L.vct_normalize_noise_dev.argtypes = [vp, vp, C.c_double, C.c_uint64]
    L.vct_fbp.argtypes = [vp, vp, C.c_int, C.c_int, vp]
    L.vct_fbp_dev.argtypes = [vp, vp, C.c_int, C.c_int, vp]
    L.vct_fbp_filtered_dev.argtypes = [vp, C.POINTER(vp)]
    L.vct_fbp_transpose.argtypes = [vp, vp, C.c_int, vp]
    L.vct_fbp_transpose_dev.argtypes = [vp, vp, C.c_int, vp]
    L.vct_fbp_noalloc.argtypes = [C.POINTER(_CGeometry), vp, C.c_int, C.c_int, vp, vp]
    L.vct_set_density_scale.argtypes = [vp, C.c_double]
    L.vct_lengthproj.argtypes = [vp, vp, C.c_double, C.c_double, vp]
    L.vct_beam_hardening.argtypes = [vp, vp, C.c_double, C.c_double, vp]
    L.vct_lengthproj2.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, vp]
    L.vct_lengthproj2_dev.argtypes = [vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, vp]
    L.vct_ir_update_dev.argtypes = [vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, vp]
    L.vct_squdiff_dev.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, vp]
    L.vct_ir_step.argtypes = [vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double,
                              C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), vp]
    L.vct_beam_hardening_dev.argtypes = [vp, vp, C.c_double, C.c_double]
    L.vct_set_beam_hardening.argtypes = [vp, C.c_double, C.c_double]
    L.vct_lengthproj_dev.argtypes = [vp, vp, C.c_double, C.c_double, vp]
    L.vct_descent_step_dev.argtypes = [vp, vp, vp, C.c_double, C.c_double, vp, C.c_longlong, vp]
    L.vct_descent_step_scaled_dev.argtypes = [vp, vp, vp, C.c_longlong, C.c_double, C.c_double, vp, C.c_longlong,
                                              vp]
    L.vct_forward_adjoint.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_double)]
    L.vct_forward_adjoint_dev.argtypes = [vp, vp, vp, vp, vp]
    L.vct_forward_vjp_dev.argtypes = [vp, vp, vp]
    L.vct_adjoint_rays_dev.argtypes = [vp, vp, vp]
    L.vct_batch_create.argtypes = [C.POINTER(_CJob), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(vp)]
    L.vct_batch_run.argtypes = [vp, vp]
    L.vct_batch_synchronize.argtypes = [vp]
    L.vct_batch_config.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]
    L.vct_batch_destroy.argtypes = [vp]
    L.vct_batch_destroy.restype = None
    L.vct_forward_batched.argtypes = [C.POINTER(_CJob), C.c_int, C.c_int, C.c_int]
    L.vct_last_segment_count.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.vct_set_stage_timing.argtypes = [vp, C.c_int]
    L.vct_stage_times.argtypes = [vp, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_float), C.POINTER(C.c_int)]
    L.vct_kernel_launches.argtypes = [vp]
    L.vct_kernel_launches.restype = C.c_longlong
    L.vct_philox4x32_10.argtypes = [vp, vp, vp]
    L.vct_philox4x32_10.restype = None
    L.vct_mbfpa_many.argtypes = [vp, C.c_int, vp, C.c_int, C.c_double, C.c_uint64, vp, vp]
    L.vct_forward_views_dev.argtypes = [vp, C.c_int, C.c_int, vp, vp]
    L.vct_normalize_noise_rows_dev.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_double, C.c_uint64]
    L.vct_fbp_band_count.argtypes = [vp, C.POINTER(C.c_int)]
    L.vct_fbp_band_dev.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp]
    L.vct_bounds_violations.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_int)]
    L.vct_load_mb_config.argtypes = [C.c_char_p, vp]
    L.vct_raw_layout_default.argtypes = [vp]
    L.vct_raw_layout_default.restype = None
    L.vct_load_measured.argtypes = [vp, vp, C.c_int, vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.vct_load_measured_dev.argtypes = [vp, vp, vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp]
    L.vct_helical_sinogram.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, C.c_int]
    L.vct_helical_sinogram_dev.argtypes = [vp, C.c_int, C.c_int, C.c_int, vp, vp]
    _lib = L
    return L


def _check(rc: int, where: str) -> None:
    if rc != VCT_OK:
        msg = lib().vct_last_error().decode(errors="replace")
        raise VctError(rc, where, msg)


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def attenuation_coefficient(spectrum_path, elements=HUMAN_ELEMENTS, nthin: int = 1):
    """Spectrum pdf [NE] and mass attenuation mu [M][NE] (cm^2/g), bit-identical
    to MB/prior_weight_production.cpp:180-297 for the same elements."""
    Z = np.array([ELEMENT_Z[e] for e in elements], np.int32)
    mu = np.zeros(len(Z) * MAX_BINS, np.float32)
    pdf = np.zeros(MAX_BINS, np.float32)
    ne = C.c_int(0)
    _check(lib().vct_attenuation_coefficient(str(spectrum_path).encode(), nthin, _ptr(Z), len(Z), _ptr(mu),
                                             _ptr(pdf), C.byref(ne)), "vct_attenuation_coefficient")
    n = ne.value
    return mu[: len(Z) * n].reshape(len(Z), n).copy(), pdf[:n].copy()


def philox4x32_10(ctr, key):
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().vct_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


class Context:
    """One device context (vct_ctx): geometry tables, maps, spectrum and
    scratch buffers live on the GPU between calls."""

    def __init__(self, geometry: Geometry | None = None, device: int = 0):
        self.geometry = geometry or Geometry()
        self._g = self.geometry.to_c()
        self._h = C.c_void_p()
        _check(lib().vct_create(C.byref(self._g), device, C.byref(self._h)), "vct_create")
        self.device = device
        self._M = 0

    # lifetime ---------------------------------------------------------------
    def close(self) -> None:
        if self._h:
            lib().vct_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(lib().vct_set_stream(self._h, stream_ptr or None), "vct_set_stream")

    def synchronize(self) -> None:
        _check(lib().vct_synchronize(self._h), "vct_synchronize")

    @property
    def kernel_launches(self) -> int:
        return int(lib().vct_kernel_launches(self._h))

    def set_stage_timing(self, on: bool = True) -> None:
        """Record CUDA events around every kernel stage of later calls."""
        _check(lib().vct_set_stage_timing(self._h, 1 if on else 0), "vct_set_stage_timing")

    def stage_times(self) -> list:
        """[(stage name, ms)] of the last timed call (waits for it)."""
        cap = 16
        names = (C.c_char_p * cap)()
        ms = (C.c_float * cap)()
        n = C.c_int(0)
        _check(lib().vct_stage_times(self._h, cap, names, ms, C.byref(n)), "vct_stage_times")
        return [(names[i].decode(), float(ms[i])) for i in range(min(n.value, cap))]

    @property
    def last_segment_count(self) -> int:
        n = C.c_longlong(0)
        _check(lib().vct_last_segment_count(self._h, C.byref(n)), "vct_last_segment_count")
        return n.value

    # MBFPA -------------------------------------------------------------------
    def set_maps(self, maps) -> None:
        """maps: int16 [M][N][N] (element density x 1000), host array or a CUDA
        tensor (anything with ``data_ptr()`` is taken as a device pointer)."""
        if hasattr(maps, "data_ptr"):
            M = int(maps.shape[0])
            _check(lib().vct_set_maps_dev(self._h, maps.data_ptr(), M), "vct_set_maps_dev")
            self._M = M
            return
        a = np.ascontiguousarray(maps, np.int16)
        N = self.geometry.recon_size
        if a.ndim != 3 or a.shape[1:] != (N, N):
            raise ValueError(f"maps must be [M][{N}][{N}] int16, got {a.shape}")
        _check(lib().vct_set_maps(self._h, _ptr(a), a.shape[0]), "vct_set_maps")
        self._M = a.shape[0]

    def set_density_scale(self, units_per_gcc: float) -> None:
        """Map units per g/cm^3 (default 1000)."""
        _check(lib().vct_set_density_scale(self._h, float(units_per_gcc)), "vct_set_density_scale")

    def set_spectrum(self, mu, pdf) -> None:
        mu = np.ascontiguousarray(mu, np.float32)
        pdf = np.ascontiguousarray(pdf, np.float32)
        M, NE = mu.shape
        if pdf.shape != (NE,):
            raise ValueError("pdf must have NE entries")
        _check(lib().vct_set_spectrum(self._h, _ptr(mu), _ptr(pdf), M, NE), "vct_set_spectrum")

    def set_sum_mode(self, mode: int) -> None:
        _check(lib().vct_set_sum_mode(self._h, mode), "vct_set_sum_mode")

    def set_walk_mode(self, mode: int) -> None:
        _check(lib().vct_set_walk_mode(self._h, mode), "vct_set_walk_mode")

    def _sino(self) -> np.ndarray:
        return np.zeros((self.geometry.views, self.geometry.width), np.float32)

    def forward(self) -> np.ndarray:
        """Un-normalised polyenergetic sinogram [views][width]."""
        out = self._sino()
        _check(lib().vct_forward(self._h, _ptr(out)), "vct_forward")
        return out

    def forward_dev(self, out) -> None:
        _check(lib().vct_forward_dev(self._h, out.data_ptr()), "vct_forward_dev")

    def line_integrals_dev(self, out) -> None:
        _check(lib().vct_line_integrals_dev(self._h, out.data_ptr()), "vct_line_integrals_dev")

    def mbfpa(self, sigma: float = 0.0, seed: int = 1, return_stats: bool = False):
        """MB/main.cpp:492-530: forward, max-normalise, Gaussian noise."""
        out = self._sino()
        st = np.zeros(3, np.float32)
        _check(lib().vct_mbfpa(self._h, float(sigma), int(seed), _ptr(out), _ptr(st)), "vct_mbfpa")
        return (out, st) if return_stats else out

    def mbfpa_many(self, maps, sigma: float = 0.0, seed: int = 1, out=None, return_stats: bool = False):
        """vct_mbfpa_many: a list of host int16 [M][N][N] arrays (pinned ones,
        e.g. torch pin_memory().numpy(), overlap the copies); returns the
        [n][views][width] sinograms (or writes the given list of arrays)."""
        g = self.geometry
        arrs = [np.ascontiguousarray(m, np.int16) for m in maps]
        n = len(arrs)
        if out is None:
            out = [np.empty((g.views, g.width), np.float32) for _ in range(n)]
        if len(out) != n or any(o.dtype != np.float32 or o.size != g.views * g.width or not o.flags.c_contiguous
                                for o in out):
            raise ValueError("out must hold n contiguous float32 [views][width] arrays")
        M = arrs[0].shape[0] if n else self._M or 1
        pin = (C.c_void_p * max(n, 1))(*[a.ctypes.data for a in arrs])
        pout = (C.c_void_p * max(n, 1))(*[o.ctypes.data for o in out])
        st = np.zeros((max(n, 1), 3), np.float32)
        _check(lib().vct_mbfpa_many(self._h, n, pin, M, float(sigma), int(seed), pout,
                                    _ptr(st) if return_stats else None), "vct_mbfpa_many")
        if n:
            self._M = M
        return (out, st[:n]) if return_stats else out

    # one slice over several ranks (virtualct_b200.sharded)
    def forward_views_dev(self, v0: int, v1: int, out, maxmin) -> None:
        _check(lib().vct_forward_views_dev(self._h, int(v0), int(v1), out.data_ptr(), maxmin.data_ptr()),
               "vct_forward_views_dev")

    def normalize_noise_rows_dev(self, sino, r0: int, r1: int, maxmin, sigma: float, seed: int) -> None:
        _check(lib().vct_normalize_noise_rows_dev(self._h, sino.data_ptr(), int(r0), int(r1), maxmin.data_ptr(),
                                                  float(sigma), int(seed)), "vct_normalize_noise_rows_dev")

    def fbp_band_count(self) -> int:
        n = C.c_int(0)
        _check(lib().vct_fbp_band_count(self._h, C.byref(n)), "vct_fbp_band_count")
        return n.value

    def fbp_band_dev(self, sino, b0: int, b1: int, img, filter: int = 1, in_mode: bool = False) -> None:
        _check(lib().vct_fbp_band_dev(self._h, sino.data_ptr(), filter, int(in_mode), int(b0), int(b1),
                                      img.data_ptr()), "vct_fbp_band_dev")

    def mbfpa_dev(self, sigma: float, seed: int, out) -> None:
        _check(lib().vct_mbfpa_dev(self._h, float(sigma), int(seed), out.data_ptr()), "vct_mbfpa_dev")

    def normalize_noise_dev(self, sino, sigma: float, seed: int) -> None:
        _check(lib().vct_normalize_noise_dev(self._h, sino.data_ptr(), float(sigma), int(seed)),
               "vct_normalize_noise_dev")

    def beam_hardening(self, sino, alpha: float, beta: float) -> np.ndarray:
        """Beam-hardening correction of a [views][width] transmission sinogram."""
        s = np.ascontiguousarray(sino, np.float32)
        if s.shape != (self.geometry.views, self.geometry.width):
            raise ValueError("sinogram must be [views][width]")
        out = np.empty_like(s)
        _check(lib().vct_beam_hardening(self._h, _ptr(s), float(alpha), float(beta), _ptr(out)), "vct_beam_hardening")
        return out

    def beam_hardening_dev(self, sino, alpha: float, beta: float) -> None:
        _check(lib().vct_beam_hardening_dev(self._h, sino.data_ptr(), float(alpha), float(beta)),
               "vct_beam_hardening_dev")

    def set_beam_hardening(self, alpha: float, beta: float) -> None:
        """Apply the correction inside every later FBP (alpha 0: off)."""
        _check(lib().vct_set_beam_hardening(self._h, float(alpha), float(beta)), "vct_set_beam_hardening")

    def lengthproj(self, proj, z: float = 0.0, couch_speed: float = 0.0) -> np.ndarray:
        """lengthproj_TOMO: npf [N][N] from proj [views/2*2][width]."""
        g = self.geometry
        p = np.ascontiguousarray(proj, np.float32)
        if p.shape != (g.views // 2 * 2, g.width):
            raise ValueError(f"proj must be [{g.views // 2 * 2}][{g.width}]")
        out = np.zeros((g.recon_size, g.recon_size), np.float32)
        _check(lib().vct_lengthproj(self._h, _ptr(p), float(z), float(couch_speed), _ptr(out)), "vct_lengthproj")
        return out

    def lengthproj2(self, proj, ite: int, thinout: int, z: float = 0.0, couch_speed: float = 0.0) -> np.ndarray:
        """lengthproj_TOMO_2 of the iterative step: npf [N][N]."""
        g = self.geometry
        p = np.ascontiguousarray(proj, np.float32)
        out = np.zeros((g.recon_size, g.recon_size), np.float32)
        _check(lib().vct_lengthproj2(self._h, _ptr(p), float(z), float(couch_speed), int(ite), int(thinout), _ptr(out)),
               "vct_lengthproj2")
        return out

    def ir_update_dev(self, before, npf, npf_re, after, wbefore, w_tv, w_prior=0.0, ite=1, thinout=1,
                      prior=None) -> None:
        _check(lib().vct_ir_update_dev(self._h, before.data_ptr(), _dp(prior), npf.data_ptr(), npf_re.data_ptr(),
                                       float(wbefore), float(w_tv), float(w_prior), int(ite), int(thinout),
                                       after.data_ptr()), "vct_ir_update_dev")

    def ir_step(self, proj, npf, before, *, ite=1, thinout=10, num_ite=500, w_tv=1e-4, w_prior=0.0, wbefore=0.0105,
                objective=1e7, z=0.0, couch_speed=0.0, prior=None, after=None):
        """One pass of the reference's iterative step; returns (after, wbefore,
        objective, quadratic)."""
        N = self.geometry.recon_size
        p = np.ascontiguousarray(proj, np.float32)
        out = np.zeros((N, N), np.float32) if after is None else np.array(after, np.float32, copy=True)
        wb, ob, qd = C.c_double(wbefore), C.c_double(objective), C.c_double(0.0)
        pr = None if prior is None else np.ascontiguousarray(prior, np.float32)
        _check(lib().vct_ir_step(self._h, _ptr(p), _ptr(np.ascontiguousarray(npf, np.float32)),
                                 _ptr(np.ascontiguousarray(before, np.float32)), None if pr is None else _ptr(pr),
                                 float(z), float(couch_speed), int(ite), int(thinout), int(num_ite), float(w_tv),
                                 float(w_prior), C.byref(wb), C.byref(ob), C.byref(qd), _ptr(out)), "vct_ir_step")
        return out, wb.value, ob.value, qd.value

    def squdiff_dev(self, proj, reproj, out2, ite: int, thinout: int, num_ite: int) -> None:
        _check(lib().vct_squdiff_dev(self._h, proj.data_ptr(), reproj.data_ptr(), int(ite), int(thinout), int(num_ite),
                                     out2.data_ptr()), "vct_squdiff_dev")

    def lengthproj_dev(self, proj, npf, z: float = 0.0, couch_speed: float = 0.0) -> None:
        _check(lib().vct_lengthproj_dev(self._h, proj.data_ptr(), float(z), float(couch_speed), npf.data_ptr()),
               "vct_lengthproj_dev")

    # Adjoint -----------------------------------------------------------------
    def forward_adjoint(self, meas, weights=None):
        """Loss 1/2 sum w (ln(y/ynorm) - ln p)^2 and its gradient w.r.t. the
        element densities (g/cm^3), [M][N][N]; meas (and weights) [views][width]."""
        g = self.geometry
        m = np.ascontiguousarray(meas, np.float32)
        if m.shape != (g.views, g.width):
            raise ValueError(f"measured sinogram must be [{g.views}][{g.width}]")
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        grad = np.zeros((self._M, g.recon_size, g.recon_size), np.float32)
        loss = C.c_double()
        _check(lib().vct_forward_adjoint(self._h, _ptr(m), None if w is None else _ptr(w), _ptr(grad),
                                         C.byref(loss)), "vct_forward_adjoint")
        return loss.value, grad

    def forward_adjoint_dev(self, meas, grad, weights=None, loss=None) -> None:
        _check(lib().vct_forward_adjoint_dev(self._h, meas.data_ptr(), None if weights is None else weights.data_ptr(),
                                             grad.data_ptr(), None if loss is None else loss.data_ptr()),
               "vct_forward_adjoint_dev")

    def forward_vjp_dev(self, dy, grad) -> None:
        _check(lib().vct_forward_vjp_dev(self._h, dy.data_ptr(), grad.data_ptr()), "vct_forward_vjp_dev")

    def adjoint_rays_dev(self, g, out) -> None:
        _check(lib().vct_adjoint_rays_dev(self._h, g.data_ptr(), out.data_ptr()), "vct_adjoint_rays_dev")

    # FBP ---------------------------------------------------------------------
    def fbp(self, sino, filter: int = 1, in_mode: bool = False) -> np.ndarray:
        s = np.ascontiguousarray(sino, np.float32)
        if s.shape != (self.geometry.views, self.geometry.width):
            raise ValueError(f"sinogram must be [{self.geometry.views}][{self.geometry.width}]")
        N = self.geometry.recon_size
        img = np.zeros((N, N), np.float32)
        _check(lib().vct_fbp(self._h, _ptr(s), filter, int(in_mode), _ptr(img)), "vct_fbp")
        return img

    def fbp_dev(self, sino, img, filter: int = 1, in_mode: bool = False) -> None:
        _check(lib().vct_fbp_dev(self._h, sino.data_ptr(), filter, int(in_mode), img.data_ptr()), "vct_fbp_dev")

    def fbp_transpose(self, u, filter: int = 1) -> np.ndarray:
        """W^T F^T B^T u: the transpose of the FBP (in_mode 0) as a map from
        lam = -ln p [views][width] to the image, applied to u [N][N]."""
        N = self.geometry.recon_size
        a = np.ascontiguousarray(u, np.float32)
        if a.shape != (N, N):
            raise ValueError(f"u must be [{N}][{N}]")
        out = self._sino()
        _check(lib().vct_fbp_transpose(self._h, _ptr(a), filter, _ptr(out)), "vct_fbp_transpose")
        return out

    def fbp_transpose_dev(self, u, out, filter: int = 1) -> None:
        _check(lib().vct_fbp_transpose_dev(self._h, u.data_ptr(), filter, out.data_ptr()), "vct_fbp_transpose_dev")

    def fbp_filtered_ptr(self) -> int:
        p = C.c_void_p()
        _check(lib().vct_fbp_filtered_dev(self._h, C.byref(p)), "vct_fbp_filtered_dev")
        return p.value


def _dp(t):
    return None if t is None else t.data_ptr()


class Job:
    """One slice of a Batch.  Device buffers are CUDA tensors (anything with
    ``data_ptr()``); mu [M][NE] and pdf [NE] are host arrays."""

    def __init__(self, geometry: Geometry, maps, mu, pdf, *, sino=None, img=None, filter: int = 1,
                 sigma: float = 0.0, seed: int = 1, meas=None, weights=None, grad=None, loss=None,
                 density_units: float = 0.0):
        self.geometry = geometry
        self.maps, self.sino, self.img, self.meas, self.weights, self.grad, self.loss = (
            maps, sino, img, meas, weights, grad, loss)
        self.mu = np.ascontiguousarray(mu, np.float32)
        self.pdf = np.ascontiguousarray(pdf, np.float32)
        self.filter, self.sigma, self.seed = filter, sigma, seed
        self.density_units = density_units

    def to_c(self) -> _CJob:
        j = _CJob()
        j.geo = self.geometry.to_c()
        j.d_maps = self.maps.data_ptr()
        j.mu = self.mu.ctypes.data
        j.pdf = self.pdf.ctypes.data
        j.NE = int(self.pdf.shape[0])
        j.sigma = float(self.sigma)
        j.seed = int(self.seed)
        j.d_sino, j.d_img, j.filter = _dp(self.sino), _dp(self.img), int(self.filter)
        j.d_meas, j.d_weights, j.d_grad, j.d_loss = _dp(self.meas), _dp(self.weights), _dp(self.grad), _dp(self.loss)
        j.density_units = float(self.density_units)
        return j


class Batch:
    """vct_batch: many slices in one captured CUDA graph (see include/vct.h)."""

    def __init__(self, jobs, M: int = 6, device: int = 0, tune: bool = True):
        self.jobs = list(jobs)  # keeps the buffers alive
        arr = (_CJob * len(self.jobs))(*[j.to_c() for j in self.jobs])
        self._h = C.c_void_p()
        _check(lib().vct_batch_create(arr, len(self.jobs), M, device, int(tune), C.byref(self._h)),
               "vct_batch_create")

    def run(self, stream_ptr: int | None = None) -> None:
        _check(lib().vct_batch_run(self._h, stream_ptr), "vct_batch_run")

    def synchronize(self) -> None:
        _check(lib().vct_batch_synchronize(self._h), "vct_batch_synchronize")

    def config(self) -> dict:
        t, b, v, k = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().vct_batch_config(self._h, C.byref(t), C.byref(b), C.byref(v), C.byref(k)), "vct_batch_config")
        return {"tile_rays": t.value, "blocks_per_sm": b.value, "view_groups": v.value, "kernels_per_run": k.value}

    def close(self) -> None:
        if self._h:
            lib().vct_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bounds_violations() -> tuple[int, int]:
    """(failed index checks since the last call, unit * 100000 + line of one);
    only the index-checked build (VCT_LIB=bounds) has them."""
    h, w = C.c_ulonglong(0), C.c_int(0)
    _check(lib().vct_bounds_violations(C.byref(h), C.byref(w)), "vct_bounds_violations")
    return h.value, w.value


def load_measured(cfg: MbConfig, layout: RawLayout | None = None, device: int = 0):
    """vct_load_measured: (volume [rotations][views][width], mask, rotations,
    max_value).  Raises VctError (code VCT_E_IO for a missing file,
    VCT_E_RANGE for the IN-mode stop)."""
    lay = layout or RawLayout.default()
    shape = (cfg.total_proj_number, cfg.proj_height, cfg.proj_width)
    vol = np.zeros(shape, np.float32)
    mask = np.zeros(shape, np.uint8)
    rot, mx = C.c_int(0), C.c_double(0.0)
    _check(lib().vct_load_measured(C.byref(cfg), C.byref(lay), device, _ptr(vol), _ptr(mask), C.byref(rot),
                                   C.byref(mx)), "vct_load_measured")
    return vol, mask, rot.value, mx.value


def helical_sinogram(volume, device: int = 0, out=None) -> np.ndarray:
    """vct_helical_sinogram: [views][width] from [rotations][views][width]."""
    v = np.ascontiguousarray(volume, np.float32)
    R, V, W = v.shape
    o = np.zeros((V, W), np.float32) if out is None else out
    _check(lib().vct_helical_sinogram(_ptr(v), R, V, W, _ptr(o), device), "vct_helical_sinogram")
    return o


def helical_sinogram_dev(volume, out, stream_ptr: int | None = None) -> None:
    R, V, W = volume.shape
    _check(lib().vct_helical_sinogram_dev(volume.data_ptr(), R, V, W, out.data_ptr(), stream_ptr),
           "vct_helical_sinogram_dev")


def descent_step_scaled_dev(rho, grad, scale, step: float, units: float, maps, stream_ptr: int | None = None) -> None:
    """rho -= step * grad * scale (scale broadcast over leading dimensions),
    clamped at 0; maps = round(rho * units)."""
    if rho.numel() % scale.numel():
        raise ValueError("the scale table must tile rho")
    _check(lib().vct_descent_step_scaled_dev(rho.data_ptr(), grad.data_ptr(), scale.data_ptr(), scale.numel(),
                                             float(step), float(units), maps.data_ptr(), rho.numel(), stream_ptr),
           "vct_descent_step_scaled_dev")


def descent_step_dev(rho, grad_a, grad_b, step: float, units: float, maps, stream_ptr: int | None = None) -> None:
    """rho -= step * (grad_a + grad_b), clamped at 0; maps = round(rho * units)
    (device tensors of the same element count; grad_b may be None)."""
    _check(lib().vct_descent_step_dev(rho.data_ptr(), grad_a.data_ptr(), _dp(grad_b), float(step), float(units),
                                      maps.data_ptr(), rho.numel(), stream_ptr), "vct_descent_step_dev")
