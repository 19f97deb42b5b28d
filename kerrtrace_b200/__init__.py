"""kerrtrace_b200 — B200-native KerrTrace geodesic hot path (Python host binding).

The product is the C-ABI library ``libkerrtrace.so`` (include/kerrtrace.h) built from
``csrc/`` for sm_100a.  This module binds it with ctypes and mirrors the reference's renderer
interface (src/renderer/mod.rs: ``CudaRenderer::{new, submit_render, ready_frame,
finish_frame}``) plus the kernel-level entry points that replace the reference's three launches.
Nothing here computes on the CPU: if the library is missing the import of the binding fails.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libkerrtrace.so"

KT_OK = 0
KT_ERR_INVALID_ARG = 1
KT_ERR_CUDA = 2
KT_ERR_LUT_OVERFLOW = 3
KT_ERR_NOT_READY = 4
KT_ERR_QUEUE_ORDER = 5
KT_ERR_NO_DEVICE = 6
KT_ERR_UNSUPPORTED = 7
KT_ERR_TIMEOUT = 8

MODE_REF, MODE_SPEC = 0, 1
PREC_FP32, PREC_MIXED, PREC_FP64 = 0, 1, 2
SCHED_PLAIN, SCHED_WAVEFRONT, SCHED_AUTO = 0, 1, 2
ORDER_TILES, ORDER_LONG_FIRST = 0, 1
NOALLOC_MAX_VIEWS = 64
BATCH_MAX_JOBS = 64


class KtConfig(C.Structure):
    """Mirror of ``kt_config`` (the reference's config.yaml fields, src/main.rs:15-122)."""

    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("block_dim", C.c_uint32 * 2),
        ("bloom_enabled", C.c_int32), ("bloom_intensity", C.c_float), ("bloom_radius", C.c_float),
        ("lut_size", C.c_uint32), ("lut_max_temp", C.c_float),
        ("wavelength_start", C.c_float), ("wavelength_end", C.c_float), ("wavelength_step", C.c_float),
        ("use_fast_math", C.c_int32),
        ("spp", C.c_uint32), ("exposure_scale", C.c_float),
        ("sky_grid_divisions", C.c_uint32), ("sky_line_thickness", C.c_float), ("sky_intensity", C.c_float),
        ("spin", C.c_float), ("mass", C.c_float),
        ("disk_outer_radius", C.c_float), ("disk_temperature_scale", C.c_float),
        ("initial_step", C.c_float), ("tolerance", C.c_float),
        ("max_steps", C.c_uint32), ("max_attempts", C.c_uint32),
        ("transmittance_cutoff", C.c_float), ("horizon_epsilon", C.c_float), ("escape_radius", C.c_float),
        ("noise_enabled", C.c_int32), ("noise_scale", C.c_float), ("noise_strength", C.c_float),
        ("noise_winding", C.c_float), ("noise_detail", C.c_uint32),
        ("mode", C.c_int32), ("precision", C.c_int32), ("noise_seed", C.c_uint32),
        ("noise_phase", C.c_float), ("bloom_threshold", C.c_float), ("photon_zone_factor", C.c_float),
    ]

    def copy(self) -> "KtConfig":
        c = KtConfig()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(KtConfig))
        return c

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name == "block_dim" else v
        return out


class KtKerrParams(C.Structure):
    """Mirror of ``kt_kerr_params`` / the reference's KerrParams (cuda/kerr_math.cuh:3-9)."""

    _fields_ = [(n, C.c_float) for n in ("a", "m", "aa", "inv_m", "a_norm", "rh", "disk_inner",
                                         "inv_w_2", "inv_h_2", "aspect_ratio", "disk_noise_scale",
                                         "disk_noise_strength", "disk_noise_winding")] + [
        ("disk_noise_enabled", C.c_int32), ("disk_noise_detail", C.c_int32)]


class KtCamera(C.Structure):
    _fields_ = [("cam_pos", C.c_float * 3), ("fwd", C.c_float * 3), ("rgt", C.c_float * 3),
                ("up", C.c_float * 3), ("fov_scale", C.c_float)]


class KtTraceStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("rays", "steps", "attempts", "rhs_evals", "frozen_rays", "fp64_steps")]


class KtTuning(C.Structure):
    """Mirror of ``kt_tuning``: the launch shape that KT_SCHED_AUTO runs."""

    _fields_ = [("schedule", C.c_int32), ("block_x", C.c_int32), ("block_y", C.c_int32),
                ("blocks_per_sm", C.c_int32), ("refill_min", C.c_int32), ("order", C.c_int32),
                ("keep_frozen", C.c_int32)]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


TUNE_MAX_CANDIDATES = 64


class KtTuneEntry(C.Structure):
    """Mirror of ``kt_tune_entry``: one candidate of the autotuner."""

    _fields_ = [("tuning", KtTuning), ("ms", C.c_float), ("identical", C.c_int32)]


class KtDiffParams(C.Structure):
    """Mirror of ``kt_diff_params``: the differentiable parameters theta."""

    _fields_ = [("spin", C.c_double), ("inclination_deg", C.c_double), ("temperature_scale", C.c_double),
                ("disk_outer_radius", C.c_double)]

    def as_list(self) -> list[float]:
        return [self.spin, self.inclination_deg, self.temperature_scale, self.disk_outer_radius]


class KtDiffView(C.Structure):
    """Mirror of ``kt_diff_view``: the fixed part of the differentiable view."""

    _fields_ = [("observer_r", C.c_float), ("azimuth_deg", C.c_float), ("fov_deg", C.c_float),
                ("base_temperature_scale", C.c_float)]


class KtDiffInfo(C.Structure):
    _fields_ = [("segments_used", C.c_uint64), ("segments_capacity", C.c_uint64), ("overflow_rays", C.c_uint64),
                ("record_bytes", C.c_uint64), ("device_bytes", C.c_uint64)]


class KtJob(C.Structure):
    """Mirror of ``kt_job``: one render of a batch."""

    _fields_ = [("cfg", KtConfig), ("cam", KtCamera), ("hdr_out", C.c_void_p), ("err_word", C.c_void_p)]


class KtView(C.Structure):
    """Mirror of ``kt_view``: camera position, yaw / pitch / fov in degrees (src/app.rs)."""

    _fields_ = [("cam_pos", C.c_float * 3), ("yaw_deg", C.c_float), ("pitch_deg", C.c_float),
                ("fov_deg", C.c_float)]


class KtViewState(C.Structure):
    """Mirror of ``kt_view_state``: the last submitted view and whether a frame exists."""

    _fields_ = [("prev", KtView), ("has_frame", C.c_int32)]


class KtError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"kerrtrace status {status}: {message}")
        self.status = status


_lib = None

# (name, restype, argtypes) of every exported entry point of include/kerrtrace.h
SIGNATURES = [
    ("kt_status_str", C.c_char_p, [C.c_int]),
    ("kt_last_error", C.c_char_p, []),
    ("kt_abi_version", C.c_int, []),
    ("kt_config_default", C.c_int, [C.POINTER(KtConfig)]),
    ("kt_build_kerr_params", C.c_int, [C.POINTER(KtConfig), C.POINTER(KtKerrParams)]),
    ("kt_calc_isco", C.c_float, [C.c_float, C.c_int, C.c_float]),
    ("kt_generate_blackbody_lut", C.c_int, [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]),
    ("kt_generate_disk_lut", C.c_int, [C.POINTER(KtKerrParams), C.c_float, C.c_uint32, C.c_void_p]),
    ("kt_build_defines", C.c_int, [C.POINTER(KtConfig), C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    ("kt_validate_bloom", C.c_int, [C.POINTER(KtConfig), C.POINTER(C.c_int32), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    ("kt_camera_basis", C.c_int, [C.c_float, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                  C.POINTER(C.c_float)]),
    ("kt_fov_scale", C.c_float, [C.c_float]),
    ("kt_context_create", C.c_int, [C.POINTER(KtConfig), C.c_int, C.POINTER(C.c_void_p)]),
    ("kt_context_create_with_luts", C.c_int, [C.POINTER(KtConfig), C.c_int, C.c_void_p, C.c_void_p, C.c_uint32,
                                              C.POINTER(C.c_void_p)]),
    ("kt_context_create_device_luts", C.c_int, [C.POINTER(KtConfig), C.c_int, C.POINTER(C.c_void_p)]),
    ("kt_context_destroy", None, [C.c_void_p]),
    ("kt_context_params", C.c_int, [C.c_void_p, C.POINTER(KtKerrParams)]),
    ("kt_trace", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtCamera), C.c_int32, C.c_void_p, C.c_void_p]),
    ("kt_trace_counted", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtCamera), C.c_int32, C.c_void_p, C.c_void_p,
                                   C.POINTER(KtTraceStats), C.c_void_p]),
    ("kt_trace_progressive", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtCamera), C.c_uint32, C.c_uint32,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_context_set_tuning", C.c_int, [C.c_void_p, C.POINTER(KtTuning)]),
    ("kt_context_get_tuning", C.c_int, [C.c_void_p, C.POINTER(KtTuning)]),
    ("kt_renderer_set_tuning", C.c_int, [C.c_void_p, C.POINTER(KtTuning)]),
    ("kt_context_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtCamera), C.c_uint32, C.c_void_p,
                                      C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]),
    ("kt_renderer_autotune", C.c_int, [C.c_void_p, C.POINTER(KtCamera), C.c_uint32]),
    ("kt_bloom_horizontal", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_post_process", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_post_fused", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_trace_noalloc", C.c_int, [C.POINTER(KtConfig), C.POINTER(KtCamera), C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_diff_create", C.c_int, [C.POINTER(KtConfig), C.POINTER(KtDiffView), C.c_uint32, C.c_int,
                                 C.POINTER(C.c_void_p)]),
    ("kt_diff_forward", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtDiffParams), C.c_void_p, C.c_void_p]),
    ("kt_diff_replay", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtDiffParams), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    ("kt_diff_backward", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_diff_backward_fp64", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("kt_diff_replay_fp64", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(KtDiffParams), C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p]),
    ("kt_diff_get_info", C.c_int, [C.c_void_p, C.POINTER(KtDiffInfo)]),
    ("kt_diff_orbit_camera", C.c_int, [C.c_float, C.c_float, C.c_float, C.c_float, C.POINTER(KtCamera),
                                       C.POINTER(KtCamera)]),
    ("kt_diff_destroy", None, [C.c_void_p]),
    ("kt_batch_create", C.c_int, [C.c_void_p, C.c_uint32, C.c_int, C.POINTER(C.c_void_p)]),
    ("kt_batch_set_block", C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    ("kt_batch_set_camera", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(KtCamera)]),
    ("kt_batch_set_tuning", C.c_int, [C.c_void_p, C.POINTER(KtTuning)]),
    ("kt_batch_get_tuning", C.c_int, [C.c_void_p, C.POINTER(KtTuning)]),
    ("kt_batch_autotune", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.POINTER(C.c_uint32)]),
    ("kt_batch_trace", C.c_int, [C.c_void_p, C.c_void_p]),
    ("kt_batch_trace_graph", C.c_int, [C.c_void_p, C.c_void_p]),
    ("kt_batch_trace_sequential", C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    ("kt_batch_rays", C.c_uint64, [C.c_void_p]),
    ("kt_batch_destroy", None, [C.c_void_p]),
    ("kt_renderer_new", C.c_int, [C.POINTER(KtConfig), C.c_int, C.POINTER(C.c_void_p)]),
    ("kt_renderer_submit_render", C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                            C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                            C.POINTER(C.c_int32)]),
    ("kt_renderer_ready_frame", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.POINTER(C.c_uint32)),
                                          C.POINTER(C.c_float)]),
    ("kt_renderer_finish_frame", C.c_int, [C.c_void_p, C.c_uint32]),
    ("kt_renderer_wait", C.c_int, [C.c_void_p]),
    ("kt_renderer_set_schedule", C.c_int, [C.c_void_p, C.c_int32]),
    ("kt_renderer_frame_hdr", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("kt_renderer_destroy", None, [C.c_void_p]),
    ("kt_view_state_init", C.c_int, [C.POINTER(KtViewState), C.POINTER(KtView)]),
    ("kt_should_render", C.c_int32, [C.POINTER(KtViewState), C.POINTER(KtView)]),
    ("kt_renderer_submit_view", C.c_int, [C.c_void_p, C.POINTER(KtViewState), C.POINTER(KtView),
                                          C.POINTER(C.c_int32)]),
    ("kt_write_png", C.c_int, [C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(C.c_int32)]),
    ("kt_fma_peak", C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    ("kt_generate_blackbody_lut_device", C.c_int, [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float,
                                                   C.c_void_p, C.c_void_p]),
    ("kt_generate_disk_lut_device", C.c_int, [C.POINTER(KtKerrParams), C.c_float, C.c_uint32, C.c_void_p,
                                              C.c_void_p]),
]


def lib() -> C.CDLL:
    """Loads the in-tree C-ABI library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m kerrtrace_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != KT_OK:
        msg = lib().kt_last_error().decode() or lib().kt_status_str(status).decode()
        raise KtError(status, msg)


# ---- host precompute ----------------------------------------------------------------------

def config_default() -> KtConfig:
    c = KtConfig()
    check(lib().kt_config_default(C.byref(c)))
    return c


def build_kerr_params(cfg: KtConfig) -> KtKerrParams:
    p = KtKerrParams()
    check(lib().kt_build_kerr_params(C.byref(cfg), C.byref(p)))
    return p


def generate_blackbody_lut(size, max_temp, wl_start, wl_end, wl_step):
    import numpy as np
    out = np.zeros((size, 4), dtype=np.float32)
    check(lib().kt_generate_blackbody_lut(size, max_temp, wl_start, wl_end, wl_step, out.ctypes.data))
    return out


def generate_disk_lut(params: KtKerrParams, disk_outer: float, size: int):
    import numpy as np
    out = np.zeros(size, dtype=np.float32)
    check(lib().kt_generate_disk_lut(C.byref(params), disk_outer, size, out.ctypes.data))
    return out


def generate_blackbody_lut_device(size, max_temp, wl_start, wl_end, wl_step, dev_ptr: int, stream: int = 0):
    """The blackbody table computed on the device into dev_ptr (float[4 * size])."""
    check(lib().kt_generate_blackbody_lut_device(size, max_temp, wl_start, wl_end, wl_step, C.c_void_p(dev_ptr),
                                                 C.c_void_p(stream)))


def generate_disk_lut_device(params: KtKerrParams, disk_outer: float, size: int, dev_ptr: int, stream: int = 0):
    """The disk temperature table computed on the device into dev_ptr (float[size])."""
    check(lib().kt_generate_disk_lut_device(C.byref(params), disk_outer, size, C.c_void_p(dev_ptr),
                                            C.c_void_p(stream)))


def build_defines(cfg: KtConfig) -> str:
    n = C.c_size_t(0)
    check(lib().kt_build_defines(C.byref(cfg), None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    check(lib().kt_build_defines(C.byref(cfg), buf, n.value + 1, C.byref(n)))
    return buf.value.decode()


def camera_basis(yaw_deg: float, pitch_deg: float):
    """calculate_camera_basis (src/math.rs:3-14): (forward, right, up) with world-up +y."""
    f = (C.c_float * 3)()
    r = (C.c_float * 3)()
    u = (C.c_float * 3)()
    check(lib().kt_camera_basis(yaw_deg, pitch_deg, f, r, u))
    return list(f), list(r), list(u)


def make_camera(pos, yaw_deg: float, pitch_deg: float, fov_deg: float) -> KtCamera:
    """Camera of submit_render from a position, yaw/pitch and vertical FOV (src/app.rs:158-170)."""
    f, r, u = camera_basis(yaw_deg, pitch_deg)
    cam = KtCamera()
    for i in range(3):
        cam.cam_pos[i] = pos[i]
        cam.fwd[i] = f[i]
        cam.rgt[i] = r[i]
        cam.up[i] = u[i]
    cam.fov_scale = lib().kt_fov_scale(fov_deg)
    return cam


def _orbit(r_obs: float, incl_deg: float, azimuth_deg: float):
    i = math.radians(incl_deg)
    az = math.radians(azimuth_deg)
    pos = (r_obs * math.sin(i) * math.cos(az), r_obs * math.cos(i), r_obs * math.sin(i) * math.sin(az))
    d = [-p / r_obs for p in pos]
    pitch = math.degrees(math.asin(max(-1.0, min(1.0, d[1]))))
    yaw = math.degrees(math.atan2(d[0], -d[2]))
    return pos, yaw, pitch


def orbit_camera(r_obs: float, incl_deg: float, fov_deg: float, azimuth_deg: float = 0.0) -> KtCamera:
    """Observer at Kerr-Schild radius r_obs, inclination from the spin axis (+y), looking at the
    hole.  Azimuth 0 puts the camera in the x-y plane; yaw/pitch follow src/math.rs:3-14."""
    pos, yaw, pitch = _orbit(r_obs, incl_deg, azimuth_deg)
    return make_camera(pos, yaw, pitch, fov_deg)


def orbit_view(r_obs: float, incl_deg: float, fov_deg: float, azimuth_deg: float = 0.0) -> "KtView":
    """The same observer as the app holds it (position, yaw, pitch, fov)."""
    pos, yaw, pitch = _orbit(r_obs, incl_deg, azimuth_deg)
    return make_view(pos, yaw, pitch, fov_deg)


# ---- device objects -----------------------------------------------------------------------

class Context:
    """Device context: LUT textures + scene constants (replaces the reference's NVRTC module,
    `c_params` upload and texture creation, src/renderer/init.rs:74-140)."""

    def __init__(self, cfg: KtConfig, device: int = 0, luts=None):
        """luts: None (host tables, the reference's), "device" (tables generated on the device) or
        a pair of arrays (blackbody rows, disk table)."""
        self.cfg = cfg.copy()
        h = C.c_void_p()
        if isinstance(luts, str) and luts == "device":
            check(lib().kt_context_create_device_luts(C.byref(self.cfg), device, C.byref(h)))
        elif luts is None:
            check(lib().kt_context_create(C.byref(self.cfg), device, C.byref(h)))
        else:
            import numpy as np
            bb = np.ascontiguousarray(luts[0], dtype=np.float32)
            dk = np.ascontiguousarray(luts[1], dtype=np.float32)
            check(lib().kt_context_create_with_luts(C.byref(self.cfg), device, bb.ctypes.data, dk.ctypes.data,
                                                    dk.shape[0], C.byref(h)))
        self.handle = h

    def params(self) -> KtKerrParams:
        p = KtKerrParams()
        check(lib().kt_context_params(self.handle, C.byref(p)))
        return p

    def trace(self, cam: KtCamera, hdr_ptr: int, err_ptr: int, stream: int = 0, schedule: int = SCHED_WAVEFRONT):
        check(lib().kt_trace(self.handle, C.c_void_p(stream), C.byref(cam), schedule, C.c_void_p(hdr_ptr),
                             C.c_void_p(err_ptr)))

    def trace_counted(self, cam: KtCamera, hdr_ptr: int, err_ptr: int, stream: int = 0,
                      schedule: int = SCHED_WAVEFRONT, aux_ptr: int = 0) -> KtTraceStats:
        st = KtTraceStats()
        check(lib().kt_trace_counted(self.handle, C.c_void_p(stream), C.byref(cam), schedule, C.c_void_p(hdr_ptr),
                                     C.c_void_p(err_ptr), C.byref(st), C.c_void_p(aux_ptr or None)))
        return st

    def trace_progressive(self, cam: KtCamera, first_sample: int, n_samples: int, accum_ptr: int, hdr_ptr: int,
                          err_ptr: int, stream: int = 0):
        """Samples [first_sample, first_sample + n_samples) added to the running sum in accum;
        hdr = the image of all samples so far."""
        check(lib().kt_trace_progressive(self.handle, C.c_void_p(stream), C.byref(cam), first_sample, n_samples,
                                         C.c_void_p(accum_ptr), C.c_void_p(hdr_ptr), C.c_void_p(err_ptr)))

    def set_tuning(self, schedule: int = SCHED_WAVEFRONT, block_x: int = 0, block_y: int = 0,
                   blocks_per_sm: int = 4, refill_min: int = 1, order: int = 0, keep_frozen: int = 0):
        """keep_frozen=1 lets NaN-frozen rays iterate to max_steps as the reference's do (same
        image; for timing the reference's amount of work)."""
        t = KtTuning(schedule, block_x, block_y, blocks_per_sm, refill_min, order, keep_frozen)
        check(lib().kt_context_set_tuning(self.handle, C.byref(t)))

    def tuning(self) -> KtTuning:
        t = KtTuning()
        check(lib().kt_context_get_tuning(self.handle, C.byref(t)))
        return t

    def bloom_horizontal(self, hdr_ptr: int, bloom_ptr: int, stream: int = 0):
        check(lib().kt_bloom_horizontal(self.handle, C.c_void_p(stream), C.c_void_p(hdr_ptr), C.c_void_p(bloom_ptr)))

    def post_process(self, hdr_ptr: int, bloom_ptr: int, image_ptr: int, stream: int = 0):
        check(lib().kt_post_process(self.handle, C.c_void_p(stream), C.c_void_p(hdr_ptr), C.c_void_p(bloom_ptr),
                                    C.c_void_p(image_ptr)))

    def post_fused(self, hdr_ptr: int, image_ptr: int, stream: int = 0):
        check(lib().kt_post_fused(self.handle, C.c_void_p(stream), C.c_void_p(hdr_ptr), C.c_void_p(image_ptr)))

    def close(self):
        if self.handle:
            lib().kt_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def diff_orbit_camera(observer_r: float, incl_deg: float, azimuth_deg: float, fov_deg: float):
    """The differentiable trace's orbit camera and its derivative in the inclination (degrees)."""
    cam, dcam = KtCamera(), KtCamera()
    check(lib().kt_diff_orbit_camera(observer_r, incl_deg, azimuth_deg, fov_deg, C.byref(cam), C.byref(dcam)))
    return cam, dcam


class Diff:
    """Differentiable trace (kt_diff_*): forward with step records, frozen-step replay and the
    discrete adjoint of the linear HDR image in (spin, inclination, temperature scale, r_out)."""

    def __init__(self, cfg: KtConfig, view: KtDiffView, segment_capacity: int = 0, device: int = 0):
        self.cfg = cfg.copy()
        self.view = view
        h = C.c_void_p()
        check(lib().kt_diff_create(C.byref(self.cfg), C.byref(view), segment_capacity, device, C.byref(h)))
        self.handle = h

    @staticmethod
    def params(theta) -> KtDiffParams:
        return theta if isinstance(theta, KtDiffParams) else KtDiffParams(*[float(v) for v in theta])

    def forward(self, theta, hdr_ptr: int, err_ptr: int, stream: int = 0):
        p = self.params(theta)
        check(lib().kt_diff_forward(self.handle, C.c_void_p(stream), C.byref(p), C.c_void_p(hdr_ptr),
                                    C.c_void_p(err_ptr)))

    def replay(self, theta, hdr_ptr: int, flags_ptr: int, err_ptr: int, stream: int = 0, hdr64_ptr: int = 0):
        p = self.params(theta)
        check(lib().kt_diff_replay(self.handle, C.c_void_p(stream), C.byref(p), C.c_void_p(hdr_ptr),
                                   C.c_void_p(hdr64_ptr or None), C.c_void_p(flags_ptr or None), C.c_void_p(err_ptr)))

    def replay_fp64(self, theta, hdr64_ptr: int, flags_ptr: int, err_ptr: int, hdr_ptr: int, stream: int = 0):
        """The recorded step sequence at theta in double arithmetic (FP32 records replayed in FP64)."""
        p = self.params(theta)
        check(lib().kt_diff_replay_fp64(self.handle, C.c_void_p(stream), C.byref(p), C.c_void_p(hdr64_ptr),
                                        C.c_void_p(flags_ptr or None), C.c_void_p(err_ptr), C.c_void_p(hdr_ptr)))

    def backward(self, dl_dhdr_ptr: int, grad_ptr: int, stream: int = 0):
        check(lib().kt_diff_backward(self.handle, C.c_void_p(stream), C.c_void_p(dl_dhdr_ptr), C.c_void_p(grad_ptr)))

    def backward_fp64(self, dl_dhdr_ptr: int, grad_ptr: int, stream: int = 0):
        """The adjoint of the FP64 replay of the records (kt_diff_backward_fp64)."""
        check(lib().kt_diff_backward_fp64(self.handle, C.c_void_p(stream), C.c_void_p(dl_dhdr_ptr),
                                          C.c_void_p(grad_ptr)))

    def info(self) -> KtDiffInfo:
        i = KtDiffInfo()
        check(lib().kt_diff_get_info(self.handle, C.byref(i)))
        return i

    def close(self):
        if self.handle:
            lib().kt_diff_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many renders (scenes, cameras, resolutions) traced in one launch (kt_batch_*)."""

    def __init__(self, jobs: list, device: int = 0):
        """jobs: list of (KtConfig, KtCamera, hdr_dev_ptr, err_dev_ptr)."""
        arr = (KtJob * len(jobs))()
        for i, (cfg, cam, hdr, err) in enumerate(jobs):
            arr[i].cfg = cfg
            arr[i].cam = cam
            arr[i].hdr_out = hdr
            arr[i].err_word = err
        h = C.c_void_p()
        check(lib().kt_batch_create(arr, len(jobs), device, C.byref(h)))
        self.handle = h

    def rays(self) -> int:
        return int(lib().kt_batch_rays(self.handle))

    def set_block(self, bx: int, by: int):
        check(lib().kt_batch_set_block(self.handle, bx, by))

    def set_camera(self, j: int, cam: KtCamera):
        check(lib().kt_batch_set_camera(self.handle, j, C.byref(cam)))

    def set_tuning(self, schedule: int = SCHED_PLAIN, block_x: int = 16, block_y: int = 16, blocks_per_sm: int = 4,
                   **_ignored):
        """SCHED_PLAIN: tiles of block_x x block_y; SCHED_WAVEFRONT: the persistent launch of
        32-pixel units with blocks_per_sm resident 128-thread blocks per SM."""
        t = KtTuning(schedule, block_x, block_y, blocks_per_sm, 1, 0, 0)
        check(lib().kt_batch_set_tuning(self.handle, C.byref(t)))

    def tuning(self) -> KtTuning:
        t = KtTuning()
        check(lib().kt_batch_get_tuning(self.handle, C.byref(t)))
        return t

    def autotune(self, reps: int = 3, stream: int = 0) -> list:
        """kt_batch_autotune: installs the fastest bit-identical launch shape; returns the rows
        (ms, tuning dict, identical)."""
        table = (KtTuneEntry * TUNE_MAX_CANDIDATES)()
        n = C.c_uint32(0)
        check(lib().kt_batch_autotune(self.handle, C.c_void_p(stream), reps, table, C.byref(n)))
        return [(float(table[i].ms), table[i].tuning.as_dict(), bool(table[i].identical)) for i in range(n.value)]

    def trace(self, stream: int = 0):
        check(lib().kt_batch_trace(self.handle, C.c_void_p(stream)))

    def trace_graph(self, stream: int = 0):
        check(lib().kt_batch_trace_graph(self.handle, C.c_void_p(stream)))

    def trace_sequential(self, stream: int = 0, schedule: int = SCHED_PLAIN):
        check(lib().kt_batch_trace_sequential(self.handle, C.c_void_p(stream), schedule))

    def close(self):
        if self.handle:
            lib().kt_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LutOverflow(KtError):
    def __init__(self, temp: float, message: str):
        super().__init__(KT_ERR_LUT_OVERFLOW, message)
        self.temp = temp


class Renderer:
    """Mirror of the reference's CudaRenderer (src/renderer/mod.rs:52-293)."""

    def __init__(self, cfg: KtConfig, device: int = 0):
        self.cfg = cfg.copy()
        h = C.c_void_p()
        check(lib().kt_renderer_new(C.byref(self.cfg), device, C.byref(h)))
        self.handle = h

    def set_schedule(self, schedule: int):
        check(lib().kt_renderer_set_schedule(self.handle, schedule))

    def set_tuning(self, tuning: KtTuning):
        check(lib().kt_renderer_set_tuning(self.handle, C.byref(tuning)))

    def autotune(self, cam: KtCamera, reps: int = 3):
        """kt_renderer_autotune: tunes the launch shape of submit_render for the view `cam`."""
        check(lib().kt_renderer_autotune(self.handle, C.byref(cam), reps))

    def submit_render(self, cam_pos, fwd, rgt, up, fov_scale: float) -> bool:
        arr = lambda v: (C.c_float * 3)(*v)  # noqa: E731
        sub = C.c_int32(0)
        check(lib().kt_renderer_submit_render(self.handle, arr(cam_pos), arr(fwd), arr(rgt), arr(up), fov_scale,
                                              C.byref(sub)))
        return bool(sub.value)

    def ready_frame(self):
        """Returns (index, numpy u32 view of the frame) or None when no frame is complete."""
        import numpy as np
        idx = C.c_uint32(0)
        data = C.POINTER(C.c_uint32)()
        temp = C.c_float(0.0)
        st = lib().kt_renderer_ready_frame(self.handle, C.byref(idx), C.byref(data), C.byref(temp))
        if st == KT_ERR_NOT_READY:
            return None
        if st == KT_ERR_LUT_OVERFLOW:
            raise LutOverflow(temp.value, lib().kt_last_error().decode())
        check(st)
        n = self.cfg.width * self.cfg.height
        view = np.ctypeslib.as_array(data, shape=(n,))
        return idx.value, view

    def finish_frame(self, index: int):
        check(lib().kt_renderer_finish_frame(self.handle, index))

    def wait(self):
        check(lib().kt_renderer_wait(self.handle))

    def submit_view(self, state: "ViewState", view: KtView) -> bool:
        """App::update_render_if_needed: submits when the view changed enough (or no frame yet)."""
        sub = C.c_int32(0)
        check(lib().kt_renderer_submit_view(self.handle, C.byref(state.s), C.byref(view), C.byref(sub)))
        return bool(sub.value)

    def frame_hdr_ptr(self, index: int) -> int:
        p = C.c_void_p()
        check(lib().kt_renderer_frame_hdr(self.handle, index, C.byref(p)))
        return p.value

    def close(self):
        if self.handle:
            lib().kt_renderer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = [n for n in dir() if not n.startswith("_")]


def make_view(cam_pos, yaw_deg: float, pitch_deg: float, fov_deg: float) -> KtView:
    return KtView((C.c_float * 3)(*cam_pos), yaw_deg, pitch_deg, fov_deg)


class ViewState:
    """The app's record of the last submitted view (src/app.rs:25-34, 43-56)."""

    def __init__(self, initial: KtView):
        self.s = KtViewState()
        check(lib().kt_view_state_init(C.byref(self.s), C.byref(initial)))

    def should_render(self, view: KtView) -> bool:
        r = lib().kt_should_render(C.byref(self.s), C.byref(view))
        if r < 0:
            raise KtError(KT_ERR_INVALID_ARG, "NULL argument")
        return bool(r)


def write_png(path, pixels, width: int, height: int) -> bool:
    """First-frame writer: 0x00RRGGBB u32 pixels (numpy, row-major) -> RGBA8 PNG.  Returns False
    when the file already exists (it is not replaced)."""
    import numpy as np
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    if px.size != width * height:
        raise ValueError("pixel count does not match the size")
    done = C.c_int32(0)
    check(lib().kt_write_png(str(path).encode(), px.ctypes.data_as(C.c_void_p), width, height, C.byref(done)))
    return bool(done.value)


def fma_peak(device: int = 0, iters: int = 4096) -> tuple[float, float]:
    """Measured FP32 FMA throughput of the device: (TFLOP/s, ms of the best launch)."""
    tf = C.c_double(0.0)
    ms = C.c_float(0.0)
    check(lib().kt_fma_peak(device, iters, C.byref(tf), C.byref(ms)))
    return tf.value, ms.value
