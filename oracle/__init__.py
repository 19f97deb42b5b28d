"""CPU oracle and reference-kernel harness bindings.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU-baseline / reference legs of bench.py use
this package, as the checker.  The product (kerrtrace_b200) never imports it.

  Oracle      libkt_oracle.so  — kt_oracle.cpp: the reference algorithm restated on the CPU
              (f64, or an f32 emulation), its LUT generators and post-processing.
  RefKernel   _ref/libktref_<scene>.so — the reference's own cuda/kernel.cu compiled from its
              source with the scene's #define header, launched like src/renderer/mod.rs.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "libkt_oracle.so"
REF_DIR = HERE / "_ref"


class KtoScene(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("spin", C.c_float), ("mass", C.c_float),
        ("spp", C.c_uint32), ("sky_grid_divisions", C.c_uint32), ("max_steps", C.c_uint32),
        ("max_attempts", C.c_uint32),
        ("exposure_scale", C.c_float), ("sky_line_thickness", C.c_float), ("sky_intensity", C.c_float),
        ("disk_outer_radius", C.c_float), ("disk_temperature_scale", C.c_float),
        ("initial_step", C.c_float), ("tolerance", C.c_float), ("transmittance_cutoff", C.c_float),
        ("horizon_epsilon", C.c_float), ("escape_radius", C.c_float), ("wavelength_step", C.c_float),
        ("noise_enabled", C.c_int32), ("noise_scale", C.c_float), ("noise_strength", C.c_float),
        ("noise_winding", C.c_float), ("noise_detail", C.c_uint32),
        ("lut_size", C.c_uint32), ("lut_max_temp", C.c_float),
        ("bb_lut", C.c_void_p), ("disk_lut", C.c_void_p),
        ("mode", C.c_int32), ("tex_mode", C.c_int32), ("retire_frozen", C.c_int32),
        ("noise_seed", C.c_uint32), ("noise_phase", C.c_float),
        ("cam_pos", C.c_float * 3), ("fwd", C.c_float * 3), ("rgt", C.c_float * 3), ("up", C.c_float * 3),
        ("fov_scale", C.c_float),
    ]


class KtoRayInfo(C.Structure):
    _fields_ = [("term", C.c_int32), ("hits", C.c_int32), ("crossings", C.c_int32), ("steps", C.c_int32),
                ("attempts", C.c_int32), ("rhs", C.c_int32), ("first_r", C.c_double), ("first_g", C.c_double),
                ("first_T", C.c_double)]


INFO_DTYPE = np.dtype([("term", np.int32), ("hits", np.int32), ("crossings", np.int32), ("steps", np.int32),
                       ("attempts", np.int32), ("rhs", np.int32), ("first_r", np.float64),
                       ("first_g", np.float64), ("first_T", np.float64)])
assert INFO_DTYPE.itemsize == C.sizeof(KtoRayInfo)

TERM_BUDGET, TERM_HORIZON, TERM_ESCAPE, TERM_FROZEN = 0, 1, 2, 3

_olib = None


def olib() -> C.CDLL:
    global _olib
    if _olib is None:
        if not ORACLE_LIB.exists():
            raise ImportError(f"{ORACLE_LIB} missing: run `python oracle/build.py`")
        L = C.CDLL(str(ORACLE_LIB))
        L.kto_render.argtypes = [C.POINTER(KtoScene), C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int]
        L.kto_render.restype = C.c_int
        L.kto_post.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_int, C.c_float, C.c_float, C.c_int, C.c_float,
                               C.c_void_p, C.c_void_p]
        L.kto_blackbody_lut.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
        L.kto_disk_lut.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_void_p]
        L.kto_params.argtypes = [C.POINTER(KtoScene), C.c_void_p]
        L.kto_camera_basis.argtypes = [C.c_float, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
        L.kto_camera_basis.restype = None
        L.kto_fov_scale.argtypes = [C.c_float]
        L.kto_fov_scale.restype = C.c_float
        L.kto_isco.argtypes = [C.c_float, C.c_int, C.c_float]
        L.kto_isco.restype = C.c_float
        L.kto_nt_factor.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float]
        L.kto_nt_factor.restype = C.c_float
        L.kto_define_value.argtypes = [C.c_float]
        L.kto_define_value.restype = C.c_double
        L.kto_pcg32.argtypes = [C.c_uint64]
        L.kto_pcg32.restype = C.c_uint32
        L.kto_ks_radius.argtypes = [C.c_double] * 4
        L.kto_ks_radius.restype = C.c_double
        L.kto_rhs.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p]
        L.kto_rhs_reference.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p]
        L.kto_dense.argtypes = [C.c_void_p, C.c_double]
        L.kto_dense.restype = C.c_double
        L.kto_dense_slope.argtypes = [C.c_void_p, C.c_double]
        L.kto_dense_slope.restype = C.c_double
        L.kto_crossing_root.argtypes = [C.c_void_p, C.c_double]
        L.kto_crossing_root.restype = C.c_double
        L.kto_diff_render.argtypes = [C.POINTER(KtoScene), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int]
        L.kto_diff_render.restype = C.c_int
        L.kto_fbm.argtypes = [C.c_double, C.c_double, C.c_int, C.c_uint32]
        L.kto_fbm.restype = C.c_double
        L.kto_aces.argtypes = [C.c_double]
        L.kto_aces.restype = C.c_double
        L.kto_srgb.argtypes = [C.c_double]
        L.kto_srgb.restype = C.c_double
        L.kto_dp5_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                   C.c_void_p]
        L.kto_null_init.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        _olib = L
    return _olib


def blackbody_lut(size, max_temp, wl_start, wl_end, wl_step) -> np.ndarray:
    out = np.zeros((size, 4), np.float32)
    if olib().kto_blackbody_lut(size, max_temp, wl_start, wl_end, wl_step, out.ctypes.data) != 0:
        raise ValueError("invalid blackbody LUT arguments")
    return out


def disk_lut(spin, mass, disk_outer, size) -> np.ndarray:
    out = np.zeros(size, np.float32)
    if olib().kto_disk_lut(spin, mass, disk_outer, size, out.ctypes.data) != 0:
        raise ValueError("invalid disk LUT arguments")
    return out


# ---- the reference host's set-up values, restated ------------------------------------------
# The reference derives its kernel inputs on the host (src/renderer/utils.rs, blackbody.rs,
# src/math.rs, src/app.rs).  These functions give those values from the oracle's own
# restatement, so that a run of the reference kernel (RefKernel) takes none of its inputs from
# the product library.

# config.yaml:1-67, the fields the kernel path reads (window size, renderer block, bloom,
# blackbody LUT, cuda, kernel, disk_noise); the YAML's max_steps 1e2 is the integer 100.
CONFIG_YAML = {
    "width": 2100, "height": 900, "block_dim": (16, 16),
    "bloom_enabled": 1, "bloom_intensity": 0.5, "bloom_radius": 48.0,
    "lut_size": 4096, "lut_max_temp": 3e4, "wavelength_start": 380.0, "wavelength_end": 720.0,
    "wavelength_step": 10.0, "use_fast_math": 1,
    "spp": 4, "exposure_scale": 3e-3, "sky_grid_divisions": 40, "sky_line_thickness": 5e-4, "sky_intensity": 30.0,
    "spin": -0.45, "mass": 0.5, "disk_outer_radius": 40.0, "disk_temperature_scale": 3e4,
    "initial_step": 1.0, "tolerance": 1e-5, "max_steps": 100, "max_attempts": 3, "transmittance_cutoff": 1e-2,
    "horizon_epsilon": 5e-7, "escape_radius": 80.0,
    "noise_enabled": 1, "noise_scale": 0.1, "noise_strength": 0.6, "noise_winding": 50.0, "noise_detail": 10,
}


class KtoKerrParams(C.Structure):
    """The reference's KerrParams (src/renderer/init.rs:15-33, cuda/kerr_math.cuh:3-9)."""

    _fields_ = [(n, C.c_float) for n in ("a", "m", "aa", "inv_m", "a_norm", "rh", "disk_inner",
                                         "inv_w_2", "inv_h_2", "aspect_ratio", "disk_noise_scale",
                                         "disk_noise_strength", "disk_noise_winding")] + [
        ("disk_noise_enabled", C.c_int32), ("disk_noise_detail", C.c_int32)]


def config_default(cfg_type):
    """A `cfg_type` structure (any ctypes structure with the config field names) holding
    config.yaml's values; fields config.yaml does not have stay zero, except the stated-physics
    extension `photon_zone_factor`, whose default is 1.5."""
    c = cfg_type()
    names = {n for n, _ in cfg_type._fields_}
    for k, v in CONFIG_YAML.items():
        if k == "block_dim":
            c.block_dim[0], c.block_dim[1] = v
        else:
            setattr(c, k, v)
    if "photon_zone_factor" in names:
        c.photon_zone_factor = 1.5
    return c


def _scene_of(cfg) -> "KtoScene":
    s = KtoScene()
    for name, _ in KtoScene._fields_:
        if name in ("bb_lut", "disk_lut", "mode", "tex_mode", "retire_frozen", "cam_pos", "fwd", "rgt", "up",
                    "fov_scale", "noise_seed", "noise_phase"):
            continue
        setattr(s, name, getattr(cfg, name))
    return s


def kerr_params(cfg) -> KtoKerrParams:
    """build_kerr_params (src/renderer/utils.rs:53-113) from the oracle's restatement."""
    v = np.zeros(10, np.float32)
    if olib().kto_params(C.byref(_scene_of(cfg)), v.ctypes.data) != 0:
        raise ValueError("invalid scene for the Kerr parameters")
    return KtoKerrParams(*[float(x) for x in v], float(cfg.noise_scale), float(cfg.noise_strength),
                         float(cfg.noise_winding), 1 if cfg.noise_enabled else 0, int(cfg.noise_detail))


def camera_basis(yaw_deg: float, pitch_deg: float):
    """calculate_camera_basis (src/math.rs:3-14): (forward, right, up)."""
    f, r, u = (C.c_float * 3)(), (C.c_float * 3)(), (C.c_float * 3)()
    olib().kto_camera_basis(yaw_deg, pitch_deg, f, r, u)
    return list(f), list(r), list(u)


def fov_scale(fov_deg: float) -> float:
    """tan(fov.to_radians() / 2) (src/app.rs:163)."""
    return float(olib().kto_fov_scale(fov_deg))


class Host:
    """The host arithmetic a named scene needs (config defaults, the horizon radius, the disk
    table's peak, the camera basis), taken from the oracle's restatement.  Passed to the scene
    builders of kerrtrace_b200.workloads by the runs of the reference kernel, so that those runs
    map no product library."""

    def config_default(self):
        from kerrtrace_b200 import KtConfig  # the structure layout only; no library is loaded
        return config_default(KtConfig)

    def horizon_radius(self, cfg) -> float:
        return float(kerr_params(cfg).rh)

    def disk_lut(self, cfg) -> np.ndarray:
        return disk_lut(cfg.spin, cfg.mass, cfg.disk_outer_radius, cfg.lut_size)

    def camera(self, pos, yaw_deg: float, pitch_deg: float, fov_deg: float):
        from kerrtrace_b200 import KtCamera
        f, r, u = camera_basis(yaw_deg, pitch_deg)
        cam = KtCamera()
        for i in range(3):
            cam.cam_pos[i], cam.fwd[i], cam.rgt[i], cam.up[i] = pos[i], f[i], r[i], u[i]
        cam.fov_scale = fov_scale(fov_deg)
        return cam


def reference_inputs(cfg):
    """(KerrParams, blackbody LUT, disk LUT) as the reference host builds them for `cfg`, from
    the oracle's restatement (utils.rs:53-113, blackbody.rs:56-124, utils.rs:172-201)."""
    p = kerr_params(cfg)
    bb = blackbody_lut(cfg.lut_size, cfg.lut_max_temp, cfg.wavelength_start, cfg.wavelength_end, cfg.wavelength_step)
    dk = disk_lut(cfg.spin, cfg.mass, cfg.disk_outer_radius, cfg.lut_size)
    return p, bb, dk


class Scene:
    """Oracle scene built from a product config + camera (plain values; the oracle derives the
    Kerr parameters and LUTs itself)."""

    def __init__(self, cfg, cam, mode=None, tex_mode: int = 1, retire_frozen: bool = True, luts=None):
        s = KtoScene()
        for name, _ in KtoScene._fields_:
            if name in ("bb_lut", "disk_lut", "mode", "tex_mode", "retire_frozen", "cam_pos", "fwd", "rgt", "up",
                        "fov_scale"):
                continue
            setattr(s, name, getattr(cfg, name))
        s.mode = cfg.mode if mode is None else mode
        s.tex_mode = tex_mode
        s.retire_frozen = 1 if retire_frozen else 0
        for k in ("cam_pos", "fwd", "rgt", "up"):
            for i in range(3):
                getattr(s, k)[i] = getattr(cam, k)[i]
        s.fov_scale = cam.fov_scale
        if luts is None:
            self.bb = blackbody_lut(cfg.lut_size, cfg.lut_max_temp, cfg.wavelength_start, cfg.wavelength_end,
                                    cfg.wavelength_step)
            self.disk = disk_lut(cfg.spin, cfg.mass, cfg.disk_outer_radius, cfg.lut_size)
        else:
            self.bb = np.ascontiguousarray(luts[0], np.float32)
            self.disk = np.ascontiguousarray(luts[1], np.float32)
        s.bb_lut = self.bb.ctypes.data
        s.disk_lut = self.disk.ctypes.data
        self.s = s
        self.cfg = cfg

    def params(self) -> np.ndarray:
        out = np.zeros(10, np.float32)
        if olib().kto_params(C.byref(self.s), out.ctypes.data) != 0:
            raise ValueError("invalid scene")
        return out

    def render(self, precision: int = 2, pixels=None, threads: int = 0):
        """Returns (rgba float32 [n,4], infos [n], err u32[2]).  pixels: flat indices or None."""
        n = self.s.width * self.s.height if pixels is None else len(pixels)
        rgba = np.zeros((n, 4), np.float32)
        infos = np.zeros(n, INFO_DTYPE)
        err = np.zeros(2, np.uint32)
        pix = None
        if pixels is not None:
            pix = np.ascontiguousarray(pixels, np.int64)
        rc = olib().kto_render(C.byref(self.s), precision, None if pix is None else pix.ctypes.data, n,
                               rgba.ctypes.data, infos.ctypes.data, err.ctypes.data, threads)
        if rc != 0:
            raise ValueError(f"oracle render failed ({rc})")
        return rgba, infos, err


def post(hdr: np.ndarray, width: int, height: int, radius: int, sigma: float, intensity: float, mode: int = 0,
         threshold: float = 0.0):
    hdr = np.ascontiguousarray(hdr, np.float32).reshape(-1, 4)
    img = np.zeros(width * height, np.uint32)
    olib().kto_post(hdr.ctypes.data, width, height, radius, sigma, intensity, mode, threshold, img.ctypes.data, None)
    return img


# ---- reference kernel harness -----------------------------------------------------------

class KtrefTextures(C.Structure):
    _fields_ = [("bb_arr", C.c_void_p), ("disk_arr", C.c_void_p), ("bb_tex", C.c_uint64), ("disk_tex", C.c_uint64)]


def ref_lib_path(scene: str) -> Path:
    return REF_DIR / f"libktref_{scene}.so"


class RefKernel:
    """The reference's cuda/kernel.cu, compiled with the defines of `scene`, driven like
    src/renderer/mod.rs: c_params upload, LUT textures, trace/bloom/post launches."""

    def __init__(self, scene: str):
        p = ref_lib_path(scene)
        if not p.exists():
            raise FileNotFoundError(f"{p} missing: run `python oracle/build.py` where the reference tree exists")
        L = C.CDLL(str(p))
        L.ktref_set_params.argtypes = [C.c_void_p, C.c_size_t]
        L.ktref_make_textures.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(KtrefTextures)]
        L.ktref_free_textures.argtypes = [C.POINTER(KtrefTextures)]
        L.ktref_trace.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_uint64, C.c_int, C.c_float,
                                  C.c_void_p, C.c_uint64, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int,
                                  C.c_void_p]
        L.ktref_bloom.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                  C.c_int, C.c_void_p]
        L.ktref_post.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                 C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.ktref_tex_probe.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        self.L = L
        self.scene = scene
        self.tex = None

    def setup(self, params_struct, bb: np.ndarray, disk: np.ndarray):
        """params_struct: a ctypes KerrParams mirror (kerrtrace_b200.KtKerrParams layout)."""
        rc = self.L.ktref_set_params(C.byref(params_struct), C.sizeof(params_struct))
        if rc != 0:
            raise RuntimeError(f"ktref_set_params failed: {rc}")
        self._bb = np.ascontiguousarray(bb, np.float32)
        self._disk = np.ascontiguousarray(disk, np.float32)
        t = KtrefTextures()
        rc = self.L.ktref_make_textures(self._bb.ctypes.data, self._disk.ctypes.data, int(self._disk.shape[0]),
                                        C.byref(t))
        if rc != 0:
            raise RuntimeError(f"ktref_make_textures failed: {rc}")
        self.tex = t

    def trace(self, hdr_ptr, cfg, cam, lut_max_temp, err_ptr, disk_inner, stream=0):
        cam12 = (C.c_float * 12)(*cam.cam_pos, *cam.fwd, *cam.rgt, *cam.up)
        rc = self.L.ktref_trace(C.c_void_p(hdr_ptr), cfg.width, cfg.height, cam12, self.tex.bb_tex, cfg.lut_size,
                                lut_max_temp, C.c_void_p(err_ptr), self.tex.disk_tex, disk_inner,
                                cfg.disk_outer_radius, cam.fov_scale, cfg.block_dim[0], cfg.block_dim[1],
                                C.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"ktref_trace failed: {rc}")

    def bloom(self, hdr_ptr, bloom_ptr, cfg, radius, sigma, enabled, stream=0):
        rc = self.L.ktref_bloom(C.c_void_p(hdr_ptr), C.c_void_p(bloom_ptr), cfg.width, cfg.height, radius, sigma,
                                enabled, cfg.block_dim[0], cfg.block_dim[1], C.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"ktref_bloom failed: {rc}")

    def post(self, hdr_ptr, bloom_ptr, image_ptr, cfg, radius, sigma, intensity, enabled, stream=0):
        rc = self.L.ktref_post(C.c_void_p(hdr_ptr), C.c_void_p(bloom_ptr), C.c_void_p(image_ptr), cfg.width,
                               cfg.height, radius, sigma, intensity, enabled, cfg.block_dim[0], cfg.block_dim[1],
                               C.c_void_p(stream))
        if rc != 0:
            raise RuntimeError(f"ktref_post failed: {rc}")

    def tex_probe(self, which: str, us_ptr, out_ptr, n):
        tex = self.tex.bb_tex if which == "bb" else self.tex.disk_tex
        rc = self.L.ktref_tex_probe(tex, C.c_void_p(us_ptr), C.c_void_p(out_ptr), n, 4 if which == "bb" else 1)
        if rc != 0:
            raise RuntimeError(f"ktref_tex_probe failed: {rc}")

    def close(self):
        if self.tex is not None:
            self.L.ktref_free_textures(C.byref(self.tex))
            self.tex = None


def diff_render(cfg, view, theta, pixels=None, threads: int = 0):
    """Forward-mode f64 reference of the differentiable trace (stated physics, spp 1, no noise):
    returns (colour [n,3], d colour / d theta [n,3,4], info [n,3] = term, hits, steps) for the
    flat pixel indices `pixels` (all pixels when None).  view: the product's KtDiffView;
    theta = (spin, inclination deg, temperature scale, disk outer radius)."""
    from kerrtrace_b200 import KtCamera
    sc = Scene(cfg, KtCamera(), mode=1, tex_mode=0)
    n = cfg.width * cfg.height if pixels is None else len(pixels)
    pix = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    v = np.array([view.observer_r, view.azimuth_deg, view.fov_deg, view.base_temperature_scale], np.float64)
    th = np.ascontiguousarray(theta, np.float64)
    col = np.zeros((n, 3))
    dcol = np.zeros((n, 3, 4))
    info = np.zeros((n, 3), np.int32)
    rc = olib().kto_diff_render(C.byref(sc.s), v.ctypes.data, th.ctypes.data, None if pix is None else pix.ctypes.data,
                                n, col.ctypes.data, dcol.ctypes.data, info.ctypes.data, threads)
    if rc != 0:
        raise ValueError(f"oracle diff render failed ({rc})")
    return col, dcol, info
