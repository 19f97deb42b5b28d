"""Named scenes: the benchmark configurations and the small parity scenes.

Each function returns ``(KtConfig, KtCamera)``.  Values the benchmark description leaves open
(LUT range, exposure, peak temperature, escape radius) are fixed here.

  c1   256x256, FOV 30, r_obs 50, inclination 80, a = 0.9, tolerance 1e-8, h0 0.1,
       20000 steps, horizon at 1.01 r_h, escape 1000, disk to 20 M, 256-entry LUTs over
       380-780 nm in 5 nm steps, peak disk temperature 1e7 K, no noise, no bloom.
  c2   1920x1080, FOV 25, r_obs 100, inclination 85, a = 0.998, tolerance 1e-6, 20000 steps,
       disk to 30 M, FBM noise with 5 octaves, bloom radius 24 (sigma 8), ACES + sRGB.
  t1   96x64 general parity scene (2 spp, noise, bloom radius 6) - seconds on the oracle.
  t2   80x48 parity scene aimed at the sky grid and rejected steps (max_attempts 1).
"""
from __future__ import annotations

from . import (KtCamera, KtConfig, _orbit, build_kerr_params, config_default, generate_disk_lut,
               make_camera)


class LibraryHost:
    """Host arithmetic of a scene (config.yaml defaults, the horizon radius, the disk table, the
    camera basis) from this library's host entry points.  A scene builder takes any object with
    these four methods; runs of the reference kernel pass the oracle's restatement instead, so
    that they load no product code."""

    def config_default(self) -> KtConfig:
        return config_default()

    def horizon_radius(self, cfg: KtConfig) -> float:
        return float(build_kerr_params(cfg).rh)

    def disk_lut(self, cfg: KtConfig):
        return generate_disk_lut(build_kerr_params(cfg), cfg.disk_outer_radius, cfg.lut_size)

    def camera(self, pos, yaw_deg: float, pitch_deg: float, fov_deg: float) -> KtCamera:
        return make_camera(pos, yaw_deg, pitch_deg, fov_deg)


_LIBRARY = LibraryHost()


def _host(host):
    return _LIBRARY if host is None else host


def _peak_scale(cfg: KtConfig, peak_temp: float, host=None) -> float:
    """disk_temperature_scale that puts the largest disk-LUT entry at `peak_temp` kelvin (the
    reference scales an un-normalised f^(1/4), src/renderer/utils.rs:172-201)."""
    peak = float(_host(host).disk_lut(cfg).max())
    # the reference's flux formula is identically 0 for some negative spins: no disk emission
    return float(peak_temp / peak) if peak > 0 else 0.0


def _horizon_eps(cfg: KtConfig, factor: float, host=None) -> float:
    return float(_host(host).horizon_radius(cfg) * factor)


def orbit_camera(r_obs: float, incl_deg: float, fov_deg: float, azimuth_deg: float = 0.0, host=None) -> KtCamera:
    """kerrtrace_b200.orbit_camera with the camera basis of `host`."""
    pos, yaw, pitch = _orbit(r_obs, incl_deg, azimuth_deg)
    return _host(host).camera(pos, yaw, pitch, fov_deg)


def c1(host=None) -> tuple[KtConfig, KtCamera]:
    c = _host(host).config_default()
    c.width, c.height = 256, 256
    c.spp = 1
    c.spin, c.mass = 0.9, 1.0
    c.tolerance = 1e-8
    c.initial_step = 0.1
    c.max_steps = 20000
    c.max_attempts = 3
    c.escape_radius = 1000.0
    c.horizon_epsilon = _horizon_eps(c, 0.01, host)
    c.disk_outer_radius = 20.0
    c.lut_size = 256
    c.wavelength_start, c.wavelength_end, c.wavelength_step = 380.0, 780.0, 5.0
    c.lut_max_temp = 4e7
    c.disk_temperature_scale = _peak_scale(c, 1e7, host)
    c.noise_enabled = 0
    c.bloom_enabled = 0
    c.exposure_scale = 1.0
    return c, orbit_camera(50.0, 80.0, 30.0, host=host)


def c2(host=None) -> tuple[KtConfig, KtCamera]:
    c = _host(host).config_default()
    c.width, c.height = 1920, 1080
    c.spp = 1
    c.spin, c.mass = 0.998, 1.0
    c.tolerance = 1e-6
    c.initial_step = 0.1
    c.max_steps = 20000
    c.max_attempts = 3
    c.escape_radius = 1000.0
    c.horizon_epsilon = _horizon_eps(c, 0.01, host)
    c.disk_outer_radius = 30.0
    c.lut_size = 4096
    c.wavelength_start, c.wavelength_end, c.wavelength_step = 380.0, 720.0, 10.0
    c.lut_max_temp = 1e5
    c.disk_temperature_scale = _peak_scale(c, 1e4, host)
    c.exposure_scale = 3e-3
    c.noise_enabled, c.noise_detail = 1, 5
    c.noise_scale, c.noise_strength, c.noise_winding = 0.1, 0.6, 50.0
    c.noise_seed, c.noise_phase = 42, 0.0
    c.bloom_enabled, c.bloom_radius, c.bloom_intensity = 1, 24.0, 0.5
    c.bloom_threshold = 1.0
    return c, orbit_camera(100.0, 85.0, 25.0, host=host)


def t1(host=None) -> tuple[KtConfig, KtCamera]:
    c = _host(host).config_default()
    c.width, c.height = 96, 64
    c.spp = 2
    c.spin, c.mass = 0.9, 1.0
    c.tolerance = 1e-5
    c.initial_step = 0.5
    c.max_steps = 3000
    c.escape_radius = 200.0
    c.horizon_epsilon = _horizon_eps(c, 0.01, host)
    c.disk_outer_radius = 25.0
    c.lut_size = 256
    c.lut_max_temp = 1e5
    c.disk_temperature_scale = _peak_scale(c, 1.2e4, host)
    c.exposure_scale = 3e-3
    c.noise_enabled, c.noise_detail = 1, 3
    c.bloom_enabled, c.bloom_radius, c.bloom_intensity = 1, 6.0, 0.5
    return c, orbit_camera(30.0, 75.0, 40.0, host=host)


def t2(host=None) -> tuple[KtConfig, KtCamera]:
    c = _host(host).config_default()
    c.width, c.height = 80, 48
    c.spp = 1
    c.spin, c.mass = -0.8, 1.0
    c.tolerance = 2e-5
    c.initial_step = 1.0
    c.max_steps = 1500
    c.max_attempts = 1
    c.escape_radius = 120.0
    c.horizon_epsilon = 5e-7
    c.disk_outer_radius = 18.0
    c.lut_size = 128
    c.lut_max_temp = 1e5
    c.disk_temperature_scale = _peak_scale(c, 9e3, host)
    c.exposure_scale = 3e-3
    c.sky_grid_divisions = 12
    c.sky_line_thickness = 2e-2
    c.noise_enabled = 0
    c.bloom_enabled, c.bloom_radius, c.bloom_intensity = 1, 3.0, 0.8
    return c, orbit_camera(40.0, 60.0, 70.0, azimuth_deg=30.0, host=host)


def c3_draws(n: int = 8, seed: int = 7) -> list[tuple[float, float]]:
    """(spin, inclination in degrees) of the mixed-precision ablation: spin ~ U[-0.99, 0.99],
    inclination ~ U[5, 89], drawn in that order per draw from numpy's default generator."""
    import numpy as np
    rng = np.random.default_rng(seed)
    return [(float(rng.uniform(-0.99, 0.99)), float(rng.uniform(5.0, 89.0))) for _ in range(n)]


def c3(draw: int = 0, size: int = 4096, host=None) -> tuple[KtConfig, KtCamera]:
    """Mixed-precision ablation scene: 4096x4096, FOV 20, r_obs 60, 1 spp, stated physics,
    mixed precision (switch `precision` for the FP32 / FP64 runs), tolerance 1e-6."""
    spin, incl = c3_draws()[draw]
    c = _host(host).config_default()
    c.width = c.height = size
    c.spp = 1
    c.mode, c.precision = 1, 1
    c.spin, c.mass = spin, 1.0
    c.tolerance = 1e-6
    c.initial_step = 0.1
    c.max_steps = 20000
    c.max_attempts = 3
    c.escape_radius = 1000.0
    c.horizon_epsilon = _horizon_eps(c, 0.01, host)
    c.disk_outer_radius = 30.0
    c.lut_size = 4096
    c.wavelength_start, c.wavelength_end, c.wavelength_step = 380.0, 720.0, 10.0
    c.lut_max_temp = 2e5
    c.disk_temperature_scale = _peak_scale(c, 1e4, host)
    c.exposure_scale = 3e-3
    c.noise_enabled = 0
    c.bloom_enabled = 0
    return c, orbit_camera(60.0, incl, 20.0, host=host)


def c4_jobs(seed: int = 123, scale: int = 1, host=None) -> list[tuple[KtConfig, KtCamera]]:
    """Batched-launch workload: 64 independent renders, 16 each of 256^2, 512^2, 1024^2 and
    1920x1080 (divided by `scale`), with spin ~ U[-0.99, 0.99], inclination ~ U[5, 89] deg,
    observer radius ~ U[30, 200] M and disk outer radius ~ U[10, 50] M drawn per job (in that
    order) from numpy's default generator; tolerance 1e-6, reference semantics."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = [(256, 256)] * 16 + [(512, 512)] * 16 + [(1024, 1024)] * 16 + [(1920, 1080)] * 16
    jobs = []
    for w, h in sizes:
        spin = float(rng.uniform(-0.99, 0.99))
        incl = float(rng.uniform(5.0, 89.0))
        r_obs = float(rng.uniform(30.0, 200.0))
        r_out = float(rng.uniform(10.0, 50.0))
        c, _ = c2(host)
        c.width, c.height = max(8, w // scale), max(8, h // scale)
        c.spin = spin
        c.horizon_epsilon = _horizon_eps(c, 0.01, host)
        c.disk_outer_radius = r_out
        c.lut_max_temp = 2e5
        c.disk_temperature_scale = _peak_scale(c, 1e4, host)
        jobs.append((c, orbit_camera(r_obs, incl, 25.0, host=host)))
    return jobs


C5_TARGET = (0.7, 60.0, 1.0, 25.0)   # spin, inclination (deg), temperature scale, disk outer radius
C5_START = (0.5, 50.0, 0.8, 20.0)


def c5(size: int = 512, precision: int = 0, host=None):
    """Differentiable inverse problem: 512x512, FOV 30, r_obs 50, stated physics, spp 1, no
    noise, tolerance 1e-6.  Returns (KtConfig, KtDiffView); theta = C5_TARGET renders the
    target, C5_START is the starting point.  The view's base temperature scale puts the
    disk-LUT peak at 1e4 K at the target's spin and r_out, so theta's temperature scale is a
    plain multiplier."""
    from . import KtDiffView
    c = _host(host).config_default()
    c.width = c.height = size
    c.spp = 1
    c.mode, c.precision = 1, precision
    c.spin, c.mass = C5_TARGET[0], 1.0
    c.tolerance = 1e-6
    c.initial_step = 0.1
    c.max_steps = 20000
    c.max_attempts = 3
    c.escape_radius = 1000.0
    c.horizon_epsilon = 0.01
    c.disk_outer_radius = C5_TARGET[3]
    c.lut_size = 1024
    c.wavelength_start, c.wavelength_end, c.wavelength_step = 380.0, 720.0, 10.0
    c.lut_max_temp = 1e5
    c.disk_temperature_scale = _peak_scale(c, 1e4, host)
    c.exposure_scale = 3e-3
    c.noise_enabled = 0
    c.bloom_enabled = 0
    view = KtDiffView(50.0, 0.0, 30.0, float(c.disk_temperature_scale))
    return c, view


SCENES = {"c1": c1, "c2": c2, "t1": t1, "t2": t2, "c3": c3}


def scene(name: str, host=None) -> tuple[KtConfig, KtCamera]:
    """The named scene; `host` supplies its host arithmetic (default: this library's)."""
    return SCENES[name](host=host)


def scaled(cfg: KtConfig, width: int, height: int) -> KtConfig:
    """Same scene at another resolution (everything else, including the defines, unchanged)."""
    c = cfg.copy()
    c.width, c.height = width, height
    return c


def rays(cfg: KtConfig) -> int:
    return int(cfg.width) * int(cfg.height) * int(cfg.spp)


def camera_list(cam: KtCamera) -> list[float]:
    return [*cam.cam_pos, *cam.fwd, *cam.rgt, *cam.up]

