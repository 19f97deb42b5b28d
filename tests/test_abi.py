"""C-ABI library: exports, host precompute (params, LUTs, defines, bloom validation) against the
reference's Rust host semantics and against the oracle's independent restatement.  CPU only."""
from __future__ import annotations

import ctypes as C
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "kerrtrace.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kt_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(kt):
    lib_path = kt.LIB_PATH
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib_path)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (kt_[a-z0-9_]+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    bound = {name for name, _, _ in kt.SIGNATURES}
    assert set(declared_symbols()) <= bound | {"kt_status_str"}, set(declared_symbols()) - bound


def test_library_loads_and_versions(kt):
    L = kt.lib()
    assert L.kt_abi_version() == 3
    assert L.kt_status_str(kt.KT_ERR_LUT_OVERFLOW).decode().startswith("colour temperature")


def test_config_default_is_reference_config_yaml(kt):
    c = kt.config_default()
    # config.yaml of the reference (window 2100x900, spp 4, spin -0.45, mass 0.5, ...)
    assert (c.width, c.height, list(c.block_dim)) == (2100, 900, [16, 16])
    assert (c.spp, c.max_steps, c.max_attempts, c.lut_size) == (4, 100, 3, 4096)
    assert c.spin == np.float32(-0.45) and c.mass == np.float32(0.5)
    assert c.tolerance == np.float32(1e-5) and c.horizon_epsilon == np.float32(5e-7)
    assert c.bloom_radius == 48.0 and c.noise_detail == 10 and c.use_fast_math == 1


def test_kerr_params_match_oracle_and_formulas(kt, orc):
    from kerrtrace_b200 import workloads
    for name in workloads.SCENES:
        cfg, cam = workloads.scene(name)
        p = kt.build_kerr_params(cfg)
        o = orc.Scene(cfg, cam).params()
        got = np.array([p.a, p.m, p.aa, p.inv_m, p.a_norm, p.rh, p.disk_inner, p.inv_w_2, p.inv_h_2, p.aspect_ratio],
                       np.float32)
        assert np.array_equal(got.view(np.uint32), o.view(np.uint32)), (name, got, o)
        m, a = float(cfg.mass), float(cfg.spin)
        assert abs(p.rh - (m + math.sqrt(m * m - a * a))) < 1e-6
        assert p.inv_w_2 == np.float32(2.0 / cfg.width) and p.aspect_ratio == np.float32(cfg.width / cfg.height)


def test_kerr_params_errors(kt):
    base = kt.config_default()
    for field, value in (("width", 0), ("height", 0), ("mass", 0.0), ("spin", float("nan")),
                         ("noise_scale", float("inf"))):
        c = base.copy()
        setattr(c, field, value)
        with pytest.raises(kt.KtError) as e:
            kt.build_kerr_params(c)
        assert e.value.status == kt.KT_ERR_INVALID_ARG


def test_isco_known_values(kt):
    isco = kt.lib().kt_calc_isco
    assert abs(isco(0.0, 1, 1.0) - 6.0) < 1e-5
    assert abs(isco(0.0, 0, 1.0) - 6.0) < 1e-5
    assert abs(isco(0.9, 1, 1.0) - 2.320883) < 1e-5          # Bardeen-Press-Teukolsky
    assert abs(isco(0.9, 0, 1.0) - 8.717352) < 1e-4          # retrograde
    assert abs(isco(0.998, 1, 1.0) - 1.236970) < 1e-4
    assert isco(1.0, 1, 1.0) == pytest.approx(1.0, abs=1e-3)
    assert isco(0.9, 1, 2.0) == pytest.approx(2 * isco(0.9, 1, 1.0), rel=1e-6)
    assert isco(-0.9, 1, 1.0) == isco(0.9, 1, 1.0)             # even in a (the reference's ISCO)


@pytest.mark.parametrize("args", [
    (256, 4e7, 380.0, 780.0, 5.0), (4096, 3e4, 380.0, 720.0, 10.0), (128, 1e5, 380.0, 720.0, 10.0),
    (17, 9e3, 400.0, 700.0, 7.5), (2, 1e6, 380.0, 380.0, 1.0), (64, -5e3, 380.0, 720.0, 10.0)])
def test_blackbody_lut_matches_oracle_bitwise(kt, orc, args):
    a = kt.generate_blackbody_lut(*args)
    b = orc.blackbody_lut(*args)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_blackbody_lut_properties(kt):
    lut = kt.generate_blackbody_lut(256, 4e7, 380.0, 780.0, 5.0)
    assert np.all(lut[0] == 0.0)                     # T = 0 row (blackbody.rs:99-104)
    assert np.all(lut[:, 3] == 0.0)
    y = 0.2126 * lut[:, 0] + 0.7152 * lut[:, 1] + 0.0722 * lut[:, 2]
    assert np.all(np.diff(y[1:]) > 0)                 # luminance grows with T
    hot = lut[-1, :3] / lut[-1, :3].max()
    assert hot[2] > hot[0]                            # very hot blackbody is blue-white
    with pytest.raises(kt.KtError):
        kt.generate_blackbody_lut(1, 1e4, 380.0, 720.0, 10.0)
    with pytest.raises(kt.KtError):
        kt.generate_blackbody_lut(16, 1e4, 380.0, 720.0, 0.0)


@pytest.mark.parametrize("spin,mass,outer,size", [(0.9, 1.0, 20.0, 256), (0.998, 1.0, 30.0, 4096), (-0.45, 0.5, 40.0, 4096),
                                                  (0.0, 1.0, 12.0, 64), (-0.8, 1.0, 18.0, 128), (0.3, 2.0, 50.0, 3)])
def test_disk_lut_matches_oracle_bitwise(kt, orc, spin, mass, outer, size):
    c = kt.config_default()
    c.spin, c.mass = spin, mass
    p = kt.build_kerr_params(c)
    a = kt.generate_disk_lut(p, outer, size)
    b = orc.disk_lut(spin, mass, outer, size)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_disk_lut_properties(kt):
    c = kt.config_default()
    c.spin, c.mass = 0.9, 1.0
    p = kt.build_kerr_params(c)
    lut = kt.generate_disk_lut(p, 20.0, 256)
    assert lut[0] == 0.0                 # zero flux at the ISCO
    assert np.all(lut >= 0.0)
    # the reference's log-sum formula clamps a band just outside the ISCO to 0, then is positive
    nz = np.nonzero(lut)[0]
    assert len(nz) > 0.5 * len(lut) and np.all(lut[nz[0]:] > 0.0)
    assert 0 < int(np.argmax(lut)) < 255  # the flux peaks inside the disk
    with pytest.raises(kt.KtError):
        kt.generate_disk_lut(p, 1.0, 256)  # outer below inner


def test_defines_text_matches_rust_formatting(kt):
    import oracle.build as obuild
    from kerrtrace_b200 import workloads
    for name in workloads.SCENES:
        cfg, _ = workloads.scene(name)
        assert kt.build_defines(cfg) == obuild.defines_text(cfg)
    c = kt.config_default()
    txt = kt.build_defines(c)
    assert "#define CONFIG_INTEGRATOR_TOLERANCE 0.0000100000\n" in txt
    assert "#define CONFIG_HORIZON_EPSILON 0.0000005000\n" in txt
    assert "#define CONFIG_INTEGRATOR_MAX_STEPS 100\n" in txt


def test_validate_bloom(kt):
    c = kt.config_default()
    en, inten, rad, ri = C.c_int32(), C.c_float(), C.c_float(), C.c_int32()
    for r, expect in ((48.0, 48), (24.2, 25), (0.0, 0), (0.3, 1)):
        c.bloom_radius = r
        kt.check(kt.lib().kt_validate_bloom(C.byref(c), C.byref(en), C.byref(inten), C.byref(rad), C.byref(ri)))
        assert ri.value == expect
    for bad in (("bloom_radius", -1.0), ("bloom_intensity", -0.5), ("bloom_radius", float("nan")),
                ("bloom_radius", 3e9)):
        d = kt.config_default()
        setattr(d, *bad)
        assert kt.lib().kt_validate_bloom(C.byref(d), None, None, None, None) == kt.KT_ERR_INVALID_ARG


def test_camera_basis_convention(kt):
    f, r, u = kt.camera_basis(-90.0, -10.0)
    f, r, u = map(np.array, (f, r, u))
    assert np.allclose(f, [-math.cos(math.radians(10)), -math.sin(math.radians(10)), 0.0], atol=1e-6)
    for v in (f, r, u):
        assert abs(np.linalg.norm(v) - 1) < 1e-6
    assert abs(f @ r) < 1e-6 and abs(f @ u) < 1e-6 and abs(r @ u) < 1e-6
    assert u[1] > 0 and abs(r[1]) < 1e-7          # right is horizontal (world up +y, math.rs:10-12)
    assert kt.lib().kt_fov_scale(90.0) == pytest.approx(1.0, rel=1e-6)
    cam = kt.orbit_camera(50.0, 80.0, 30.0)
    pos = np.array(cam.cam_pos)
    assert np.allclose(pos, [50 * math.sin(math.radians(80)), 50 * math.cos(math.radians(80)), 0], atol=1e-4)
    assert np.allclose(np.array(cam.fwd), -pos / np.linalg.norm(pos), atol=1e-5)


def test_context_without_device_fails_loudly(kt):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    cfg = kt.config_default()
    with pytest.raises(kt.KtError) as e:
        kt.Context(cfg)
    assert e.value.status in (kt.KT_ERR_NO_DEVICE, kt.KT_ERR_CUDA)


def test_invalid_configs_rejected_before_device(kt):
    cfg = kt.config_default()
    for field, value in (("use_fast_math", 0), ("mode", 7), ("precision", 9), ("lut_size", 1)):
        c = cfg.copy()
        setattr(c, field, value)
        h = C.c_void_p()
        st = kt.lib().kt_context_create(C.byref(c), 0, C.byref(h))
        assert st in (kt.KT_ERR_INVALID_ARG, kt.KT_ERR_UNSUPPORTED), (field, st)
    c = cfg.copy()
    c.block_dim[0], c.block_dim[1] = 64, 32
    assert kt.lib().kt_context_create(C.byref(c), 0, C.byref(C.c_void_p())) == kt.KT_ERR_INVALID_ARG
    c = cfg.copy()
    c.mode, c.precision = kt.MODE_REF, kt.PREC_FP64
    assert kt.lib().kt_context_create(C.byref(c), 0, C.byref(C.c_void_p())) == kt.KT_ERR_INVALID_ARG
    # frames beyond 32768 on a side (the pixel index stays a 32-bit int, as in the reference's
    # kernel) and empty frames
    for w, h in ((40000, 16), (16, 40000), (0, 16), (16, 0)):
        c = cfg.copy()
        c.width, c.height = w, h
        assert kt.lib().kt_context_create(C.byref(c), 0, C.byref(C.c_void_p())) == kt.KT_ERR_INVALID_ARG, (w, h)


def test_diff_rejects_unsupported_configurations(kt):
    """The differentiable trace needs stated physics, spp 1, noise off and FP32 or FP64; the checks
    run before any device work."""
    from kerrtrace_b200 import workloads
    cfg, view = workloads.c5(32, kt.PREC_FP64)
    for field, value in (("mode", kt.MODE_REF), ("spp", 2), ("noise_enabled", 1), ("precision", kt.PREC_MIXED)):
        c = cfg.copy()
        setattr(c, field, value)
        with pytest.raises(kt.KtError):
            kt.Diff(c, view)


def test_diff_entry_points_refuse_null_arguments(kt):
    """The adjoint entry points check their arguments on the host, before any device work."""
    L = kt.lib()
    g = (C.c_double * 4)()
    for fn in (L.kt_diff_backward, L.kt_diff_backward_fp64):
        assert fn(None, None, None, None) == kt.KT_ERR_INVALID_ARG
        assert fn(None, None, C.cast(g, C.c_void_p), C.cast(g, C.c_void_p)) == kt.KT_ERR_INVALID_ARG


def _struct_bytes(s) -> bytes:
    return bytes(C.string_at(C.addressof(s), C.sizeof(s)))


def test_oracle_host_restatement_equals_the_library_host(kt, orc):
    """The runs of the reference kernel take their scene values, KerrParams, LUTs and cameras
    from the oracle's restatement of the reference host (oracle.Host, oracle.reference_inputs);
    the tests and the bench arm of the product take them from the library.  Both restatements
    must give the same bits for every named scene, else the two arms would not see one scene."""
    from kerrtrace_b200 import workloads
    host = orc.Host()
    assert _struct_bytes(host.config_default()) == _struct_bytes(kt.config_default())
    for name in workloads.SCENES:
        c_lib, cam_lib = workloads.scene(name)
        c_orc, cam_orc = workloads.scene(name, host=host)
        assert _struct_bytes(c_lib) == _struct_bytes(c_orc), name
        assert _struct_bytes(cam_lib) == _struct_bytes(cam_orc), name
        p_orc, bb, dk = orc.reference_inputs(c_orc)
        assert _struct_bytes(p_orc) == _struct_bytes(kt.build_kerr_params(c_lib)), name
        bb_lib = kt.generate_blackbody_lut(c_lib.lut_size, c_lib.lut_max_temp, c_lib.wavelength_start,
                                           c_lib.wavelength_end, c_lib.wavelength_step)
        dk_lib = kt.generate_disk_lut(kt.build_kerr_params(c_lib), c_lib.disk_outer_radius, c_lib.lut_size)
        assert np.array_equal(bb.view(np.uint32), bb_lib.view(np.uint32)), name
        assert np.array_equal(dk.view(np.uint32), dk_lib.view(np.uint32)), name
    for (c1, k1), (c2, k2) in zip(workloads.c4_jobs(), workloads.c4_jobs(host=host)):
        assert _struct_bytes(c1) == _struct_bytes(c2) and _struct_bytes(k1) == _struct_bytes(k2)
    rng = np.random.default_rng(11)
    for yaw, pitch in zip(rng.uniform(-180, 180, 200), rng.uniform(-89, 89, 200)):
        assert kt.camera_basis(float(yaw), float(pitch)) == orc.camera_basis(float(yaw), float(pitch))
    for fov in rng.uniform(1.0, 120.0, 200):
        assert np.float32(kt.lib().kt_fov_scale(float(fov))) == np.float32(orc.fov_scale(float(fov)))


@pytest.mark.gpu
def test_autotune_through_the_c_abi(kt):
    """kt_context_autotune (C++, CUDA events) on the 1080p scene at 320 x 180: every candidate of
    the built-in list is timed, all give the default shape's image bit for bit, and the
    installed tuning (KT_SCHED_AUTO) reproduces that image."""
    import torch
    from kerrtrace_b200 import workloads
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg, cam = workloads.scene("c2")
    cfg = workloads.scaled(cfg, 320, 180)
    ctx = kt.Context(cfg)
    n = cfg.width * cfg.height
    base = torch.zeros((n, 4), device="cuda")
    out = torch.zeros((n, 4), device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    ctx.trace(base_cam := cam, base.data_ptr(), err.data_ptr(), 0, kt.SCHED_WAVEFRONT)
    table = (kt.KtTuneEntry * kt.TUNE_MAX_CANDIDATES)()
    n_rows = C.c_uint32(0)
    kt.check(kt.lib().kt_context_autotune(ctx.handle, None, C.byref(base_cam), 2, None, 0, table, C.byref(n_rows)))
    rows = [table[i] for i in range(n_rows.value)]
    assert len(rows) == 56  # FP32 reference semantics: 2 orders x (6 + 6 plain + 16 wavefront)
    assert all(r.identical == 1 and r.ms > 0 for r in rows)
    best = ctx.tuning()
    assert min(r.ms for r in rows) == next(r.ms for r in rows if r.tuning.as_dict() == best.as_dict())
    ctx.trace(cam, out.data_ptr(), err.data_ptr(), 0, kt.SCHED_AUTO)
    torch.cuda.synchronize()
    assert torch.equal(out.view(torch.int32), base.view(torch.int32))
    bad = kt.KtTuning(kt.SCHED_PLAIN, 0, 0, 4, 1, 0, 0)
    assert kt.lib().kt_context_autotune(ctx.handle, None, C.byref(cam), 0, None, 0, None, None) == kt.KT_ERR_INVALID_ARG
    assert kt.lib().kt_context_autotune(ctx.handle, None, C.byref(cam), 1, C.byref(bad), 0, None, None) == \
        kt.KT_ERR_INVALID_ARG
    ctx.close()
