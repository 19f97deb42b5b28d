"""Known-answer tests that pin the CPU oracle.  The reference ships no tests or golden vectors, so
the pins come from the mathematics of the path (Kerr-Schild geometry, Hamilton's equations,
Dormand-Prince order conditions, Hairer's dense output, Schwarzschild capture) and, in
test_golden.py, from outputs of the reference kernel itself."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle
from oracle import olib


def ks_r(x, y, z, a):
    return olib().kto_ks_radius(x, y, z, a)


def rhs(st, pt, a, m):
    s = np.ascontiguousarray(st, np.float64)
    d = np.zeros(6)
    olib().kto_rhs(s.ctypes.data, pt, a, m, d.ctypes.data)
    return d


def hamiltonian(st, pt, a, m):
    """H = 1/2 (|p|^2 - p_t^2 - 2 Hk (l.p - p_t)^2) for the Kerr-Schild metric, spin along +y."""
    x, y, z, px, py, pz = st
    r = ks_r(x, y, z, a)
    D = r * r + a * a
    l = np.array([(r * x - a * z) / D, y / r, (r * z + a * x) / D])
    Hk = m * r ** 3 / (r ** 4 + a * a * y * y)
    lp = l @ np.array([px, py, pz]) - pt
    return 0.5 * (px * px + py * py + pz * pz - pt * pt - 2 * Hk * lp * lp)


def test_ks_radius():
    rng = np.random.default_rng(0)
    for _ in range(200):
        x, y, z = rng.normal(size=3) * 10
        assert ks_r(x, y, z, 0.0) == pytest.approx(math.sqrt(x * x + y * y + z * z), rel=1e-14)
        a = rng.uniform(-1, 1)
        r = ks_r(x, y, z, a)
        rho2 = x * x + y * y + z * z
        assert abs(r ** 4 - (rho2 - a * a) * r * r - a * a * y * y) <= 1e-12 * r ** 4
    assert ks_r(5.0, 0.0, 0.0, 0.9) == pytest.approx(math.sqrt(25 - 0.81), rel=1e-14)


@pytest.mark.parametrize("a", [0.0, 0.5, -0.9, 0.998])
def test_rhs_is_hamiltons_equations(a):
    """dx/dl = dH/dp and dp/dl = -dH/dx (central differences of the Hamiltonian)."""
    rng = np.random.default_rng(1)
    for _ in range(20):
        st = np.concatenate([rng.normal(size=3) * 6 + np.array([0, 0, 8]), rng.normal(size=3)])
        pt = -rng.uniform(0.5, 1.5)
        d = rhs(st, pt, a, 1.0)
        fd = np.zeros(6)
        for i in range(6):
            e = np.zeros(6)
            h = 1e-6 * max(1.0, abs(st[i]))
            e[i] = h
            fd[i] = (hamiltonian(st + e, pt, a, 1.0) - hamiltonian(st - e, pt, a, 1.0)) / (2 * h)
        np.testing.assert_allclose(d[:3], fd[3:], rtol=1e-6, atol=1e-8)
        np.testing.assert_allclose(d[3:], -fd[:3], rtol=1e-6, atol=1e-8)


def test_reference_rhs_keeps_the_reference_y_gradient():
    """Reference mode integrates the reference's d(r^2)/dy = y (1 + (u + 4a^2)/(2s))
    (cuda/kerr_math.cuh:97).  It differs from Hamilton's equations only in the momentum
    derivatives and only off the equatorial plane; on y = 0 both forms agree exactly."""
    rng = np.random.default_rng(4)
    for a in (0.0, 0.9):
        for _ in range(20):
            st = np.concatenate([rng.normal(size=3) * 6 + np.array([0, 0, 8]), rng.normal(size=3)])
            pt = -1.0
            exact = rhs(st, pt, a, 1.0)
            ref = np.zeros(6)
            s = np.ascontiguousarray(st)
            olib().kto_rhs_reference(s.ctypes.data, pt, a, 1.0, ref.ctypes.data)
            assert np.array_equal(ref[:3], exact[:3])
            assert np.abs(ref[3:] - exact[3:]).max() > 1e-6
            st[1] = 0.0
            s = np.ascontiguousarray(st)
            olib().kto_rhs_reference(s.ctypes.data, pt, a, 1.0, ref.ctypes.data)
            assert np.allclose(ref, rhs(st, pt, a, 1.0), rtol=1e-15, atol=0)


def null_init(cam, direction, a, m=1.0):
    cam = np.ascontiguousarray(cam, np.float64)
    d = np.ascontiguousarray(direction, np.float64)
    st = np.zeros(6)
    pt = C.c_double(0)
    olib().kto_null_init(cam.ctypes.data, d.ctypes.data, C.c_double(a), C.c_double(m), st.ctypes.data, C.byref(pt))
    return st, pt.value


def dp5(st, pt, a, m, h, with_stages=False):
    out, err, k = np.zeros(6), np.zeros(6), np.zeros((7, 6))
    s = np.ascontiguousarray(st, np.float64)
    olib().kto_dp5_step(s.ctypes.data, C.c_double(pt), C.c_double(a), C.c_double(m), C.c_double(h), out.ctypes.data,
                        err.ctypes.data, k.ctypes.data)
    return (out, err, k) if with_stages else (out, err)


def test_null_initialisation_and_conservation():
    """The initial momentum is null (H = 0) and DP5 steps keep H near 0."""
    for a in (0.0, 0.9, -0.7):
        st, pt = null_init([40.0, 7.0, 3.0], [-1.0, -0.1, 0.05], a)
        assert abs(hamiltonian(st, pt, a, 1.0)) < 1e-13
        assert pt < 0
        s = st.copy()
        for _ in range(200):
            s, _ = dp5(s, pt, a, 1.0, 0.05)
        assert abs(hamiltonian(s, pt, a, 1.0)) < 1e-9


def kerr_constants(st, pt, a):
    """E = -p_t, the angular momentum about the spin axis (y) and the Carter constant of a
    Kerr-Schild Cartesian state; p_theta comes from the spheroidal coordinates of the point,
    X + iY = (r + i a) e^{i phi} sin(theta), Z = r cos(theta) with (X, Y, Z) = (x, -z, y).  The
    trace kernels' long-ray predictor uses these expressions."""
    x, y, z, px, py, pz = st
    r = ks_r(x, y, z, a)
    E = -pt
    L = z * px - x * pz
    ct = y / r
    s2 = 1.0 - ct * ct
    pth = ct / math.sqrt(s2) * (x * px + z * pz) - r * math.sqrt(s2) * py
    Q = pth * pth + ct * ct * (L * L / s2 - a * a * E * E)
    return E, L, Q


@pytest.mark.parametrize("a", [0.0, 0.9, -0.7])
@pytest.mark.parametrize("d", [[-1.0, -0.12, 0.35], [-1.0, 0.3, 0.3]])
def test_kerr_constants_of_motion_are_conserved(a, d):
    """L and Q stay constant along the oracle's (exact-gradient) integration of a ray that
    passes the hole within 11 M, which pins both the expressions and the oracle's dynamics."""
    st, pt = null_init([20.0, 3.0, 2.0], d, a)
    E0, L0, Q0 = kerr_constants(st, pt, a)
    s = st.copy()
    r_min = 1e9
    for _ in range(600):
        s, _ = dp5(s, pt, a, 1.0, 0.05)
        r_min = min(r_min, ks_r(s[0], s[1], s[2], a))
    E1, L1, Q1 = kerr_constants(s, pt, a)
    assert r_min < 11.0 and ks_r(s[0], s[1], s[2], a) > r_min + 2.0  # passed the hole
    assert abs(L1 - L0) < 1e-10 * max(1.0, abs(L0))
    assert abs(Q1 - Q0) < 1e-10 * max(1.0, abs(Q0))


def test_dp5_orders():
    """Local error of the 5th-order update is O(h^6); the embedded estimate is O(h^5)."""
    st, pt = null_init([12.0, 2.0, 1.0], [-1.0, 0.2, 0.3], 0.6)

    def fine(h, n=64):
        s = st.copy()
        for _ in range(n):
            s, _ = dp5(s, pt, 0.6, 1.0, h / n)
        return s

    errs, ests = [], []
    for h in (0.4, 0.2, 0.1):
        y, e = dp5(st, pt, 0.6, 1.0, h)
        errs.append(np.linalg.norm(y - fine(h)))
        ests.append(np.linalg.norm(e))
    p_loc = math.log2(errs[0] / errs[1]), math.log2(errs[1] / errs[2])
    p_est = math.log2(ests[0] / ests[1]), math.log2(ests[1] / ests[2])
    assert all(5.3 < p < 6.7 for p in p_loc), p_loc
    assert all(4.3 < p < 5.7 for p in p_est), p_est


def test_dense_output_interpolates_the_step():
    rng = np.random.default_rng(2)
    for _ in range(50):
        q = rng.normal(size=9)
        q[8] = abs(q[8]) + 0.1  # h
        y0, y1, k1, k7, h = q[0], q[1], q[2], q[7], q[8]
        d = lambda t: olib().kto_dense(q.ctypes.data, t)  # noqa: E731
        ds = lambda t: olib().kto_dense_slope(q.ctypes.data, t)  # noqa: E731
        assert d(0.0) == pytest.approx(y0, abs=1e-12)
        assert d(1.0) == pytest.approx(y1, abs=1e-12)
        assert ds(0.0) == pytest.approx(h * k1, abs=1e-12)
        assert ds(1.0) == pytest.approx(h * k7, abs=1e-12)
        t = rng.uniform(0.05, 0.95)
        assert (d(t + 1e-6) - d(t - 1e-6)) / 2e-6 == pytest.approx(ds(t), rel=1e-5, abs=1e-7)


def test_crossing_root_converges():
    """The safeguarded Newton root of y(t) = 0 on the dense output lands on the root (|y| at
    rounding level) for steps whose y changes sign, including the case where the last Newton
    update rounds to the bracket end (which must end the iteration, not restart a bisection)."""
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(3000):
        q = np.zeros(9)
        q[0] = rng.uniform(0.05, 3.0) * rng.choice([-1.0, 1.0])   # y0
        q[1] = -np.sign(q[0]) * rng.uniform(0.05, 3.0)            # y1: opposite sign
        q[8] = rng.uniform(0.05, 1.0)                              # h
        slope = (q[1] - q[0]) / q[8]
        q[2:8] = slope * (1.0 + 0.05 * rng.normal(size=6))         # stage slopes near the chord
        t0 = q[0] / (q[0] - q[1])
        t = olib().kto_crossing_root(q.ctypes.data, t0)
        assert 0.0 <= t <= 1.0
        y = olib().kto_dense(q.ctypes.data, t)
        worst = max(worst, abs(y) / max(abs(q[0]), abs(q[1])))
    assert worst < 1e-12, worst


def test_dense_output_accuracy_on_a_ray():
    """Interpolating inside one DP5 step agrees with re-integrating to that point (4th order)."""
    st, pt = null_init([10.0, 1.0, 2.0], [-1.0, 0.1, -0.2], 0.9)
    h = 0.3
    y, _, K = dp5(st, pt, 0.9, 1.0, h, with_stages=True)
    assert np.allclose(K[0], rhs(st, pt, 0.9, 1.0), rtol=1e-15)
    for frac in (0.25, 0.5, 0.8):
        ys, _ = dp5(st, pt, 0.9, 1.0, frac * h)
        for c in range(6):
            q = np.array([st[c], y[c], K[0][c], K[2][c], K[3][c], K[4][c], K[5][c], K[6][c], h])
            assert olib().kto_dense(q.ctypes.data, frac) == pytest.approx(ys[c], abs=5e-6)


def pcg32_py(state: int) -> int:
    x = (state * 6364136223846793005 + 1442695040888963407) & (2 ** 64 - 1)
    xs = (((x >> 18) ^ x) >> 27) & 0xFFFFFFFF
    rot = x >> 59
    return ((xs >> rot) | (xs << ((32 - rot) & 31))) & 0xFFFFFFFF


def test_pcg32_hash():
    for s in (0, 1, 42, 0xda3e39cb94b95bdb, (123 << 32) | 7, 2 ** 64 - 1):
        assert olib().kto_pcg32(s) == pcg32_py(s)


def test_fbm_and_tone_map():
    rng = np.random.default_rng(5)
    vals = [olib().kto_fbm(u, v, 5, 0) for u, v in rng.normal(size=(500, 2)) * 20]
    assert 0.0 <= min(vals) and max(vals) <= 1.0 and np.std(vals) > 0.02
    assert olib().kto_fbm(3.3, 1.1, 0, 0) == 0.5
    assert olib().kto_fbm(3.0, 7.0, 4, 0) == pytest.approx(0.5, abs=1e-12)   # lattice point: gradient noise is 0
    assert olib().kto_aces(0.0) == 0.0
    assert olib().kto_aces(1e6) == pytest.approx(2.51 / 2.43, rel=1e-4)
    lo = olib().kto_srgb(0.0031308)
    hi = 1.055 * 0.0031308 ** (1 / 2.4) - 0.055
    assert lo == pytest.approx(hi, rel=1e-3)   # the two branches of the OETF meet


def _line_scene(kt, width=61, b_max=8.0, mode=1):
    """A 1-row image of a Schwarzschild hole seen edge-on from r = 500: pixel i has impact
    parameter b_i = 500 * sin(atan(u_i))."""
    cfg = kt.config_default()
    cfg.width, cfg.height = width, 1
    cfg.spin, cfg.mass = 0.0, 1.0
    cfg.spp = 1
    cfg.mode = mode
    cfg.tolerance, cfg.initial_step, cfg.max_steps = 1e-9, 1.0, 20000
    cfg.escape_radius, cfg.horizon_epsilon = 1000.0, 0.02
    cfg.disk_temperature_scale = 0.0
    cfg.disk_outer_radius = 7.0
    cfg.lut_size = 16
    cfg.noise_enabled = 0
    half = math.tan(math.asin(b_max / 500.0))
    cam = kt.make_camera((500.0, 0.0, 0.0), -90.0, 0.0, 30.0)
    cam.fov_scale = half * cfg.height / cfg.width  # u = (2 (i + 0.5) / W - 1) * W/H * fov_scale spans +-half
    return cfg, cam


def test_schwarzschild_capture_threshold(kt):
    """Rays with impact parameter below 3*sqrt(3) M fall in, above it escape (stated physics)."""
    cfg, cam = _line_scene(kt)
    _, info, _ = oracle.Scene(cfg, cam).render(2)
    half = cam.fov_scale * cfg.width / cfg.height
    u = ((np.arange(cfg.width) + 0.5) * (2.0 / cfg.width) - 1.0) * half
    b = 500.0 * np.sin(np.arctan(np.abs(u)))
    bc = 3 * math.sqrt(3)
    term = info["term"]
    captured = term == oracle.TERM_HORIZON
    escaped = term == oracle.TERM_ESCAPE
    assert np.all(captured[b < bc - 0.15]), (b[~captured & (b < bc - 0.15)])
    assert np.all(escaped[b > bc + 0.15]), (b[~escaped & (b > bc + 0.15)])


def test_diff_reference_gradient_against_its_own_differences():
    """The oracle's forward-mode gradient of the stated-physics image: in the temperature scale
    and the disk outer radius (which leave the step sequence alone) it equals central
    differences of the oracle's own trace, pixel by pixel."""
    from kerrtrace_b200 import workloads
    cfg, view = workloads.c5(32, 2)
    th = np.array(workloads.C5_START)
    col, dcol, info = oracle.diff_render(cfg, view, th)
    assert (info[:, 1] > 0).sum() > 200
    for j, e, tol in ((2, 1e-6, 1e-8), (3, 1e-5, 1e-4)):
        tp, tm = th.copy(), th.copy()
        tp[j] += e
        tm[j] -= e
        cp, _, ip = oracle.diff_render(cfg, view, tp)
        cm, _, im = oracle.diff_render(cfg, view, tm)
        same = (ip == info).all(1) & (im == info).all(1) & (col.max(1) > 0)
        fd = (cp - cm) / (2 * e)
        a = dcol[:, :, j]
        rel = np.abs(a - fd)[same].max(1) / (np.abs(fd[same]).max(1) + 1e-9 * np.abs(fd).max())
        assert np.median(rel) < tol, (j, np.median(rel))
