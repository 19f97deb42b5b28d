// kt_diff_host.cpp — C ABI of the differentiable trace (kt_diff_*).
//
// The parameters theta = (spin, inclination, temperature scale, disk outer radius) enter the
// device scene through the Kerr parameters, the camera, the disk temperature scale and the disk
// temperature LUT.  Per call the host builds the scene at theta (the renderer's own scene and
// LUT builders), the camera with its inclination tangent, and the derivatives of the
// theta-dependent scene inputs: d(ISCO)/d(spin) and d(LUT entry)/d(spin, r_out) from the
// Page-Thorne flux differentiated with dual numbers in double.  The FP64 path also takes theta,
// the camera and the disk LUT in double, so that its image is a smooth function of theta down
// to double rounding (which central differences of small steps need).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "kt_diff.h"
#include "kt_internal.h"

namespace {

kt_status err_cuda(cudaError_t e, const char* what) {
    char buf[256];
    std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return ktd::set_error(KT_ERR_CUDA, buf);
}
kt_status err_arg(const char* msg) { return ktd::set_error(KT_ERR_INVALID_ARG, msg); }

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        cudaSetDevice(dev);
    }
    ~DevGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// ---- dual numbers (double, derivatives in spin and r_out) --------------------------------------
struct HD {
    double v, d[2];
    HD(double x = 0.0, double d0 = 0.0, double d1 = 0.0) : v(x), d{d0, d1} {}
};
HD operator+(HD a, HD b) { return HD(a.v + b.v, a.d[0] + b.d[0], a.d[1] + b.d[1]); }
HD operator-(HD a, HD b) { return HD(a.v - b.v, a.d[0] - b.d[0], a.d[1] - b.d[1]); }
HD operator-(HD a) { return HD(-a.v, -a.d[0], -a.d[1]); }
HD operator*(HD a, HD b) { return HD(a.v * b.v, a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1]); }
HD operator/(HD a, HD b) {
    const double q = a.v / b.v;
    return HD(q, (a.d[0] - q * b.d[0]) / b.v, (a.d[1] - q * b.d[1]) / b.v);
}
HD chain(HD x, double f, double df) { return HD(f, df * x.d[0], df * x.d[1]); }
HD hsqrt(HD x) { const double s = std::sqrt(x.v); return chain(x, s, s > 0.0 ? 0.5 / s : 0.0); }
HD hcbrt(HD x) { const double c = std::cbrt(x.v); return chain(x, c, c != 0.0 ? 1.0 / (3.0 * c * c) : 0.0); }
HD hlog(HD x) { return chain(x, std::log(x.v), 1.0 / x.v); }
HD hcos(HD x) { return chain(x, std::cos(x.v), -std::sin(x.v)); }
HD hacos(HD x) { return chain(x, std::acos(x.v), -1.0 / std::sqrt(1.0 - x.v * x.v)); }

// ISCO (Bardeen, Press & Teukolsky), prograde, in units of M (isco_f32 of the host builders).
HD isco_d(HD an) {
    const HD one(1.0);
    const HD z1 = one + hcbrt(one - an * an) * (hcbrt(one + an) + hcbrt(one - an));
    const HD z2 = hsqrt(HD(3.0) * an * an + z1 * z1);
    HD inside = (HD(3.0) - z1) * (HD(3.0) + z1 + HD(2.0) * z2);
    if (inside.v < 0.0) inside = HD(0.0);
    return HD(3.0) + z2 - hsqrt(inside);
}

// Page-Thorne flux factor (nt_factor_f32 of the host builders) in double with derivatives.
HD nt_factor_d(HD r, HD an, HD r_isco, double inv_m) {
    if (!(r.v > r_isco.v)) return HD(0.0);
    const HD rn = r * HD(inv_m), rin = r_isco * HD(inv_m);
    const HD x = hsqrt(rn), xms = hsqrt(rin);
    const HD base = hacos(-an) * HD(1.0 / 3.0);
    const double step = 2.0943951023931957;
    const HD roots[3] = {HD(2.0) * hcos(base), HD(2.0) * hcos(base - HD(step)), HD(2.0) * hcos(base + HD(step))};
    HD sum(0.0);
    for (int i = 0; i < 3; ++i) {
        const HD xi = roots[i];
        const HD den = xi * (xi - roots[(i + 1) % 3]) * (xi - roots[(i + 2) % 3]);
        if (!(den.v > 0.0)) continue;
        const HD coef = HD(3.0) * (xi - an) * (xi - an) / den;
        const HD val = (x - xi) / (xms - xi);
        if (val.v > 0.0) sum = sum + coef * hlog(val);
    }
    const HD q = x - xms - HD(1.5) * an * hlog(x / xms) - sum;
    const HD geo = rn * (rn * x - HD(3.0) * x + HD(2.0) * an);
    const HD f = q / geo;
    return f.v > 0.0 ? f : HD(0.0);
}

// Orbit camera at (r, inclination i from +y, azimuth) looking at the origin, and its derivative
// in i (degrees).  forward = -position / r, right = (sin az, 0, -cos az) (independent of i),
// up = right x forward: the basis kt_camera_basis builds from the matching yaw / pitch.
void orbit_camera(double r, double incl_deg, double az_deg, double fov_deg, kt_camera* cam, kt_camera* dcam,
                  ktd::CameraD* camd = nullptr, ktd::CameraD* dcamd = nullptr) {
    const double d2r = 3.14159265358979323846 / 180.0;
    const double i = incl_deg * d2r, az = az_deg * d2r;
    const double pos[3] = {r * std::sin(i) * std::cos(az), r * std::cos(i), r * std::sin(i) * std::sin(az)};
    const double dpos[3] = {r * std::cos(i) * std::cos(az) * d2r, -r * std::sin(i) * d2r,
                            r * std::cos(i) * std::sin(az) * d2r};
    double f[3], df[3];
    for (int c = 0; c < 3; ++c) {
        f[c] = -pos[c] / r;
        df[c] = -dpos[c] / r;
    }
    const double rt[3] = {std::sin(az), 0.0, -std::cos(az)};
    auto cross = [](const double* a, const double* b, double* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    double up[3], dup[3];
    cross(rt, f, up);
    cross(rt, df, dup);
    const float fs = (float)std::tan(fov_deg * d2r / 2.0);
    for (int c = 0; c < 3; ++c) {
        cam->cam_pos[c] = (float)pos[c];
        cam->fwd[c] = (float)f[c];
        cam->rgt[c] = (float)rt[c];
        cam->up[c] = (float)up[c];
        if (dcam) {
            dcam->cam_pos[c] = (float)dpos[c];
            dcam->fwd[c] = (float)df[c];
            dcam->rgt[c] = 0.0f;
            dcam->up[c] = (float)dup[c];
        }
    }
    cam->fov_scale = fs;
    if (dcam) dcam->fov_scale = 0.0f;
    if (camd && dcamd) {
        for (int c = 0; c < 3; ++c) {
            camd->pos[c] = pos[c];
            camd->fwd[c] = f[c];
            camd->rgt[c] = rt[c];
            camd->up[c] = up[c];
            dcamd->pos[c] = dpos[c];
            dcamd->fwd[c] = df[c];
            dcamd->rgt[c] = 0.0;
            dcamd->up[c] = dup[c];
        }
        camd->fov_scale = std::tan(fov_deg * d2r / 2.0);
        dcamd->fov_scale = 0.0;
    }
}

ktd::Camera to_dev_camera(const kt_camera& c) {
    ktd::Camera o;
    for (int i = 0; i < 3; ++i) {
        o.pos[i] = c.cam_pos[i];
        o.fwd[i] = c.fwd[i];
        o.rgt[i] = c.rgt[i];
        o.up[i] = c.up[i];
    }
    o.fov_scale = c.fov_scale;
    return o;
}

}  // namespace

// One LUT set per parameter point in use (the recorded one, and the replay one).
struct kt_diff_luts {
    float* disk = nullptr;       // float LUT (FP32 path: the renderer's LUT)
    double* disk_d = nullptr;    // double LUT (FP64 path)
    double* dlut_da = nullptr;
    double* dlut_dro = nullptr;
};

struct kt_diff {
    int device = 0;
    kt_config cfg{};        // base configuration
    kt_diff_view view{};
    uint32_t n_px = 0, cap = 0;
    size_t seg_bytes = 0;
    ktd::DiffRay* rays = nullptr;
    void* segs = nullptr;
    unsigned* ctl = nullptr;  // [0] pool cursor, [1] overflow count
    ktd::DiffWork work{};     // the adjoint's work ordering
    float4* bb = nullptr;     // blackbody LUT (does not depend on theta)
    kt_diff_luts lut_rec, lut_rep;
    // the recorded point
    bool have_record = false;
    ktd::Scene sc_rec{};
    ktd::Camera cam_rec{};
    ktd::CameraD camd_rec{}, dcamd_rec{};
    ktd::DiffLut dl_rec{};
    kt_diff_params theta_rec{};
};

namespace {

void free_luts(kt_diff_luts& l) {
    cudaFree(l.disk);
    cudaFree(l.disk_d);
    cudaFree(l.dlut_da);
    cudaFree(l.dlut_dro);
    l = kt_diff_luts{};
}

void destroy(kt_diff* d) {
    if (!d) return;
    DevGuard g(d->device);
    cudaFree(d->rays);
    cudaFree(d->segs);
    cudaFree(d->ctl);
    cudaFree(d->bb);
    cudaFree(d->work.bucket);
    cudaFree(d->work.order);
    cudaFree(d->work.ctl);
    free_luts(d->lut_rec);
    free_luts(d->lut_rep);
    delete d;
}

// Scene, camera and derivative inputs at theta; LUTs uploaded into `luts` on `st`.  The float
// fields come from the float configuration at theta (the renderer's scene); the FP64 path also
// gets theta in double: spin, disk radii, temperature scale, camera and a double disk LUT.
kt_status prepare(kt_diff* d, const kt_diff_params* th, kt_diff_luts& luts, cudaStream_t st, ktd::Scene* sc,
                  ktd::Camera* cam, ktd::CameraD* camd, ktd::CameraD* dcamd, ktd::DiffLut* dl, bool force64 = false) {
    if (!std::isfinite(th->spin) || !std::isfinite(th->inclination_deg) || !std::isfinite(th->temperature_scale) ||
        !std::isfinite(th->disk_outer_radius))
        return err_arg("diff parameters must be finite");
    kt_config c = d->cfg;
    if (force64) c.precision = KT_PREC_FP64;
    c.spin = (float)th->spin;
    c.disk_outer_radius = (float)th->disk_outer_radius;
    c.disk_temperature_scale = (float)((double)d->view.base_temperature_scale * th->temperature_scale);
    kt_status s = ktd::scene_from_config(&c, sc);
    if (s != KT_OK) return s;
    kt_kerr_params kp;
    if ((s = kt_build_kerr_params(&c, &kp)) != KT_OK) return s;
    const uint32_t n = c.lut_size;
    std::vector<float> disk(n);
    std::vector<double> disk_d(n), da(n), dro(n);
    if ((s = kt_generate_disk_lut(&kp, c.disk_outer_radius, n, disk.data())) != KT_OK) return s;
    // entries f(r_i)^(1/4), r_i = r_in + i / (n - 1) (r_out - r_in), with their derivatives
    const double m = (double)c.mass, inv_m = 1.0 / m;
    const HD an(th->spin * inv_m, inv_m, 0.0);
    const HD r_in = isco_d(an) * HD(m);
    const HD r_out(th->disk_outer_radius, 0.0, 1.0);
    if (!(r_out.v > r_in.v)) return err_arg("disk outer radius must exceed the ISCO");
    for (uint32_t i = 0; i < n; ++i) {
        const double ratio = (double)i / (double)(n - 1);
        const HD r = r_in + HD(ratio) * (r_out - r_in);
        const HD f = nt_factor_d(r, an, r_in, inv_m);
        double v = 0.0, g0 = 0.0, g1 = 0.0;
        if (f.v > 0.0) {
            v = std::pow(f.v, 0.25);
            const double k = 0.25 * v / f.v;
            g0 = k * f.d[0];
            g1 = k * f.d[1];
        }
        disk_d[i] = v;
        da[i] = g0;
        dro[i] = g1;
    }
    cudaError_t e;
    if ((e = cudaMemcpyAsync(luts.disk, disk.data(), n * sizeof(float), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(luts.disk_d, disk_d.data(), n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(luts.dlut_da, da.data(), n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(luts.dlut_dro, dro.data(), n * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return err_cuda(e, "diff LUT upload");
    // pageable sources: the copies have been staged when cudaMemcpyAsync returns
    sc->bb_lut = d->bb;
    sc->disk_lut = luts.disk;
    sc->bb_tex = 0;
    sc->disk_tex = 0;
    if (c.precision == KT_PREC_FP64) {
        sc->a_d = th->spin;
        sc->aa_d = th->spin * th->spin;
        sc->disk_inner_d = r_in.v;
        sc->disk_outer_d = th->disk_outer_radius;
        sc->temp_scale = (double)d->view.base_temperature_scale * th->temperature_scale;
        sc->disk_lut_d = luts.disk_d;
    }
    kt_camera hc, hd;
    orbit_camera(d->view.observer_r, th->inclination_deg, d->view.azimuth_deg, d->view.fov_deg, &hc, &hd, camd, dcamd);
    *cam = to_dev_camera(hc);
    dl->lut_d = luts.disk_d;
    dl->dlut_da = luts.dlut_da;
    dl->dlut_dro = luts.dlut_dro;
    dl->dr_in_da = r_in.d[0];
    dl->dtemp_ds = d->view.base_temperature_scale;
    return KT_OK;
}

ktd::DiffRecRaw record_of(kt_diff* d) {
    ktd::DiffRecRaw r;
    r.rays = d->rays;
    r.segs = d->segs;
    r.seg_count = d->ctl;
    r.cap = d->cap;
    r.status = d->ctl + 1;
    return r;
}

}  // namespace

extern "C" {

kt_status kt_diff_orbit_camera(float observer_r, float inclination_deg, float azimuth_deg, float fov_deg,
                               kt_camera* cam, kt_camera* dcam_dincl) {
    if (!cam) return err_arg("cam is NULL");
    if (!(observer_r > 0.0f) || !std::isfinite(observer_r)) return err_arg("observer radius must be positive");
    orbit_camera(observer_r, inclination_deg, azimuth_deg, fov_deg, cam, dcam_dincl);
    return KT_OK;
}

kt_status kt_diff_create(const kt_config* cfg, const kt_diff_view* view, uint32_t segment_capacity, int device,
                         kt_diff** out) {
    if (!cfg || !view || !out) return err_arg("NULL argument");
    *out = nullptr;
    if (cfg->mode != KT_MODE_SPEC) return ktd::set_error(KT_ERR_UNSUPPORTED, "diff trace needs stated-physics mode");
    if (cfg->precision != KT_PREC_FP32 && cfg->precision != KT_PREC_FP64)
        return ktd::set_error(KT_ERR_UNSUPPORTED, "diff trace runs in FP32 or FP64");
    if (cfg->spp != 1) return ktd::set_error(KT_ERR_UNSUPPORTED, "diff trace needs spp 1");
    if (cfg->noise_enabled) return ktd::set_error(KT_ERR_UNSUPPORTED, "diff trace needs disk noise off");
    if (!(view->observer_r > 0.0f) || !(view->fov_deg > 0.0f && view->fov_deg < 180.0f) ||
        !std::isfinite(view->base_temperature_scale))
        return err_arg("invalid diff view");
    ktd::Scene probe;
    kt_status s = ktd::scene_from_config(cfg, &probe);
    if (s != KT_OK) return s;
    kt_diff* d = new kt_diff;
    d->device = device;
    d->cfg = *cfg;
    d->view = *view;
    d->n_px = cfg->width * cfg->height;
    d->cap = segment_capacity ? segment_capacity : 4u * d->n_px + 1024u;
    d->seg_bytes = cfg->precision == KT_PREC_FP64 ? sizeof(ktd::DiffSeg<double>) : sizeof(ktd::DiffSeg<float>);
    DevGuard g(device);
    const uint32_t n = cfg->lut_size;
    std::vector<float> bb(4 * (size_t)n);
    if ((s = kt_generate_blackbody_lut(n, cfg->lut_max_temp, cfg->wavelength_start, cfg->wavelength_end,
                                       cfg->wavelength_step, bb.data())) != KT_OK) {
        destroy(d);
        return s;
    }
    cudaError_t e;
    if ((e = cudaMalloc(&d->rays, (size_t)d->n_px * sizeof(ktd::DiffRay))) != cudaSuccess ||
        (e = cudaMalloc(&d->segs, (size_t)d->cap * d->seg_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&d->ctl, 4 * sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMemset(d->ctl, 0, 4 * sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMalloc(&d->bb, (size_t)n * sizeof(float4))) != cudaSuccess ||
        (e = cudaMalloc(&d->work.bucket, (size_t)d->n_px * sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&d->work.order, (size_t)d->n_px * sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMalloc(&d->work.ctl, ktd::kDiffWorkCtl * sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMemcpy(d->bb, bb.data(), bb.size() * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess) {
        destroy(d);
        return err_cuda(e, "diff allocation");
    }
    for (kt_diff_luts* l : {&d->lut_rec, &d->lut_rep}) {
        if ((e = cudaMalloc(&l->disk, n * sizeof(float))) != cudaSuccess ||
            (e = cudaMalloc(&l->disk_d, n * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&l->dlut_da, n * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc(&l->dlut_dro, n * sizeof(double))) != cudaSuccess) {
            destroy(d);
            return err_cuda(e, "diff LUT allocation");
        }
    }
    *out = d;
    return KT_OK;
}

void kt_diff_destroy(kt_diff* d) { destroy(d); }

kt_status kt_diff_forward(kt_diff* d, void* stream, const kt_diff_params* theta, float* hdr_out, uint32_t* err_word) {
    if (!d || !theta || !hdr_out || !err_word) return err_arg("NULL argument");
    DevGuard g(d->device);
    cudaStream_t st = (cudaStream_t)stream;
    ktd::Scene sc;
    ktd::Camera cam;
    ktd::CameraD camd, dcamd;
    ktd::DiffLut dl;
    kt_status s = prepare(d, theta, d->lut_rec, st, &sc, &cam, &camd, &dcamd, &dl);
    if (s != KT_OK) return s;
    cudaError_t e = cudaMemsetAsync(d->ctl, 0, 4 * sizeof(unsigned), st);
    if (e != cudaSuccess) return err_cuda(e, "diff record reset");
    e = ktd::launch_diff_forward(sc, cam, camd, record_of(d), 0, reinterpret_cast<float4*>(hdr_out), nullptr,
                                 err_word, nullptr, st);
    if (e != cudaSuccess) return err_cuda(e, "diff forward launch");
    d->have_record = true;
    d->sc_rec = sc;
    d->sc_rec.max_attempts = 1;  // the backward replays recorded steps: one attempt each
    d->cam_rec = cam;
    d->camd_rec = camd;
    d->dcamd_rec = dcamd;
    d->dl_rec = dl;
    d->theta_rec = *theta;
    return KT_OK;
}

kt_status kt_diff_replay(kt_diff* d, void* stream, const kt_diff_params* theta, float* hdr_out, double* hdr64_out,
                         uint32_t* flags_out, uint32_t* err_word) {
    if (!d || !theta || !hdr_out || !err_word) return err_arg("NULL argument");
    if (!d->have_record) return ktd::set_error(KT_ERR_NOT_READY, "kt_diff_replay needs a kt_diff_forward first");
    DevGuard g(d->device);
    cudaStream_t st = (cudaStream_t)stream;
    ktd::Scene sc;
    ktd::Camera cam;
    ktd::CameraD camd, dcamd;
    ktd::DiffLut dl;
    kt_status s = prepare(d, theta, d->lut_rep, st, &sc, &cam, &camd, &dcamd, &dl);
    if (s != KT_OK) return s;
    sc.max_attempts = 1;
    const cudaError_t e = ktd::launch_diff_forward(sc, cam, camd, record_of(d), 1, reinterpret_cast<float4*>(hdr_out),
                                                   hdr64_out, err_word, flags_out, st);
    if (e != cudaSuccess) return err_cuda(e, "diff replay launch");
    return KT_OK;
}

kt_status kt_diff_replay_fp64(kt_diff* d, void* stream, const kt_diff_params* theta, double* hdr64_out,
                              uint32_t* flags_out, uint32_t* err_word, float* hdr_out) {
    if (!d || !theta || !hdr64_out || !err_word || !hdr_out) return err_arg("NULL argument");
    if (!d->have_record) return ktd::set_error(KT_ERR_NOT_READY, "kt_diff_replay_fp64 needs a kt_diff_forward first");
    DevGuard g(d->device);
    cudaStream_t st = (cudaStream_t)stream;
    ktd::Scene sc;
    ktd::Camera cam;
    ktd::CameraD camd, dcamd;
    ktd::DiffLut dl;
    kt_status s = prepare(d, theta, d->lut_rep, st, &sc, &cam, &camd, &dcamd, &dl, true);
    if (s != KT_OK) return s;
    sc.max_attempts = 1;
    const bool float_records = d->cfg.precision == KT_PREC_FP32;
    const cudaError_t e = ktd::launch_diff_forward(sc, cam, camd, record_of(d), 1, reinterpret_cast<float4*>(hdr_out),
                                                   hdr64_out, err_word, flags_out, st, float_records);
    if (e != cudaSuccess) return err_cuda(e, "diff FP64 replay launch");
    return KT_OK;
}

kt_status kt_diff_backward(kt_diff* d, void* stream, const float* dl_dhdr, double* grad_out) {
    if (!d || !dl_dhdr || !grad_out) return err_arg("NULL argument");
    if (!d->have_record) return ktd::set_error(KT_ERR_NOT_READY, "kt_diff_backward needs a kt_diff_forward first");
    DevGuard g(d->device);
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(grad_out, 0, 4 * sizeof(double), st);
    if (e != cudaSuccess) return err_cuda(e, "gradient reset");
    e = ktd::launch_diff_backward(d->sc_rec, d->cam_rec, d->camd_rec, d->dcamd_rec, record_of(d), d->dl_rec,
                                  reinterpret_cast<const float4*>(dl_dhdr), grad_out, d->work, st);
    if (e != cudaSuccess) return err_cuda(e, "diff backward launch");
    return KT_OK;
}

kt_status kt_diff_backward_fp64(kt_diff* d, void* stream, const float* dl_dhdr, double* grad_out) {
    if (!d || !dl_dhdr || !grad_out) return err_arg("NULL argument");
    if (!d->have_record) return ktd::set_error(KT_ERR_NOT_READY, "kt_diff_backward_fp64 needs a kt_diff_forward first");
    if (d->cfg.precision != KT_PREC_FP32) return kt_diff_backward(d, stream, dl_dhdr, grad_out);
    DevGuard g(d->device);
    cudaStream_t st = (cudaStream_t)stream;
    ktd::Scene sc;
    ktd::Camera cam;
    ktd::CameraD camd, dcamd;
    ktd::DiffLut dl;
    // the recorded point in double: double theta, camera and disk table (uploaded into the
    // replay's tables, like kt_diff_replay_fp64)
    kt_status s = prepare(d, &d->theta_rec, d->lut_rep, st, &sc, &cam, &camd, &dcamd, &dl, true);
    if (s != KT_OK) return s;
    sc.max_attempts = 1;
    cudaError_t e = cudaMemsetAsync(grad_out, 0, 4 * sizeof(double), st);
    if (e != cudaSuccess) return err_cuda(e, "gradient reset");
    e = ktd::launch_diff_backward(sc, cam, camd, dcamd, record_of(d), dl, reinterpret_cast<const float4*>(dl_dhdr),
                                  grad_out, d->work, st, true);
    if (e != cudaSuccess) return err_cuda(e, "diff FP64 backward launch");
    return KT_OK;
}

kt_status kt_diff_get_info(kt_diff* d, kt_diff_info* info) {
    if (!d || !info) return err_arg("NULL argument");
    DevGuard g(d->device);
    unsigned h[2] = {0, 0};
    const cudaError_t e = cudaMemcpy(h, d->ctl, sizeof h, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return err_cuda(e, "diff info");
    info->segments_used = h[0] < d->cap ? h[0] : d->cap;
    info->segments_capacity = d->cap;
    info->overflow_rays = h[1];
    info->record_bytes = (uint64_t)info->segments_used * d->seg_bytes + (uint64_t)d->n_px * sizeof(ktd::DiffRay);
    info->device_bytes = (uint64_t)d->cap * d->seg_bytes + (uint64_t)d->n_px * (sizeof(ktd::DiffRay) + 8) +
                         (uint64_t)d->cfg.lut_size * (sizeof(float4) + 2 * (sizeof(float) + 3 * sizeof(double))) +
                         4 * sizeof(unsigned);
    return KT_OK;
}

}  // extern "C"
