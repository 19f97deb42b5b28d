// kt_app.cpp — the parts of the reference's interactive loop that a headless host still needs:
// the re-render policy (src/app.rs:157-198) and the first-frame writer (src/app.rs:219-236).
//
// The policy compares the current view with the last submitted one in f32, as the app does
// with glam: a position change counts when the length of the difference is above 0, a yaw,
// pitch or fov change when it exceeds 1e-4 (App::ROTATION_EPSILON, App::FOV_EPSILON,
// src/app.rs:40-41).  The writer turns 0x00RRGGBB words into RGBA8 with alpha 255, as the app
// does before image::save_buffer; the PNG it writes uses stored (uncompressed) deflate blocks,
// so it needs no compression library and decodes to the same pixels.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/kerrtrace.h"
#include "kt_internal.h"

namespace {

kt_status app_fail(kt_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return ktd::set_error(s, buf);
}

constexpr float kRotationEpsilon = 1e-4f;
constexpr float kFovEpsilon = 1e-4f;

// CRC-32 of the PNG chunks (ISO 3309 / ITU-T V.42 polynomial, reflected: 0xEDB88320).
struct CrcTable {
    uint32_t t[256];
    CrcTable() {
        for (uint32_t n = 0; n < 256; ++n) {
            uint32_t c = n;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[n] = c;
        }
    }
};

uint32_t crc_update(uint32_t crc, const uint8_t* p, size_t n) {
    static const CrcTable table;
    for (size_t i = 0; i < n; ++i) crc = table.t[(crc ^ p[i]) & 0xffu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<uint8_t>& out, uint32_t v) {
    out.push_back((uint8_t)(v >> 24));
    out.push_back((uint8_t)(v >> 16));
    out.push_back((uint8_t)(v >> 8));
    out.push_back((uint8_t)v);
}

void put_chunk(std::vector<uint8_t>& out, const char type[4], const std::vector<uint8_t>& data) {
    put_be32(out, (uint32_t)data.size());
    const size_t start = out.size();
    out.insert(out.end(), type, type + 4);
    out.insert(out.end(), data.begin(), data.end());
    const uint32_t crc = crc_update(0xffffffffu, out.data() + start, out.size() - start) ^ 0xffffffffu;
    put_be32(out, crc);
}

}  // namespace

extern "C" {

kt_status kt_view_state_init(kt_view_state* s, const kt_view* initial) {
    if (!s || !initial) return app_fail(KT_ERR_INVALID_ARG, "NULL argument");
    s->prev = *initial;
    s->has_frame = 0;
    return KT_OK;
}

int32_t kt_should_render(const kt_view_state* s, const kt_view* v) {
    if (!s || !v) return -1;
    if (!s->has_frame) return 1;
    // (cam_pos - prev_cam_pos).length() > 0.0 (glam f32: sqrt of the dot product)
    const float dx = v->cam_pos[0] - s->prev.cam_pos[0];
    const float dy = v->cam_pos[1] - s->prev.cam_pos[1];
    const float dz = v->cam_pos[2] - s->prev.cam_pos[2];
    const float len = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (len > 0.0f) return 1;
    if (std::fabs(v->yaw_deg - s->prev.yaw_deg) > kRotationEpsilon ||
        std::fabs(v->pitch_deg - s->prev.pitch_deg) > kRotationEpsilon)
        return 1;
    return std::fabs(v->fov_deg - s->prev.fov_deg) > kFovEpsilon ? 1 : 0;
}

kt_status kt_renderer_submit_view(kt_renderer* r, kt_view_state* s, const kt_view* v, int32_t* submitted) {
    if (!r || !s || !v) return app_fail(KT_ERR_INVALID_ARG, "NULL argument");
    if (submitted) *submitted = 0;
    if (kt_should_render(s, v) != 1) return KT_OK;
    float fwd[3], rgt[3], up[3];
    kt_status st = kt_camera_basis(v->yaw_deg, v->pitch_deg, fwd, rgt, up);
    if (st != KT_OK) return st;
    int32_t sub = 0;
    st = kt_renderer_submit_render(r, v->cam_pos, fwd, rgt, up, kt_fov_scale(v->fov_deg), &sub);
    if (st != KT_OK) return st;
    if (sub) {
        s->has_frame = 1;
        s->prev = *v;
    }
    if (submitted) *submitted = sub;
    return KT_OK;
}

kt_status kt_write_png(const char* path, const uint32_t* pixels, uint32_t width, uint32_t height,
                       int32_t* written) {
    if (written) *written = 0;
    if (!path || !pixels) return app_fail(KT_ERR_INVALID_ARG, "NULL argument");
    if (width == 0 || height == 0 || width > (1u << 24) || height > (1u << 24))
        return app_fail(KT_ERR_INVALID_ARG, "bad image size %ux%u", width, height);
    if (FILE* probe = std::fopen(path, "rb")) {  // `if !path.exists()` (src/app.rs:221)
        std::fclose(probe);
        return KT_OK;
    }
    // scanlines: filter type 0, then RGBA8
    const size_t row = (size_t)width * 4 + 1;
    std::vector<uint8_t> raw(row * height);
    for (uint32_t y = 0; y < height; ++y) {
        uint8_t* o = raw.data() + y * row;
        o[0] = 0;
        const uint32_t* in = pixels + (size_t)y * width;
        for (uint32_t x = 0; x < width; ++x) {
            const uint32_t p = in[x];
            o[1 + 4 * x] = (uint8_t)((p >> 16) & 0xffu);
            o[2 + 4 * x] = (uint8_t)((p >> 8) & 0xffu);
            o[3 + 4 * x] = (uint8_t)(p & 0xffu);
            o[4 + 4 * x] = 255;
        }
    }
    // zlib stream (RFC 1950): header 78 01, stored deflate blocks (RFC 1951, BTYPE 00, at most
    // 65535 bytes each), Adler-32 of the raw data
    std::vector<uint8_t> z;
    z.reserve(raw.size() + raw.size() / 65535 * 5 + 16);
    z.push_back(0x78);
    z.push_back(0x01);
    size_t pos = 0;
    do {
        const size_t n = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + n == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)(n & 0xffu));
        z.push_back((uint8_t)(n >> 8));
        z.push_back((uint8_t)(~n & 0xffu));
        z.push_back((uint8_t)((~n >> 8) & 0xffu));
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + n);
        pos += n;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;
    for (size_t i = 0; i < raw.size(); ++i) {
        a = (a + raw[i]) % 65521u;
        b = (b + a) % 65521u;
    }
    put_be32(z, (b << 16) | a);

    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, width);
    put_be32(ihdr, height);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(6);  // colour type: RGBA
    ihdr.push_back(0);  // deflate
    ihdr.push_back(0);  // adaptive filtering
    ihdr.push_back(0);  // no interlace
    put_chunk(out, "IHDR", ihdr);
    put_chunk(out, "IDAT", z);
    put_chunk(out, "IEND", {});
    FILE* f = std::fopen(path, "wb");
    if (!f) return app_fail(KT_ERR_INVALID_ARG, "cannot open %s for writing", path);
    const size_t put = std::fwrite(out.data(), 1, out.size(), f);
    const int closed = std::fclose(f);
    if (put != out.size() || closed != 0) return app_fail(KT_ERR_INVALID_ARG, "short write to %s", path);
    if (written) *written = 1;
    return KT_OK;
}

}  // extern "C"
