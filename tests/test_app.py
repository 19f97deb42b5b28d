"""The headless parts of the reference's interactive loop (src/app.rs): the re-render policy
(should_render, App::ROTATION_EPSILON / FOV_EPSILON) and the first-frame PNG writer.  CPU only."""
from __future__ import annotations

import struct
import zlib

import numpy as np

import kerrtrace_b200 as kt


def test_should_render_follows_the_app_policy():
    v0 = kt.make_view([0.0, 2.0, 50.0], 10.0, -5.0, 60.0)
    st = kt.ViewState(v0)
    assert st.should_render(v0)                      # no frame yet (app.rs:185-187)
    st.s.has_frame = 1
    assert not st.should_render(v0)
    # rotation within / beyond ROTATION_EPSILON = 1e-4 (app.rs:41,192-196)
    assert not st.should_render(kt.make_view([0.0, 2.0, 50.0], 10.0 + 5e-5, -5.0, 60.0))
    assert st.should_render(kt.make_view([0.0, 2.0, 50.0], 10.0 + 3e-4, -5.0, 60.0))
    assert st.should_render(kt.make_view([0.0, 2.0, 50.0], 10.0, -5.0 - 3e-4, 60.0))
    # fov within / beyond FOV_EPSILON = 1e-4 (app.rs:40,197)
    assert not st.should_render(kt.make_view([0.0, 2.0, 50.0], 10.0, -5.0, 60.0 + 3e-5))
    assert st.should_render(kt.make_view([0.0, 2.0, 50.0], 10.0, -5.0, 60.0 + 2e-3))
    # any position change whose f32 length is above 0 (app.rs:188-191); a difference whose
    # square underflows in f32 has length 0
    assert st.should_render(kt.make_view([0.0, 2.0 + 1e-6, 50.0], 10.0, -5.0, 60.0))
    assert not st.should_render(kt.make_view([1e-30, 2.0, 50.0], 10.0, -5.0, 60.0))


def _chunks(data: bytes):
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, out = 8, []
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        typ = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(typ + body) & 0xffffffff
        out.append((typ, body))
        pos += 12 + n
    return out


def test_first_frame_png_decodes_to_the_frame(tmp_path):
    w, h = 300, 217                                  # > 65535 raw bytes: several stored blocks
    rng = np.random.default_rng(3)
    px = rng.integers(0, 1 << 24, size=w * h, dtype=np.uint32)
    path = tmp_path / "first_frame.png"
    assert kt.write_png(path, px, w, h)
    data = path.read_bytes()
    ch = _chunks(data)
    assert [t for t, _ in ch] == [b"IHDR", b"IDAT", b"IEND"]
    assert struct.unpack(">IIBBBBB", ch[0][1]) == (w, h, 8, 6, 0, 0, 0)
    raw = np.frombuffer(zlib.decompress(ch[1][1]), dtype=np.uint8).reshape(h, 1 + 4 * w)
    assert np.all(raw[:, 0] == 0)
    rgba = raw[:, 1:].reshape(h, w, 4)
    p = px.reshape(h, w)
    assert np.array_equal(rgba[..., 0], (p >> 16) & 0xff)
    assert np.array_equal(rgba[..., 1], (p >> 8) & 0xff)
    assert np.array_equal(rgba[..., 2], p & 0xff)
    assert np.all(rgba[..., 3] == 255)
    # an existing file is left alone (app.rs:221)
    assert not kt.write_png(path, np.zeros(w * h, np.uint32), w, h)
    assert path.read_bytes() == data
