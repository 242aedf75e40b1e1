"""Frames and state files: the recorder that replaces the reference's OpenCV
PNG writer (src/wrappers.cuh:147-152, 253-260, 323-345) and the binary state
dump/resume.  Frames are decoded here with zlib and compared with a numpy
rendering of the same density (min..max stretched to 0..255, viridis by
linear interpolation between its ten stops)."""
import os
import struct
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VIRIDIS = np.array([[68, 1, 84], [72, 40, 120], [62, 73, 137], [49, 104, 142], [38, 130, 142],
                    [31, 158, 137], [53, 183, 121], [110, 206, 88], [181, 222, 43], [253, 231, 37]], float)


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, chunks = 8, {}
    while pos < len(data):
        n, = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc, = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert crc == zlib.crc32(kind + body) & 0xFFFFFFFF, kind
        chunks[kind] = chunks.get(kind, b"") + body
        pos += 12 + n
    w, h, depth, ctype = struct.unpack(">IIBB", chunks[b"IHDR"][:10])
    assert (depth, ctype) == (8, 2)
    raw = zlib.decompress(chunks[b"IDAT"])  # checks the Adler-32 too
    rows = np.frombuffer(raw, np.uint8).reshape(h, 3 * w + 1)
    assert np.all(rows[:, 0] == 0)
    return rows[:, 1:].reshape(h, w, 3)


def render(rho):
    v = rho.astype(np.float32).astype(np.float64)
    lo, hi = v.min(), v.max()
    scale = 255.0 / (hi - lo) if hi > lo else 0.0
    level = np.clip(np.rint(v * scale - lo * scale), 0, 255)
    pos = level * 9.0 / 255.0
    s = np.minimum(pos.astype(int), 8)
    f = (pos - s)[..., None]
    return np.rint(VIRIDIS[s] + f * (VIRIDIS[s + 1] - VIRIDIS[s])).astype(np.uint8)


def handle(pkg, n=64, m=48, strategy=0, precision=0, t_end=0.05):
    h = pkg.Handle(n, m)
    h.configure(1.0, 1.0, t_end, 0.45, 1.9, 1.4, strategy, precision)
    h.set_state(pkg.scenarios.seeded_four_quadrant(n, m, 21))
    return h


@pytest.mark.parametrize("precision", [0, 3])
def test_frame_matches_numpy_rendering(pkg, tmp_path, precision):
    h = handle(pkg, precision=precision)
    h.advance(20)
    p = str(tmp_path / "f.png")
    h.write_frame_png(p)
    img = read_png(p)
    want = render(h.get_state(4)[..., 0])
    h.close()
    assert img.shape == want.shape
    d = np.abs(img.astype(int) - want.astype(int))
    assert d.max() <= 3 and (d == 0).mean() > 0.99  # a level can differ where v*scale+shift is a rounding tie


def test_recording_writes_the_reference_frames_and_changes_nothing(pkg, tmp_path):
    plain = handle(pkg)
    plain.solve()
    steps = plain.time()[1]
    U_plain = plain.get_state(4)
    plain.close()
    h = handle(pkg)
    rec = tmp_path / "frames"
    h.set_record_model(True, 7, str(rec))
    h.solve()
    assert h.time()[1] == steps
    assert np.array_equal(h.get_state(4), U_plain)
    names = sorted(os.listdir(rec), key=lambda x: int(x.split(".")[0]))
    assert names == [f"{k}.png" for k in range(0, steps, 7)]  # after step k (from 0), every 7 steps
    last = (steps - 1) // 7 * 7
    if last == steps - 1:  # the last frame is of the final state
        assert np.array_equal(read_png(str(rec / f"{last}.png")), render(U_plain[..., 0]))
    h.close()


def test_solver_mirror_records(pkg, tmp_path):
    s = pkg.RGRP_2D_CUDA(pkg.scenarios.seeded_four_quadrant(40, 40, 3))
    s.setSpatialLayout(1.0, 1.0)
    s.setTimeLayout(0.02, 0.45)
    s.setRecordModel(True, 5, str(tmp_path))
    s.solve()
    n = s.getTimeStagesCount()
    assert sorted(os.listdir(tmp_path), key=lambda x: int(x.split(".")[0])) == [f"{k}.png" for k in range(0, n, 5)]


def test_state_file_resumes_a_run(pkg, tmp_path):
    a = handle(pkg, t_end=0.2)
    a.advance(15)
    p = str(tmp_path / "state.bin")
    a.write_state(p)
    b = handle(pkg, t_end=0.2)
    b.read_state(p)
    assert b.time()[:2] == a.time()[:2]
    a.advance(10)
    b.advance(10)
    assert b.time()[:2] == a.time()[:2]
    assert np.array_equal(a.get_state(4), b.get_state(4))
    c = pkg.Handle(32, 32)
    with pytest.raises(pkg.FVM2DError):
        c.read_state(p)
    a.close(); b.close(); c.close()
