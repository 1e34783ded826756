"""Headless image output on the host (no GPU): the PNG, PPM and PFM writers
and the pixel layout of Loom's path tracers (one thread per pixel, encoded
x << 16 | y as src/smallpt/vm/enc.hpp:30-34 encodes it)."""

import struct
import zlib

import numpy as np
import pytest

from loom_b200 import render as Rd
from loom_b200 import scenes as S


def _img(w, h):
    return np.random.default_rng(1).random((w * h, 3)).astype(np.float32) * 1.5


def test_ppm_header_and_pixels(tmp_path):
    w, h = 5, 3
    img = _img(w, h)
    f = tmp_path / "a.ppm"
    S.write_image(img, w, h, str(f))
    data = f.read_bytes()
    head = f"P6\n{w} {h}\n255\n".encode()
    assert data.startswith(head) and len(data) == len(head) + w * h * 3
    px = np.frombuffer(data[len(head):], dtype=np.uint8).reshape(h, w, 3)
    want = (np.clip(img.reshape(h, w, 3), 0, 1) ** (1 / 2.2) * 255 + 0.5).astype(np.uint8)
    assert np.array_equal(px, want)


def test_pfm_keeps_radiance_bottom_up(tmp_path):
    w, h = 4, 3
    img = _img(w, h)
    f = tmp_path / "a.pfm"
    S.write_image(img, w, h, str(f))
    data = f.read_bytes()
    head = f"PF\n{w} {h}\n-1.0\n".encode()
    assert data.startswith(head) and len(data) == len(head) + w * h * 12
    px = np.frombuffer(data[len(head):], dtype="<f4").reshape(h, w, 3)
    assert np.array_equal(px[::-1].reshape(-1, 3), img)  # unclamped, rows bottom to top


def test_png_is_well_formed(tmp_path):
    w, h = 6, 2
    f = tmp_path / "a.png"
    S.write_image(_img(w, h), w, h, str(f))
    data = f.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    n = struct.unpack(">I", data[8:12])[0]
    assert data[12:16] == b"IHDR" and struct.unpack(">II", data[16:24]) == (w, h)
    crc = struct.unpack(">I", data[16 + n:20 + n])[0]
    assert crc == zlib.crc32(data[12:16 + n]) & 0xFFFFFFFF


def test_unknown_suffix_is_refused(tmp_path):
    with pytest.raises(KeyError):
        S.write_image(_img(2, 2), 2, 2, str(tmp_path / "a.bmp"))


def test_loom_pixel_layout():
    side = 7
    px = Rd.loom_pixels(side)
    assert len(px) == side * side
    x, y = px >> 16, px & 0xFFFF
    # row order: index = y * side + x
    assert np.array_equal(y * side + x, np.arange(side * side))
    # outputs of thread i land at image row y, column x
    outs = [px.astype(np.float32), (px * 2).astype(np.float32), np.zeros(side * side, np.float32)]
    img = Rd.loom_image(outs, side).reshape(side, side, 3)
    assert img[3, 5, 0] == float((5 << 16) | 3) and img[3, 5, 1] == float(2 * ((5 << 16) | 3))
