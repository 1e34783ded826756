"""Scene tables for the sphere path-tracing kernel (kernels/sphere_pt.hpp).

A render request is an instance: a resolution, a sample count, a seed, a
camera and a list of spheres.  Many requests are packed into one table of
32-bit words read by the kernel's table op, plus the instance thread offsets
that the engines use to map a thread to (instance, sample index):

  instance header, 16 words at inst * 16:
    0 width  1 height  2 log2(spp)  3 seed  4 first sphere word
    5 sphere count  6..8 camera position (f32)  9 tan(fov / 2) (f32)
  sphere record, 8 words: centre xyz, radius, colour rgb (f32), material
    (u32: 0 diffuse, 1 mirror, 2 glass, 3 emitter)

Instance i owns threads [starts[i], starts[i + 1]); thread j of it traces
sample j % spp of pixel j / spp (pixel = y * width + x).
"""

from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple

import numpy as np

DIFFUSE, MIRROR, GLASS, EMITTER = 0, 1, 2, 3
HEADER_WORDS = 16
SPHERE_WORDS = 8


@dataclasses.dataclass
class Sphere:
    centre: Tuple[float, float, float]
    radius: float
    colour: Tuple[float, float, float]
    material: int


@dataclasses.dataclass
class Request:
    width: int
    height: int
    spp: int
    seed: int
    spheres: List[Sphere]
    camera: Tuple[float, float, float]
    tan_half_fov: float

    @property
    def threads(self) -> int:
        return self.width * self.height * self.spp


def cornell_box() -> List[Sphere]:
    """A Cornell box built from spheres: six walls of radius 1e5 around the
    room [0, 100] x [0, 80] x [0, 160], a mirror ball and a glass ball
    (radius 16.5) on the floor and an emitting sphere sunk into the
    ceiling."""
    R = 1e5
    return [
        Sphere((-R, 40.0, 80.0), R, (0.70, 0.20, 0.20), DIFFUSE),  # left
        Sphere((R + 100.0, 40.0, 80.0), R, (0.20, 0.25, 0.70), DIFFUSE),  # right
        Sphere((50.0, 40.0, -R), R, (0.70, 0.70, 0.70), DIFFUSE),  # back
        Sphere((50.0, 40.0, R + 170.0), R, (0.05, 0.05, 0.05), DIFFUSE),  # front
        Sphere((50.0, -R, 80.0), R, (0.70, 0.70, 0.70), DIFFUSE),  # floor
        Sphere((50.0, R + 80.0, 80.0), R, (0.70, 0.70, 0.70), DIFFUSE),  # ceiling
        Sphere((30.0, 16.5, 55.0), 16.5, (0.95, 0.95, 0.95), MIRROR),
        Sphere((70.0, 16.5, 90.0), 16.5, (0.95, 0.95, 0.95), GLASS),
        Sphere((50.0, 105.0, 80.0), 28.0, (14.0, 14.0, 14.0), EMITTER),  # light
    ]


def cornell_request(width: int = 1024, height: int = 768, spp: int = 64, seed: int = 1) -> Request:
    return Request(width, height, spp, seed, cornell_box(), (50.0, 40.0, 165.0), math.tan(math.radians(25.0)))


def random_request(rng: np.random.Generator, seed: int) -> Request:
    """A render request drawn as in the batched workload: resolution from
    {64, 128, 256, 512}^2, spp from {1, 4, 16, 64}, 8-64 spheres with centres
    uniform in a 100^3 box, radii log-uniform in [2, 30], materials 60%
    diffuse / 20% mirror / 20% glass with albedo uniform in [0.2, 0.9], and
    1-4 of them emitting radiance uniform in [4, 16]."""
    res = int(rng.choice([64, 128, 256, 512]))
    spp = int(rng.choice([1, 4, 16, 64]))
    count = int(rng.integers(8, 65))
    emitters = int(rng.integers(1, 5))
    spheres = []
    for k in range(count):
        c = tuple(float(v) for v in rng.uniform(0.0, 100.0, 3))
        r = float(math.exp(rng.uniform(math.log(2.0), math.log(30.0))))
        if k < emitters:
            e = float(rng.uniform(4.0, 16.0))
            spheres.append(Sphere(c, r, (e, e, e), EMITTER))
            continue
        u = rng.uniform()
        mat = DIFFUSE if u < 0.6 else (MIRROR if u < 0.8 else GLASS)
        a = tuple(float(v) for v in rng.uniform(0.2, 0.9, 3))
        spheres.append(Sphere(c, r, a, mat))
    return Request(res, res, spp, seed, spheres, (50.0, 50.0, 220.0), math.tan(math.radians(22.0)))


def pack(requests: Sequence[Request]) -> Tuple[np.ndarray, np.ndarray]:
    """Returns (table words u32, instance thread offsets u64)."""
    n_inst = len(requests)
    sphere_base = n_inst * HEADER_WORDS
    total_spheres = sum(len(r.spheres) for r in requests)
    words = np.zeros(sphere_base + total_spheres * SPHERE_WORDS, dtype=np.uint32)
    f = words.view(np.float32)
    starts = np.zeros(n_inst + 1, dtype=np.uint64)
    off = sphere_base
    for i, r in enumerate(requests):
        if r.spp & (r.spp - 1):
            raise ValueError("spp must be a power of two")
        h = i * HEADER_WORDS
        words[h + 0] = r.width
        words[h + 1] = r.height
        words[h + 2] = r.spp.bit_length() - 1
        words[h + 3] = r.seed & 0xFFFFFFFF
        words[h + 4] = off
        words[h + 5] = len(r.spheres)
        f[h + 6 : h + 9] = r.camera
        f[h + 9] = r.tan_half_fov
        for s in r.spheres:
            f[off : off + 3] = s.centre
            f[off + 3] = s.radius
            f[off + 4 : off + 7] = s.colour
            words[off + 7] = s.material
            off += SPHERE_WORDS
        starts[i + 1] = starts[i] + r.threads
    return words, starts


def request_words(r: Request) -> Tuple[np.ndarray, np.ndarray]:
    """One request as a server request: its 16-word header with the first
    sphere word (header word 4) relative to the start of its body, and the
    body (its sphere records).  The server adds the body's table position to
    word 4 when it admits the request."""
    words, _ = pack([r])
    header = words[:HEADER_WORDS].copy()
    header[4] = 0
    return header, words[HEADER_WORDS:].copy()


def pixel_average(rgb: Sequence[np.ndarray], spp: int) -> np.ndarray:
    """Per-pixel mean of the per-sample radiance, summed in sample order
    (deterministic); returns (pixels, 3) float32."""
    out = []
    for c in rgb:
        s = np.asarray(c, dtype=np.float32).reshape(-1, spp)
        acc = np.zeros(s.shape[0], dtype=np.float32)
        for j in range(spp):
            acc = acc + s[:, j]
        out.append(acc / np.float32(spp))
    return np.stack(out, axis=1)


def _to_8bit(img: np.ndarray, width: int, height: int) -> np.ndarray:
    px = np.clip(img.reshape(height, width, 3), 0.0, 1.0) ** (1.0 / 2.2)
    return (px * 255.0 + 0.5).astype(np.uint8)


def to_ppm(img: np.ndarray, width: int, height: int, path: str) -> None:
    """Writes a (height*width, 3) linear image as a binary 8-bit PPM (P6),
    the format of Loom's demo output (src/smallpt/common/io.hpp:36-48), with
    the same tone curve as `to_png`."""
    data = _to_8bit(img, width, height)
    with open(path, "wb") as fh:
        fh.write(f"P6\n{width} {height}\n255\n".encode())
        fh.write(data.tobytes())


def to_pfm(img: np.ndarray, width: int, height: int, path: str) -> None:
    """Writes a (height*width, 3) linear image as a little-endian colour PFM
    (float32 radiance, unclamped; rows stored bottom to top as the format
    defines)."""
    data = np.ascontiguousarray(np.asarray(img, dtype="<f4").reshape(height, width, 3)[::-1])
    with open(path, "wb") as fh:
        fh.write(f"PF\n{width} {height}\n-1.0\n".encode())
        fh.write(data.tobytes())


def write_image(img: np.ndarray, width: int, height: int, path: str) -> None:
    """PNG, PPM or PFM by the file's suffix."""
    suffix = str(path).rsplit(".", 1)[-1].lower()
    {"png": to_png, "ppm": to_ppm, "pfm": to_pfm}[suffix](img, width, height, path)


def to_png(img: np.ndarray, width: int, height: int, path: str) -> None:
    """Writes a (height*width, 3) linear image as an 8-bit sRGB-ish PNG."""
    import struct
    import zlib

    data = _to_8bit(img, width, height)
    raw = b"".join(b"\x00" + data[y].tobytes() for y in range(height))

    def chunk(tag: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + tag + body + struct.pack(">I", zlib.crc32(tag + body) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", width, height, 8, 2, 0, 0, 0))
    png += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as fh:
        fh.write(png)
