"""Headless render: a path tracer on the GPU, written to an image file.

Loom's demo shows its renders in an OpenGL viewport (src/smallpt/vm/vm.cpp)
and can dump them as PPM (src/smallpt/common/io.hpp:36-48); here the image
goes to a file only, PNG, PPM or PFM by its suffix:

    python -m loom_b200.render --out cornell.png [--width 256 --height 192
                               --spp 16 --seed 1 --mode regroup]
    python -m loom_b200.render --kernel pt_const_512 --out loom.pfm

The sphere path tracer (`sphere_pt_f32`, the default) runs one Loom thread
per sample; the per-pixel mean is taken over the samples in sample order
(`scenes.pixel_average`).  `--random SEED` renders a random scene of the
batched workload instead of the Cornell box.  Loom's own path tracers
(`pt_const_*`, `pt2_const_*`, `primary_const_*`; square images of the side
in the name) run one thread per pixel, as Loom's demo does, with the pixel
encoded x << 16 | y (src/smallpt/vm/enc.hpp:30-34); their outputs are the
pixel's radiance.
"""

from __future__ import annotations

import argparse
import time

import numpy as np

from . import api
from . import scenes as S


def render(req: S.Request, mode: str = "regroup", **opts) -> np.ndarray:
    """Radiance per pixel, (height * width, 3) float32, row order."""
    table, starts = S.pack([req])
    n = req.threads
    with api.Function("sphere_pt_f32", n, mode, **opts) as f:
        rgb = f.launch_host([api.Instance(), api.LocalIota()], n, instance_starts=starts, table=table)
        f.stats(raise_on_device_error=True)
    return S.pixel_average(rgb, req.spp)


LOOM_KERNELS = ("pt_const_", "pt2_const_", "primary_const_")


def loom_pixels(side: int) -> np.ndarray:
    """Every pixel of a side x side render in row order, encoded as Loom's
    demo encodes them (x << 16 | y)."""
    x, y = np.meshgrid(np.arange(side, dtype=np.uint32), np.arange(side, dtype=np.uint32))
    return ((x << 16) | y).reshape(-1)


def loom_image(outputs, side: int) -> np.ndarray:
    """(side*side, 3) float32 radiance, row y = pixel y, from the first three
    outputs of one of Loom's path tracers run over `loom_pixels(side)`."""
    return np.stack([np.asarray(o, dtype=np.float32) for o in outputs[:3]], axis=1).reshape(side * side, 3)


def render_loom(kernel: str, mode: str = "plain", **opts):
    """Renders one of Loom's path tracers; returns (image, side)."""
    side = int(kernel.rsplit("_", 1)[1])
    px = loom_pixels(side)
    with api.Function(kernel, len(px), mode, **opts) as f:
        outs = f(px)
        f.stats(raise_on_device_error=True)
    return loom_image(outs, side), side


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--height", type=int, default=192)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--random", type=int, default=None, help="render a random scene drawn with this seed")
    ap.add_argument("--mode", choices=["plain", "regroup"], default=None,
                    help="engine (default: regroup for the sphere path tracer, plain for Loom's)")
    ap.add_argument("--kernel", default="sphere_pt_f32",
                    help="sphere_pt_f32, or one of Loom's compiled path tracers (pt_const_40, pt2_const_512, primary_const_256, ...)")
    a = ap.parse_args(argv)
    if a.kernel.startswith(LOOM_KERNELS):
        mode = a.mode or "plain"
        t0 = time.perf_counter()
        img, side = render_loom(a.kernel, mode)
        dt = time.perf_counter() - t0
        S.write_image(img, side, side, a.out)
        print(f"{a.out}: {a.kernel}, {side}x{side} pixels in {dt * 1e3:.1f} ms ({mode})")
        return
    if a.kernel != "sphere_pt_f32":
        raise SystemExit(f"--kernel {a.kernel}: not a path tracer this tool renders")
    a.mode = a.mode or "regroup"
    if a.random is not None:
        req = S.random_request(np.random.default_rng(a.random), seed=a.seed)
        req.width, req.height, req.spp = a.width, a.height, a.spp
    else:
        req = S.cornell_request(a.width, a.height, a.spp, seed=a.seed)
    t0 = time.perf_counter()
    img = render(req, a.mode)
    dt = time.perf_counter() - t0
    S.write_image(img, req.width, req.height, a.out)
    print(f"{a.out}: {req.width}x{req.height}, {req.spp} spp, {req.threads} paths in {dt * 1e3:.1f} ms ({a.mode})")


if __name__ == "__main__":
    main()
