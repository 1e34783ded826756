"""Headless render: the sphere path tracer on the GPU, written to a PNG file.

Loom's demo shows its renders in an OpenGL viewport (src/smallpt/vm/vm.cpp);
here the image goes to a file instead:

    python -m loom_b200.render --out cornell.png [--width 256 --height 192
                               --spp 16 --seed 1 --mode regroup]

One Loom thread traces one sample; the per-pixel mean is taken over the
samples in sample order (`scenes.pixel_average`).  `--random SEED` renders a
random scene of the batched workload instead of the Cornell box.
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


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--width", type=int, default=256)
    ap.add_argument("--height", type=int, default=192)
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--random", type=int, default=None, help="render a random scene drawn with this seed")
    ap.add_argument("--mode", choices=["plain", "regroup"], default="regroup")
    a = ap.parse_args(argv)
    if a.random is not None:
        req = S.random_request(np.random.default_rng(a.random), seed=a.seed)
        req.width, req.height, req.spp = a.width, a.height, a.spp
    else:
        req = S.cornell_request(a.width, a.height, a.spp, seed=a.seed)
    t0 = time.perf_counter()
    img = render(req, a.mode)
    dt = time.perf_counter() - t0
    S.to_png(img, req.width, req.height, a.out)
    print(f"{a.out}: {req.width}x{req.height}, {req.spp} spp, {req.threads} paths in {dt * 1e3:.1f} ms ({a.mode})")


if __name__ == "__main__":
    main()
