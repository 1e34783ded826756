"""Shared pytest configuration: the `gpu` marker and import paths."""

import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden_extra():
    """Table and instance offsets of a golden fixture (None when absent)."""
    import numpy as np

    def load(name):
        z = np.load(ROOT / "tests" / "golden" / f"{name}.npz")
        return {k: z[k] for k in ("table", "starts") if k in z.files}

    return load


@pytest.fixture(scope="session")
def golden():
    """Loads tests/golden/<kernel>.npz as (inputs, outputs)."""
    import numpy as np

    cache = {}

    def load(name):
        if name not in cache:
            z = np.load(ROOT / "tests" / "golden" / f"{name}.npz")
            ins = [z[f"in{i}"] for i in range(sum(1 for k in z.files if k.startswith("in")))]
            outs = [z[f"out{i}"] for i in range(sum(1 for k in z.files if k.startswith("out")))]
            cache[name] = (ins, outs)
        return cache[name]

    return load
