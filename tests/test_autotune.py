"""The autotuner's coordinate search and its tuning file, on the host: the
device timing is replaced by a synthetic cost of the options (no GPU)."""

import json

import pytest

from loom_b200 import autotune as T

SPACE = {"burst": [1, 2, 4, 8], "utr_lanes": [1, 8, 16], "block_size": [128, 256, 512]}
BEST = {"burst": 4, "utr_lanes": 8, "block_size": 256}


def _cost(opts):
    # separable, minimum at BEST
    return 10.0 + sum(abs(SPACE[k].index(opts[k]) - SPACE[k].index(BEST[k])) for k in SPACE)


@pytest.fixture
def fake_timing(monkeypatch):
    timed = []

    def time_launch(fn, reps=2):
        timed.append(fn.opts)
        return _cost(fn.opts)

    monkeypatch.setattr(T, "time_launch", time_launch)
    return timed


def _make_launch(opts):
    fn = lambda: None  # noqa: E731
    fn.opts = dict(opts)
    return fn


def test_coordinate_search_finds_the_optimum(fake_timing):
    seen = []
    res = T.tune(_make_launch, 1 << 20, seed=dict(burst=1, utr_lanes=16, block_size=512), space=SPACE,
                 validate=lambda: seen.append(1))
    assert {k: res["best"][k] for k in SPACE} == BEST
    assert res["ms"] == pytest.approx(10.0)
    # every point timed once, validated once, and reported
    keys = [json.dumps({k: o[k] for k in SPACE}, sort_keys=True) for o in fake_timing]
    assert len(keys) == len(set(keys)) == len(seen) == len(res["points"])
    assert res["msamples_s"] == pytest.approx((1 << 20) / 10.0 / 1e3, rel=1e-3)


def test_several_seeds_keep_the_fastest(fake_timing):
    res = T.tune(_make_launch, 1000, seed=[dict(BEST), dict(burst=8, utr_lanes=1, block_size=128)], space=SPACE)
    assert {k: res["best"][k] for k in SPACE} == BEST


def test_budget_stops_the_search(fake_timing):
    res = T.tune(_make_launch, 1000, seed=dict(burst=1, utr_lanes=1, block_size=128), space=SPACE, budget_s=0.0)
    assert len(res["points"]) == 1  # only the seed point


def test_store_and_lookup(tmp_path, monkeypatch):
    f = tmp_path / "tuning.json"
    monkeypatch.setattr(T, "TUNING_FILE", f)
    assert T.tuned("k") is None
    pts = [{"opts": {"burst": b}, "ms": 10.0 - b, "msamples_s": 1.0} for b in range(20)]
    T.store("k", "pt", {"best": {"burst": 19}, "ms": -9.0, "msamples_s": 1.0, "points": pts}, device="B200")
    T.store("k", "default", {"best": {"burst": 1}, "ms": 9.0, "msamples_s": 1.0, "points": []})
    assert T.tuned("k", "pt") == {"burst": 19}
    assert T.tuned("k", "batch") == {"burst": 1}  # falls back to the kernel's default entry
    entry = json.loads(f.read_text())["k"]["pt"]
    assert len(entry["points"]) == 12 and entry["points"][0]["ms"] == -9.0  # fastest first
    assert entry["device"] == "B200"


def test_constraint_keeps_the_fastest_eligible_point(fake_timing):
    """A constraint (e.g. a minimum lane efficiency) rules points out: the
    search returns the fastest point that meets it, and records the others
    as ineligible."""
    # the optimum (burst 4) is ruled out: the best eligible point is one step away
    res = T.tune(_make_launch, 1000, seed=dict(burst=1, utr_lanes=8, block_size=256), space=SPACE,
                 constraint=lambda o: o["burst"] != 4)
    assert res["best"]["burst"] in (2, 8) and res["ms"] == pytest.approx(11.0)
    assert any(p.get("eligible") is False and p["opts"]["burst"] == 4 for p in res["points"])
    with pytest.raises(RuntimeError):
        T.tune(_make_launch, 1000, seed=dict(BEST), space=SPACE, constraint=lambda o: False)


def test_register_cap_is_a_tuned_option(fake_timing):
    """max_regs is searched like any other option over the caps the caller
    passes (the kernel's compiled caps)."""
    space = dict(SPACE, max_regs=[0, 48, 96])

    def cost(opts):
        return _cost(opts) + {0: 1.0, 48: 0.0, 96: 2.0}[opts["max_regs"]]

    import loom_b200.autotune as TT

    TT.time_launch = lambda fn, reps=2: cost(fn.opts)
    res = T.tune(_make_launch, 1000, seed=dict(BEST, max_regs=0), space=space)
    assert res["best"]["max_regs"] == 48
    assert "max_regs" in T.DEFAULT and T.SPACE["max_regs"] == [0]
