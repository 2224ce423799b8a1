"""The autotuner's host logic without a GPU: a stand-in mesh answers each
calibration estimate with a walk-kernel time that depends on the tuning, so
the sweep, the warm-up rule, the objective (seconds per walk, since the grid
threshold changes the step count but not the walks) and the JSON cache can be
checked exactly."""
import json
from dataclasses import dataclass, field

import numpy as np

from twos_b200.autotune import DEFAULT_GRID, autotune


@dataclass
class Cfg:
    walks: int = 512
    precision: str = "mixed"
    mode: str = "compliance"
    green: bool = False
    repeat: int = 0


@dataclass
class FakeMesh:
    tuning: dict = field(default_factory=dict)
    calls: list = field(default_factory=list)

    def info(self):
        return {"faces": 1234}

    def set_tuning(self, **t):
        self.tuning = dict(t)

    def get_tuning(self):
        return dict(self.tuning)

    def estimate(self, sites, cfg, cavities=None):
        t = self.tuning
        self.calls.append((dict(t), cfg.walks, cfg.repeat, len(sites)))
        paths = len(sites) * cfg.walks
        # Fastest at block 256, step threshold 4, 8 units, grid 0.1; a low grid
        # threshold adds steps (queries) but fewer seconds per walk.
        per_walk = (1.0 + 0.1 * abs(t["block"] - 256) / 128 + 0.05 * (t["step_threshold"] != 4)
                    + 0.02 * abs(t["units"] - 8) / 4 + 0.3 * t["grid_threshold"] + 0.01 * (t["refill"] != 1)
                    + 0.1 * (t.get("entry", 1) != 1) + 0.05 * (t.get("bvh_width", 2) != 4)
                    + 0.03 * abs(t.get("lane_walks", 1) - 2))
        steps = paths * (30 if t["grid_threshold"] < 0.2 else 25)
        if cfg.repeat == 5000:  # the warm-up run is slow and must be ignored
            per_walk *= 100
        return None, {"walk_seconds": per_walk * paths * 1e-9, "paths": paths, "queries": steps + paths}


SMALL_GRID = {"block": (128, 256), "refill": (1, 4), "step_threshold": (1, 4), "blocks_per_sm": (0,),
              "grid_threshold": (0.1, 0.25), "units": (8,), "entry": (0, 1), "bvh_width": (2, 4),
              "lane_walks": (1, 2)}


def test_autotune_sweeps_a_small_grid_whole_and_picks_the_fastest(tmp_path):
    mesh = FakeMesh()
    sites = np.random.default_rng(0).normal(size=(10_000, 3))
    cache = tmp_path / "tuning.json"
    best, results = autotune(mesh, sites, Cfg(), grid=SMALL_GRID, calib_sites=100, calib_walks=64, repeats=2,
                             cache=cache)
    assert len(results) == np.prod([len(v) for v in SMALL_GRID.values()])
    assert best == {"block": 256, "refill": 1, "step_threshold": 4, "blocks_per_sm": 0, "grid_threshold": 0.1,
                    "units": 8, "entry": 1, "bvh_width": 4, "lane_walks": 2}
    assert mesh.get_tuning() == best
    # Calibration: a seeded subset of the sites, the request's walks capped, one warm-up plus two timed runs.
    assert all(n == 100 and w == 64 for _, w, _, n in mesh.calls)
    assert len(mesh.calls) == 3 * len(results)
    # Cached by mesh size and request shape; a second call reads the cache and runs nothing.
    table = json.loads(cache.read_text())
    assert list(table.values()) == [best]
    mesh2 = FakeMesh()
    again, cached = autotune(mesh2, sites, Cfg(), cache=cache)
    assert again == best and cached == [] and mesh2.calls == [] and mesh2.get_tuning() == best
    # Another precision is another key.
    mesh3 = FakeMesh()
    _, res3 = autotune(mesh3, sites, Cfg(precision="fp64"), grid=SMALL_GRID, calib_sites=50, calib_walks=32,
                       repeats=1, cache=cache)
    assert res3 and len(json.loads(cache.read_text())) == 2


def test_autotune_descends_the_default_grid_to_the_separable_optimum():
    """Coordinate descent over the default grid (864 settings) from the
    mesh's current tuning: the stand-in cost is separable, so descent reaches
    the grid's optimum, timing each setting once; the default sweeps the grid
    whole and agrees."""
    full = int(np.prod([len(v) for v in DEFAULT_GRID.values()]))
    assert full == 864
    mesh = FakeMesh(tuning={"block": 128, "refill": 4, "step_threshold": 1, "blocks_per_sm": 0,
                            "grid_threshold": 0.25, "units": 4, "entry": 0, "bvh_width": 2, "lane_walks": 1})
    sites = np.random.default_rng(1).normal(size=(1000, 3))
    best, results = autotune(mesh, sites, Cfg(), calib_sites=100, calib_walks=64, repeats=1, search="descent")
    assert best == {"block": 256, "refill": 1, "step_threshold": 4, "blocks_per_sm": 0, "grid_threshold": 0.1,
                    "units": 8, "entry": 1, "bvh_width": 4, "lane_walks": 2}
    keys = [tuple(sorted(t.items())) for t, _ in results]
    assert len(set(keys)) == len(keys) and len(keys) < 64
    # The exhaustive sweep of the same grid agrees.
    mesh2 = FakeMesh()
    best2, results2 = autotune(mesh2, sites, Cfg(), calib_sites=20, calib_walks=8, repeats=1)
    assert best2 == best and len(results2) == full


def test_autotune_rejects_an_unknown_search():
    import pytest
    with pytest.raises(ValueError):
        autotune(FakeMesh(), np.zeros((4, 3)), Cfg(), search="random")


def test_autotune_skips_settings_the_session_refuses():
    """Walk claims with the four-wide BVH are refused by the session
    (TwosError from set_tuning): the sweep skips them and picks a valid one."""
    from twos_b200._abi import TwosError

    class Refusing(FakeMesh):
        def set_tuning(self, **t):
            if t.get("bvh_width") == 4 and t.get("lane_walks", 1) > 1:
                raise TwosError(2, "invalid tuning")
            super().set_tuning(**t)

    mesh = Refusing()
    best, results = autotune(mesh, np.zeros((50, 3)), Cfg(), grid=SMALL_GRID, calib_sites=10, calib_walks=8,
                             repeats=1)
    assert all(not (t["bvh_width"] == 4 and t["lane_walks"] > 1) for t, _ in results)
    assert len(results) == np.prod([len(v) for v in SMALL_GRID.values()]) * 3 // 4
    assert not (best["bvh_width"] == 4 and best["lane_walks"] > 1)


def test_refine_stage_retimes_the_fastest_on_a_larger_calibration():
    """refine=k: the k fastest settings of the sweep are timed again on a
    larger calibration (more sites and walks) and the pick comes from those
    timings; here the larger calibration reverses the sweep's order."""
    class TailHeavy(FakeMesh):
        def estimate(self, sites, cfg, cavities=None):
            rows, s = super().estimate(sites, cfg, cavities)
            if len(sites) > 100 and self.tuning["units"] == 8:  # slower at scale
                s["walk_seconds"] *= 2.0
            return rows, s

    mesh = TailHeavy()
    sites = np.random.default_rng(2).normal(size=(5000, 3))
    grid = dict(SMALL_GRID, units=(4, 8), block=(256,), refill=(1,), step_threshold=(4,), grid_threshold=(0.1,),
                entry=(1,), bvh_width=(4,), lane_walks=(2,))
    best, results = autotune(mesh, sites, Cfg(walks=4096), grid=grid, calib_sites=50, calib_walks=16, repeats=1,
                             refine=2, refine_sites=1000, refine_walks=256)
    sweep, refined = results[:2], results[2:]
    assert min(sweep, key=lambda t: t[1])[0]["units"] == 8  # the small calibration prefers 8 units
    assert len(refined) == 2 and best["units"] == 4
    big = [c for c in mesh.calls if c[3] == 1000]
    assert len(big) == 2 * 2 and all(w == 256 for _, w, _, _ in big)
