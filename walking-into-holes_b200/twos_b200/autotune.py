"""Autotuner for the walk kernel's launch parameters.

Times a calibration estimate (a seeded random subset of the workload's sites,
the workload's own request with fewer walks) for every candidate setting of

* block size (threads per block): 128, 256, 512;
* queue-refill threshold: idle lanes before a warp refills from the queue;
* step threshold: finished queries before a warp takes its batched step;
* resident blocks per SM (occupancy cap);
* the mixed form's distance-grid threshold (grid spacings a bound must reach
  before a step skips its closest-point query);
* traversal units a lane runs per iteration of the warp loop;
* the mixed form's entry-node start (a query whose initial bound is below one
  entry cell starts at the cell's entry node instead of the BVH root);
* the mixed form's BVH width: the binary BVH or the same BVH collapsed to
  four-wide nodes;
* walks per lane: walks a lane claims from the work queue at once (not
  combined with the four-wide BVH, which the session refuses);

and leaves the fastest (walk-kernel device time per walk: every setting runs
the same walks, and only the grid threshold changes how many steps they
take) set on the mesh.  A grid of at most `max_grid` settings (the default
grid has 864, 576 of them valid; a few seconds of calibration runs) is swept whole, since the
axes interact (the step threshold and the traversal units above all); a
larger one by coordinate descent: from the mesh's current tuning, each axis
in turn takes its fastest value with the others held, until a pass over all
axes changes nothing.  Results can be
cached in a JSON file keyed by the mesh's size and the request's
precision/mode, so a service tunes once per geometry class.
"""
from __future__ import annotations

import itertools
import json
from dataclasses import replace
from pathlib import Path

import numpy as np

from ._abi import TwosError

DEFAULT_GRID = {
    "block": (128, 256, 512),
    "refill": (1, 4),
    "step_threshold": (1, 4),
    "blocks_per_sm": (0,),
    "grid_threshold": (0.1, 0.25),
    "units": (4, 8, 16),
    "entry": (0, 1),
    "bvh_width": (2, 4),
    "lane_walks": (1, 2, 4),
}


def _key(mesh, config) -> str:
    info = mesh.info()
    return f"faces={info['faces']}|precision={config.precision}|mode={config.mode}|green={int(config.green)}"


def autotune(mesh, sites, config, grid=None, calib_sites=4096, calib_walks=128, repeats=2, seed=0,
             cache: str | Path | None = None, cavities=None, search="auto", max_grid=1024, max_passes=4,
             refine=0, refine_sites=32768, refine_walks=512):
    """Pick the fastest launch tuning for `config` on `mesh`; returns
    (best tuning dict, list of (tuning, seconds per walk) for every setting
    timed).  search: "grid" sweeps every setting, "descent" runs coordinate
    descent, "auto" sweeps grids of at most max_grid settings.  refine > 0
    re-times the `refine` fastest settings on a larger calibration
    (refine_sites x refine_walks: a small one is dominated by the tail of
    the launch, where the last walks run on a nearly empty GPU) and picks
    among those; their timings follow the sweep's in the list."""
    key = _key(mesh, config)
    if cache is not None and Path(cache).exists():
        table = json.loads(Path(cache).read_text())
        if key in table:
            mesh.set_tuning(**table[key])
            return table[key], []
    grid = grid or DEFAULT_GRID
    if search not in ("auto", "grid", "descent"):
        raise ValueError(f"unknown search {search!r}")
    sites = np.asarray(sites, dtype=np.float64).reshape(-1, 3)
    rng = np.random.default_rng(seed)
    pick = sites[rng.choice(len(sites), size=min(calib_sites, len(sites)), replace=False)]
    calib = replace(config, walks=min(config.walks, calib_walks))
    names = list(grid)
    results = []
    timed = {}

    def seconds_per_walk(points, cfg):
        times = []
        for r in range(repeats + 1):
            cfg.repeat = 5000 + r
            _, s = mesh.estimate(points, cfg, cavities=cavities)
            if r:  # the first run is a warm-up
                times.append(s["walk_seconds"] / max(1, s["paths"]))
        return float(np.median(times))

    def measure(values):
        if values in timed:
            return timed[values]
        tuning = dict(zip(names, values))
        try:
            mesh.set_tuning(**tuning)
        except TwosError:  # a combination the session refuses (walk claims with the four-wide BVH)
            timed[values] = float("inf")
            return timed[values]
        timed[values] = seconds_per_walk(pick, calib)
        results.append((tuning, timed[values]))
        return timed[values]

    size = int(np.prod([len(grid[n]) for n in names]))
    if search == "grid" or (search == "auto" and size <= max_grid):
        for values in itertools.product(*(grid[n] for n in names)):
            measure(values)
    else:
        start = mesh.get_tuning()
        current = [start[n] if start.get(n) in grid[n] else grid[n][0] for n in names]
        for _ in range(max_passes):
            moved = False
            for i, n in enumerate(names):
                best_v = min(grid[n], key=lambda v: (measure(tuple(current[:i] + [v] + current[i + 1:])),
                                                     v != current[i]))
                if best_v != current[i]:
                    current[i] = best_v
                    moved = True
            if not moved:
                break
    best = min(results, key=lambda t: t[1])[0]
    if refine > 0:
        pick2 = sites[np.random.default_rng(seed + 1).choice(len(sites), size=min(refine_sites, len(sites)),
                                                              replace=False)]
        calib2 = replace(config, walks=min(config.walks, refine_walks))
        refined = []
        for tuning, _ in sorted(results, key=lambda t: t[1])[:refine]:
            mesh.set_tuning(**tuning)
            refined.append((tuning, seconds_per_walk(pick2, calib2)))
        results.extend(refined)
        best = min(refined, key=lambda t: t[1])[0]
    mesh.set_tuning(**best)
    best = mesh.get_tuning()
    if cache is not None:
        table = json.loads(Path(cache).read_text()) if Path(cache).exists() else {}
        table[key] = best
        Path(cache).write_text(json.dumps(table, indent=1, sort_keys=True) + "\n")
    return best, results
