"""TEST INFRASTRUCTURE: canonical algorithmic bytes per closest-point query.

The roofline of the walk kernel counts, per closest-point query, the bytes a
canonical traversal must read: 32 bytes per AABB test (one FP32 box plus its
child word) and 36 bytes per triangle test (three FP32 vertices), for the
oracle's binary SAH BVH (<= 4 triangles per leaf, nearest-child-first,
pruning boxes whose lower-bound distance is >= the current best).  The counts
are taken at the walk positions of the workload itself (the oracle walks the
GPU's counter stream), over >= 1e5 queries.

    python oracle/canonical_bytes.py [--sites 96] [--walks 64]

prints one JSON object; bench.py carries the resulting constant.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / "walking-into-holes_b200"))

import oracle  # noqa: E402
from twos_b200 import geometry  # noqa: E402


def noise_sphere_sites(seed_mesh=1, n_grid=64, count=96, seed=7):
    """Grid cell centres of the level-7 noise sphere's box inside the surface
    (star-shaped: |x| below 0.98 of the displaced radius along x's direction)."""
    V, F = geometry.noise_sphere(7, seed_mesh)
    pts = geometry.grid_points(V.min(0), V.max(0), n_grid)
    r = np.linalg.norm(pts, axis=1)
    keep = r > 1e-9
    pts = pts[keep]
    r = r[keep]
    rad = 1.0 + 0.15 * geometry.sh_field(pts / r[:, None], seed_mesh)
    inside = pts[r < 0.98 * rad]
    rng = np.random.default_rng(seed)
    return V, F, inside[rng.choice(len(inside), size=min(count, len(inside)), replace=False)], len(inside)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sites", type=int, default=96)
    ap.add_argument("--walks", type=int, default=64)
    a = ap.parse_args()
    oracle.build()
    V, F, sites, n_inside = noise_sphere_sites(count=a.sites)
    m = oracle.OracleMesh(V, F)
    t = time.time()
    out = m.walk_samples(sites, rng=oracle.RNG_COUNTER, walks=a.walks, seed=20260912, epsilon=1e-4,
                         max_steps=4096, source=[oracle.term(oracle.TERM_CONST, 1.0)], weight_order=1,
                         count_tests=True, query_radius=np.inf)
    queries = int(out["steps"].sum() + out["steps"].size)
    aabb = int(out["aabb_tests"].sum())
    tri = int(out["tri_tests"].sum())
    nodes, depth = m.bvh_info()
    res = {
        "workload": "noise sphere L7 (327,680 tris), f=1, eps=1e-4, counter stream",
        "sites": len(sites), "walks": a.walks, "queries": queries,
        "mean_steps": float(out["steps"].mean()),
        "aabb_tests_per_query": aabb / queries, "tri_tests_per_query": tri / queries,
        "bytes_per_query": (32 * aabb + 36 * tri) / queries,
        "canonical_bvh_nodes": nodes, "canonical_bvh_depth": depth,
        "grid_sites_inside_estimate": n_inside, "seconds": time.time() - t,
    }
    print(json.dumps(res))


if __name__ == "__main__":
    main()
