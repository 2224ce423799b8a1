"""The mixed form's distance-bound grid (built at mesh open, used by the walk
step when the bound clears grid_threshold spacings).

* The bound never exceeds the FP64 distance to the surface (inside, outside
  and near the surface), and is tight: at least d - sqrt(3) h - 3 delta - h/128
  at every point inside the grid (the bound is the best of the cell's eight
  corners, the nearest of which is within sqrt(3) h / 2; the distance is
  1-Lipschitz; the stored value is the FP32 distance less 2 delta rounded
  down to h/128).
* The grid is sized from the triangle count (128 vertices per triangle, at
  most 2^25) and TWOS_GRID_VERTICES=0 builds none.
* Walks with grid steps estimate the same field: on the unit ball the mixed
  form with the grid agrees with the analytic u and with the grid-off run
  within the Monte Carlo error, and the grid answers a good share of steps.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


def test_bound_is_a_lower_bound_and_tight(tb):
    V, F = tb.geometry.noise_sphere(5, 1)
    rng = np.random.default_rng(0)
    with tb.Mesh(V, F) as mesh:
        info = mesh.info()
        h, delta = info["grid_spacing"], info["mixed_delta"]
        assert h > 0 and np.prod(info["grid_dims"]) <= 1024 * len(F) * 1.5
        lo, hi = np.array(info["bounds_min"]), np.array(info["bounds_max"])
        far = rng.uniform(lo - 0.5 * h, hi + 0.5 * h, (200_000, 3))
        near = V[rng.integers(0, len(V), 100_000)] * (1 + rng.uniform(-3 * h, 3 * h, (100_000, 1)))
        pts = np.concatenate([far, near])
        d = mesh.closest_point(pts, precision="fp64", with_points=False)
        b = mesh.distance_bound(pts)
        # The grid spans the bounding box padded by one spacing.
        covered = np.all((pts >= lo - 0.9 * h) & (pts <= hi + 0.9 * h), axis=1)
        assert np.isfinite(b[covered]).all() and covered.sum() > 250_000
        ok = np.isfinite(b)
        assert np.all(b[ok] <= d[ok]), (b[ok] - d[ok]).max()
        assert np.all(b[ok] >= d[ok] - np.sqrt(3) * h - 3 * delta - h / 128 - 1e-12), (d[ok] - b[ok]).max()
        out = mesh.distance_bound(np.array([[lo[0] - 5 * h, 0.0, 0.0]]))
        assert np.isnan(out[0])


def test_grid_size_and_switch(tb, monkeypatch):
    V, F = tb.geometry.icosphere(3)
    with tb.Mesh(V, F) as mesh:
        dims = mesh.info()["grid_dims"]
        assert 4096 <= np.prod(dims) <= 1.5 * 1024 * len(F)
    monkeypatch.setenv("TWOS_GRID_VERTICES", "0")
    with tb.Mesh(V, F) as mesh:
        assert mesh.info()["grid_dims"] == [0, 0, 0]
        assert np.isnan(mesh.distance_bound(np.zeros((1, 3)))[0])
        _, s = mesh.estimate(np.zeros((1, 3)), tb.Config(walks=64, precision="mixed", source=tb.sources.constant(1.0)))
        assert s["grid_steps"] == 0


def test_grid_walks_estimate_the_same_field(tb):
    V, F = tb.geometry.icosphere(5)
    sites = tb.geometry.uniform_ball(64, 0.9, seed=4)
    u_exact = (1.0 - np.sum(sites ** 2, axis=1)) / 6.0
    cfg = tb.Config(walks=2048, precision="mixed", seed=9, epsilon=1e-4, source=tb.sources.constant(1.0))
    with tb.Mesh(V, F) as mesh:
        on, s_on = mesh.estimate(sites, cfg)
        on_smp = mesh.walk_samples(sites, cfg)
        mesh.set_tuning(grid_threshold=0)
        off, s_off = mesh.estimate(sites, cfg)
    assert s_off["grid_steps"] == 0
    assert s_on["grid_steps"] > 0.2 * s_on["steps"]
    assert s_on["caps"] == s_off["caps"] == 0
    se = on_smp["u"].std(axis=1, ddof=1) / np.sqrt(cfg.walks)
    z = (on["u"] - u_exact) / se
    assert np.max(np.abs(z)) < 4.5 and np.mean(np.abs(z) < 3) >= 0.95
    zz = (on["score"] - off["score"]) / np.hypot(on["score_se"], off["score_se"])
    assert np.max(np.abs(zz)) < 4.5 and abs(np.mean(zz)) < 0.5
    # Same variance per walk: the grid changes the radii, not the estimator.
    assert 0.8 < np.median(on["score_se"] / off["score_se"]) < 1.25


def test_fp64_form_with_the_grid_estimates_the_same_field(tb):
    """grid_fp64 = 1 gives the FP64 compliance form the mixed form's grid steps
    and entry nodes (a comparison of precision alone): its walks take other
    radii than the plain FP64 form's, so the two agree within the Monte Carlo
    error, and both agree with the analytic u on the unit ball."""
    V, F = tb.geometry.icosphere(5)
    sites = tb.geometry.uniform_ball(64, 0.9, seed=6)
    u_exact = (1.0 - np.sum(sites ** 2, axis=1)) / 6.0
    cfg = tb.Config(walks=2048, precision="fp64", seed=19, epsilon=1e-4, source=tb.sources.constant(1.0))
    with tb.Mesh(V, F) as mesh:
        plain, s_plain = mesh.estimate(sites, cfg)
        mesh.set_tuning(grid_fp64=1)
        grid, s_grid = mesh.estimate(sites, cfg)
        smp = mesh.walk_samples(sites, cfg)
    assert s_plain["grid_steps"] == 0 and s_grid["grid_steps"] > 0.2 * s_grid["steps"]
    assert s_grid["caps"] == 0 and s_grid["node_tests"] < s_plain["node_tests"]
    se = smp["u"].std(axis=1, ddof=1) / np.sqrt(cfg.walks)
    z = (grid["u"] - u_exact) / se
    assert np.max(np.abs(z)) < 4.5 and np.mean(np.abs(z) < 3) >= 0.95
    zz = (grid["score"] - plain["score"]) / np.hypot(grid["score_se"], plain["score_se"])
    assert np.max(np.abs(zz)) < 4.5 and abs(np.mean(zz)) < 0.5
