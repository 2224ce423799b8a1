"""The headline workload's own configuration at reduced size: the noise-
displaced icosphere L7 (327,680 triangles, harmonic seed 1) with its 2^28-
vertex distance grid and entry-node table, compliance f = 1 with u = 0,
eps 1e-4, max 1,024 steps, sites drawn from the bench's interior sites.

* Mixed (FP32 query with the grid) against FP64 (the reference's algorithm):
  2,048 sites x 512 walks, per-site z = (TD_mixed - TD_fp64) / combined SE.
  The two forms draw different walks (the grid changes the radii), so z is
  standard normal when both are unbiased: max |z| < 5, >= 99 % below 3,
  |mean z| < 0.1 (0.022 is one standard error of the mean at 2,048 sites).
* Every grid step's bound (the walk kernel's own record, 256 sites x 512
  walks) is at most the FP64 distance from the step's position to the mesh
  less delta: the ball a grid step uses (radius bound - delta) never leaves
  the domain.
* The entry-node start, walk claims and the wavefront form change no
  result: rows are equal bit for bit (same walks, same minima); the
  four-wide BVH's rows equal them except where a bound and a triangle
  distance tie within FP32 rounding (>= 99 % of sites identical).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(lib_built):
    import bench
    import twos_b200 as tb
    V, F, grid = bench.workload(64)
    sites = bench.workload_sites(grid)
    rng = np.random.default_rng(20)
    pick = sites[np.sort(rng.choice(len(sites), size=2048, replace=False))]
    mesh = tb.Mesh(V, F)
    yield tb, mesh, pick
    mesh.close()


def _cfg(tb, precision, walks=512, seed=77):
    return tb.Config(walks=walks, precision=precision, seed=seed, epsilon=1e-4, max_steps=1024,
                     source=tb.sources.constant(1.0))


def test_headline_grid_is_built(setup):
    tb, mesh, _ = setup
    info = mesh.info()
    assert info["faces"] == 327680
    assert 2 ** 27 < np.prod(info["grid_dims"]) <= 2 ** 28


def test_mixed_matches_fp64_on_the_headline_config(setup):
    tb, mesh, sites = setup
    m, sm = mesh.estimate(sites, _cfg(tb, "mixed"))
    d, sd = mesh.estimate(sites, _cfg(tb, "fp64"))
    assert sm["caps"] == sd["caps"] == 0 and sm["grid_steps"] > 0.5 * sm["steps"]
    z = (m["score"] - d["score"]) / np.hypot(m["score_se"], d["score_se"])
    assert np.max(np.abs(z)) < 5, np.max(np.abs(z))
    assert np.mean(np.abs(z) < 3) >= 0.99
    assert abs(np.mean(z)) < 0.1, np.mean(z)


def test_every_grid_step_stays_inside_the_domain(setup):
    tb, mesh, sites = setup
    delta = mesh.info()["mixed_delta"]
    pts, bounds, total = mesh.trace_grid_steps(sites[:256], _cfg(tb, "mixed"), capacity=1 << 23)
    assert total == len(bounds) and total > 500_000
    d64 = mesh.closest_point(pts, precision="fp64", with_points=False)
    slack = d64 - (bounds - delta)
    assert np.all(slack >= 0.0), slack.min()
    # The bound is a real radius, not a timid one: most steps use most of the distance.
    assert np.median(bounds / d64) > 0.5


def test_tuning_variants_change_no_result(setup):
    """Entry-node start off, walks per lane and the wavefront form: the rows
    stay those of the default tuning, bit for bit (same walks, same minima).

    The four-wide BVH (root-started four-wide queries on the 327,680-triangle
    mesh outgrow the traversal stack near the root and finish on the binary
    BVH) visits the same bounds in another order.  A node bound and an FP32
    triangle distance can tie to within rounding near the surface, where
    either traversal may keep a distance one rounding above the other's (both
    within the FP32 error bound delta of the true distance); a walk that
    meets such a tie continues on a ball an ulp larger.  So its rows equal the
    default's at all but a few sites, and those agree within their error."""
    tb, mesh, sites = setup
    s = sites[:512]
    base = mesh.get_tuning()
    try:
        ref, _ = mesh.estimate(s, _cfg(tb, "mixed", walks=256))
        for variant in (dict(entry=0), dict(lane_walks=4), dict(wavefront=1 << 21), dict(wavefront=1 << 16, entry=0)):
            mesh.set_tuning(**dict(base, **variant))
            got, _ = mesh.estimate(s, _cfg(tb, "mixed", walks=256))
            np.testing.assert_array_equal(got, ref, err_msg=str(variant))
        for variant in (dict(bvh_width=4), dict(bvh_width=4, entry=0)):
            mesh.set_tuning(**dict(base, **variant))
            got, _ = mesh.estimate(s, _cfg(tb, "mixed", walks=256))
            same = np.array([got[i] == ref[i] for i in range(len(s))])
            assert same.mean() >= 0.99, (variant, same.mean())
            z = (got["score"] - ref["score"]) / np.hypot(got["score_se"], ref["score_se"])
            assert np.all(np.abs(z[~same]) < 4.0), (variant, z[~same])
    finally:
        mesh.set_tuning(**base)
