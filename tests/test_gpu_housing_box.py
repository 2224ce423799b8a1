"""The housing-like workload's geometry and sources at test size: the box 4 x 2 x 1
minus six through-cylinders (builder-written mesher, seed 34), f = 1 on
x0 < 1, adjoint q = 1_{x0 > 3} / |{x0 > 3}| with a Green point per step.

* The mesh is closed and outward (every directed edge once, its reverse
  once; divergence-theorem volume within 0.2 % of the box minus the
  cylinders), and the device's ray parity agrees with the analytic
  membership on random points.
* Mixed and FP64 forms share samples: the cross-index scores agree within
  two combined standard errors; u and p are nonnegative and u is larger on
  the heated side.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.fixture(scope="module")
def box(tb):
    V, F, centres = tb.geometry.box_minus_cylinders(h=0.04)
    return V, F, centres


def test_mesh_closed_and_parity(tb, box):
    V, F, centres = box
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]]).astype(np.int64)
    key = e[:, 0] * len(V) + e[:, 1]
    assert len(np.unique(key)) == len(key)
    assert np.isin(key, e[:, 1] * len(V) + e[:, 0]).all()
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    vol = np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6
    assert abs(vol / (8 - 6 * np.pi * 0.15 ** 2) - 1) < 2e-3
    rng = np.random.default_rng(3)
    pts = rng.random((4000, 3)) * np.array([4.4, 2.4, 1.4]) - 0.2
    exact = np.all((pts >= 0) & (pts <= [4, 2, 1]), axis=1)
    for c in centres:
        exact &= np.hypot(pts[:, 0] - c[0], pts[:, 1] - c[1]) > 0.15
    # Keep points clear of the surface (the mesh is a polygonal approximation).
    d_box = np.min(np.abs(np.c_[pts, pts - [4, 2, 1]]), axis=1)
    d_cyl = np.min([np.abs(np.hypot(pts[:, 0] - c[0], pts[:, 1] - c[1]) - 0.15) for c in centres], axis=0)
    # The parity ray (the reference's fixed oblique direction, tfar 4,
    # wih_twos.cpp:361-394) only sees surfaces within 4 of the point: keep
    # points whose ray leaves the box's far faces within that reach.
    d = np.array([1.0, 0.3713906763541037, 0.1570796326794897])
    d /= np.linalg.norm(d)
    t_exit = np.min((np.array([4.0, 2.0, 1.0]) - pts) / d, axis=1)
    clear = (d_box > 0.01) & (d_cyl > 0.01) & (t_exit < 3.9)
    with tb.Mesh(V, F) as mesh:
        got = mesh.inside(pts)
    np.testing.assert_array_equal(got[clear], exact[clear])


def test_sources_and_forms(tb, box):
    V, F, centres = box
    big = 1e30
    f = tb.sources.box_indicator((-big, -big, -big), (1.0, big, big))
    vol = tb.geometry.box_region_volume(centres, 0.15, 3.0, right=True)
    assert 1.8 < vol < 2.0
    q = tb.sources.box_indicator((3.0, -big, -big), (big, big, big), amp=1.0 / vol)
    sites = tb.geometry.box_interior_points(64, centres, 0.15, seed=35)
    base = dict(walks=2048, mode="paired", seed=4, epsilon=1e-4, max_steps=1 << 16, green=True, source=f, adjoint=q)
    with tb.Mesh(V, F) as mesh:
        e64, s64 = mesh.estimate(sites, tb.Config(precision="fp64", **base))
        e32, s32 = mesh.estimate(sites, tb.Config(precision="mixed", **base))
    assert s64["caps"] == 0 and s32["caps"] == 0
    se = np.sqrt(e64["score_se"] ** 2 + e32["score_se"] ** 2)
    assert np.all(np.abs(e64["score"] - e32["score"]) <= 2.0 * se + 1e-15)
    # u > 0 everywhere (f >= 0, zero data), largest near the heated end.
    assert np.all(e64["u"] >= 0) and np.all(e64["p"] >= 0)
    hot = sites[:, 0] < 1.0
    assert e64["u"][hot].mean() > e64["u"][~hot].mean()
