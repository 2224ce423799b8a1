"""GPU EXACT source mode (the analytic study source, study.cpp:53-77, 96-104)
against the oracle and an independent quadrature.

Tolerances
* Closed form on the device (double-double) vs quadrature: error / (A R^2)
  below 1e-9 (the reference's own bar, matched_accuracy/check_integral.py);
  vs the oracle's long-double form below 2e-12 (the long-double form's own
  cancellation error at d = 1e-9 R is 1e-12).
* FP64 walks vs the oracle in the shared counter stream: identical step
  counts; per-walk u and p to rtol 1e-10.
"""
import numpy as np
import pytest

from conftest import GOLDEN
from test_oracle_exact_source import audit_cases

pytestmark = pytest.mark.gpu
STUDY = GOLDEN / "submission_study"


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.fixture(scope="module")
def branch(oracle_mod):
    return oracle_mod.load_ascii_ply(GOLDEN / "branch.ply.gz")


@pytest.fixture(scope="module")
def branch_mesh(tb, branch):
    m = tb.Mesh(*branch)
    yield m
    m.close()


def _study_terms(tb):
    """The config's three heat bumps (one beside the sensor, so the probe
    sites see heat) and its sensor as EXACT-mode terms: heat A = amplitude,
    sensor A = 105 / (32 pi R^3) (study.cpp:100-101)."""
    (sx, sy, sz, sr), heat = tb.sources.load_study_config(STUDY / "branch.txt")
    sensor = [tb.sources.term(tb._abi.TERM_BUMP, 105 / (32 * 3.141592653589793 * sr ** 3), c=(sx, sy, sz),
                              w=(sr, 0.0, 0.0))]
    return heat, sensor


def _oracle_terms(oracle_mod, terms):
    return [oracle_mod.term(t.kind, t.amp, t.axis, t.offset, t.div, tuple(t.c), tuple(t.w)) for t in terms]


def test_device_closed_form(tb, oracle_mod):
    cases = audit_cases()
    got = tb.ball_green_integral(cases)
    quad = np.array([oracle_mod.green_ball_quadrature(*c) for c in cases])
    scale = cases[:, 3] * cases[:, 2] ** 2
    err = np.abs(got - quad) / scale
    assert err.max() < 1e-9, (err.max(), cases[err.argmax()])
    err_o = np.abs(got - oracle_mod.exact_bump_green(cases)) / scale
    assert err_o.max() < 2e-12, (err_o.max(), cases[err_o.argmax()])


@pytest.mark.parametrize("mode", ["paired", "hot"])
def test_exact_walks_fp64_equal_oracle(tb, oracle_mod, branch, branch_mesh, mode):
    heat, sensor = _study_terms(tb)
    pts = np.loadtxt(STUDY / "gradient-0.004-6" / "points.txt").reshape(-1, 3)[:24]
    holes = np.loadtxt(STUDY / "gradient-0.004-6" / "holes.txt").reshape(-1, 3)
    cfg = tb.Config(walks=32, mode=mode, precision="fp64", seed=1866, epsilon=2e-4, max_steps=2048,
                    cavity_radius=0.065, green="exact", source=heat, adjoint=sensor)
    g = branch_mesh.walk_samples(pts, cfg, cavities=holes)
    om = oracle_mod.OracleMesh(*branch)
    o = om.walk_samples(pts, cavities=holes, mode={"paired": 1, "hot": 2}[mode], rng=oracle_mod.RNG_COUNTER,
                        walks=cfg.walks, max_steps=cfg.max_steps, seed=cfg.seed, epsilon=cfg.epsilon,
                        cavity_radius=cfg.cavity_radius, green=2, weight_order=1,
                        source=_oracle_terms(oracle_mod, heat), adjoint=_oracle_terms(oracle_mod, sensor))
    np.testing.assert_array_equal(g["steps"], o["steps"])
    np.testing.assert_allclose(g["u"], o["u"], rtol=1e-10, atol=1e-300)
    assert np.count_nonzero(g["u"]) > 0
    if mode == "paired":
        np.testing.assert_allclose(g["p"], o["p"], rtol=1e-10, atol=1e-300)
        assert np.count_nonzero(g["p"]) > 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_exact_harmonic_source_is_the_centre_rule(tb, branch_mesh, precision):
    """For constant + linear sources the exact ball integral is r^2/6 f(y):
    the EXACT and CENTER modes give identical samples (study.cpp:97-99)."""
    pts = np.loadtxt(STUDY / "gradient-0.004-6" / "points.txt").reshape(-1, 3)[:16]
    src = [tb.sources.term(tb._abi.TERM_CONST, 1.0), tb.sources.term(tb._abi.TERM_LINEAR, 0.65, axis=1)]
    base = dict(walks=16, mode="paired", precision=precision, seed=3, epsilon=2e-4, max_steps=2048, source=src,
                adjoint=src)
    a = branch_mesh.walk_samples(pts, tb.Config(green="exact", **base))
    b = branch_mesh.walk_samples(pts, tb.Config(green="center", **base))
    for k in ("u", "p", "steps"):
        np.testing.assert_array_equal(a[k], b[k])


def test_exact_mixed_shares_samples(tb, branch_mesh):
    heat, sensor = _study_terms(tb)
    pts = np.loadtxt(STUDY / "gradient-0.004-6" / "points.txt").reshape(-1, 3)[:64]
    base = dict(walks=256, mode="paired", seed=9, epsilon=2e-4, max_steps=2048, green="exact", source=heat,
                adjoint=sensor)
    s64 = branch_mesh.walk_samples(pts, tb.Config(precision="fp64", **base))
    # Distance grid off: the FP32 query alone keeps the FP64 form's paths.
    branch_mesh.set_tuning(grid_threshold=0)
    try:
        s32 = branch_mesh.walk_samples(pts, tb.Config(precision="mixed", **base))
    finally:
        branch_mesh.set_tuning()
    assert np.mean(s64["steps"] == s32["steps"]) > 0.5
    for k in ("u", "p"):
        se = s64[k].std(axis=1, ddof=1) / np.sqrt(base["walks"])
        diff = np.abs(s32[k].mean(axis=1) - s64[k].mean(axis=1))
        assert np.all(diff <= 2.0 * se + 1e-12), (k, np.max(diff / np.maximum(se, 1e-300)))
    # With the grid: other samples of the same estimator.
    sg = branch_mesh.walk_samples(pts, tb.Config(precision="mixed", **base))
    for k in ("u", "p"):
        se = np.hypot(s64[k].std(axis=1, ddof=1), sg[k].std(axis=1, ddof=1)) / np.sqrt(base["walks"])
        diff = np.abs(sg[k].mean(axis=1) - s64[k].mean(axis=1))
        assert np.all(diff <= 4.5 * se + 1e-12), (k, np.max(diff / np.maximum(se, 1e-300)))


def test_exact_rejects_non_bump_terms(tb, branch_mesh):
    pts = np.zeros((1, 3))
    cfg = tb.Config(walks=4, green="exact", source=tb.sources.housing())
    with pytest.raises(tb.TwosError, match="exact source"):
        branch_mesh.estimate(pts, cfg)
