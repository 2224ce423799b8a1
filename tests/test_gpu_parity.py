"""GPU parity: the CUDA path (through libtwos.so's C ABI) against the CPU oracle,
the reference's tracked outputs and the analytic unit ball.

Tolerances
* FP64 form vs oracle in the shared counter stream: identical integer step
  counts; per-walk values to rtol 1e-10 (the only non-identical operations are
  the device's sincospi/exp against the host's cos/sin/exp, a few ulp).
* Closest point, FP64: identical to the oracle's exact FP64 minimum (same
  Ericson arithmetic, no FMA contraction) up to 2 ulp.  Mixed: within the
  session's FP32 error bound delta.
* Monte Carlo comparisons (different streams): |z| < 4 per site and the
  fraction with |z| < 3 at least 0.95, z = difference / combined SE.
"""
import json
import subprocess

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN, PKG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.fixture(scope="module")
def bunny_mesh(tb, bunny1000):
    m = tb.Mesh(*bunny1000)
    yield m
    m.close()


@pytest.fixture(scope="module")
def housing_mesh(tb, housing):
    m = tb.Mesh(*housing)
    yield m
    m.close()


def _inside_points(mesh, V, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = V.min(0), V.max(0)
    pts = lo + (hi - lo) * rng.random((8 * n, 3))
    ins = mesh.inside(pts)
    return pts[ins][:n]


# ---------------------------------------------------------------- closest point
@pytest.mark.parametrize("which", ["bunny", "housing"])
def test_closest_point_matches_exact_fp64(tb, oracle_mod, bunny1000, housing, bunny_mesh, housing_mesh, which):
    V, F = bunny1000 if which == "bunny" else housing
    mesh = bunny_mesh if which == "bunny" else housing_mesh
    rng = np.random.default_rng(5)
    lo, hi = V.min(0), V.max(0)
    span = hi - lo
    pts = lo - 0.2 * span + 1.4 * span * rng.random((20000, 3))
    om = oracle_mod.OracleMesh(V, F)
    d_ref, c_ref, _, _ = om.closest_point(pts, brute=(which == "bunny"))
    d64, c64 = mesh.closest_point(pts, precision="fp64")
    np.testing.assert_allclose(d64, d_ref, rtol=4.5e-16, atol=1e-300)
    ok = np.isfinite(c64).all(axis=1)
    assert ok.all()
    np.testing.assert_allclose(np.linalg.norm(pts - c64, axis=1), d_ref, rtol=1e-12, atol=1e-15)
    d32, c32 = mesh.closest_point(pts, precision="mixed")
    delta = mesh.info()["mixed_delta"]
    assert np.max(np.abs(d32 - d_ref)) <= delta
    # The bound is not loose by orders of magnitude either.
    assert np.max(np.abs(d32 - d_ref)) >= delta * 1e-3


def test_closest_point_query_radius(tb, bunny_mesh):
    far = np.array([[100.0, 0.0, 0.0]])
    d = bunny_mesh.closest_point(far, precision="fp64", query_radius=4.0, with_points=False)
    assert np.isinf(d[0])
    d = bunny_mesh.closest_point(far, precision="fp64", query_radius=0.0, with_points=False)
    assert np.isfinite(d[0]) and d[0] > 99.0


# ---------------------------------------------------------------- walks vs oracle (shared counter stream)
def _oracle_kw(oracle_mod, cfg):
    return dict(mode={"compliance": 0, "paired": 1, "hot": 2}[cfg.mode], rng=oracle_mod.RNG_COUNTER,
                walks=cfg.walks, max_steps=cfg.max_steps, seed=cfg.seed, repeat=cfg.repeat, stream=cfg.stream,
                epsilon=cfg.epsilon, cavity_radius=cfg.cavity_radius, query_radius=cfg.query_radius,
                green=cfg.green, weight_order=1, threads=0)


def _terms_to_oracle(oracle_mod, terms):
    return [oracle_mod.term(t.kind, t.amp, t.axis, t.offset, t.div, tuple(t.c), tuple(t.w)) for t in terms]


def test_compliance_walks_fp64_equal_oracle(tb, oracle_mod, bunny1000, bunny_mesh, eval_points):
    cfg = tb.Config(walks=64, mode="compliance", precision="fp64", seed=77, epsilon=5e-4,
                    source=tb.sources.affine(0.65))
    sites = eval_points[:24]
    g = bunny_mesh.walk_samples(sites, cfg)
    om = oracle_mod.OracleMesh(*bunny1000)
    o = om.walk_samples(sites, source=oracle_mod.affine_source(0.65), **_oracle_kw(oracle_mod, cfg))
    np.testing.assert_array_equal(g["steps"], o["steps"])
    np.testing.assert_allclose(g["u"], o["u"], rtol=1e-10, atol=1e-300)
    est, summ = bunny_mesh.estimate(sites, cfg)
    ref = om.estimate(sites, source=oracle_mod.affine_source(0.65), **_oracle_kw(oracle_mod, cfg))
    np.testing.assert_array_equal(est["steps"], ref["steps"])
    for k in ("u", "score", "score_se", "same_index"):
        np.testing.assert_allclose(est[k], ref[k], rtol=1e-9, err_msg=k)
    assert summ["paths"] == 24 * 64 and summ["queries"] == summ["steps"] + summ["paths"]


@pytest.mark.parametrize("mode", ["paired", "hot"])
def test_paired_green_cavity_walks_fp64_equal_oracle(tb, oracle_mod, housing, housing_mesh, mode):
    d = GOLDEN / "distinct_adjoint" / "side1_seed2026091500_twos_dense_round2_rescore"
    pts = oracle_mod.read_points(d / "points.csv")[:12]
    holes = oracle_mod.read_points(d / "holes.csv")
    cfg = tb.Config(walks=48, mode=mode, precision="fp64", seed=2026091751, epsilon=5e-4, max_steps=1024,
                    cavity_radius=0.095, green=True, source=tb.sources.housing(), adjoint=tb.sources.sensor(1))
    g = housing_mesh.walk_samples(pts, cfg, cavities=holes)
    om = oracle_mod.OracleMesh(*housing)
    kw = _oracle_kw(oracle_mod, cfg)
    o = om.walk_samples(pts, cavities=holes, source=_terms_to_oracle(oracle_mod, cfg.source),
                        adjoint=_terms_to_oracle(oracle_mod, cfg.adjoint), **kw)
    np.testing.assert_array_equal(g["steps"], o["steps"])
    np.testing.assert_allclose(g["u"], o["u"], rtol=1e-10, atol=1e-300)
    if mode == "paired":
        np.testing.assert_allclose(g["p"], o["p"], rtol=1e-10, atol=1e-14)
    est, _ = housing_mesh.estimate(pts, cfg, cavities=holes)
    ref = om.estimate(pts, cavities=holes, source=_terms_to_oracle(oracle_mod, cfg.source),
                      adjoint=_terms_to_oracle(oracle_mod, cfg.adjoint), **kw)
    np.testing.assert_array_equal(est["steps"], ref["steps"])
    for k in ("u", "p", "score", "score_se", "same_index"):
        np.testing.assert_allclose(est[k], ref[k], rtol=1e-9, atol=1e-14, err_msg=k)


def test_sites_inside_cavities_give_zero_rows(tb, housing_mesh):
    d = GOLDEN / "distinct_adjoint" / "side1_seed2026091500_twos_dense_round2_rescore"
    holes = np.loadtxt(d / "holes.csv", delimiter=",").reshape(-1, 3)
    sites = holes[:1] + np.array([[0.01, 0.0, 0.0]])
    cfg = tb.Config(walks=8, mode="paired", precision="mixed", seed=1, cavity_radius=0.095, green=True,
                    source=tb.sources.housing(), adjoint=tb.sources.sensor(1), max_steps=1024)
    est, _ = housing_mesh.estimate(sites, cfg, cavities=holes)
    for k in ("u", "p", "score", "same_index"):
        assert est[k][0] == 0.0
    assert est["steps"][0] == 0


# ---------------------------------------------------------------- mixed form
def test_mixed_shares_samples_with_fp64(tb, bunny_mesh, eval_points):
    # Distance grid off: the FP32 query alone keeps the FP64 form's paths.
    sites = eval_points[:64]
    base = dict(walks=256, mode="compliance", seed=11, epsilon=5e-4, source=tb.sources.affine(0.65))
    bunny_mesh.set_tuning(grid_threshold=0)
    try:
        g64 = bunny_mesh.walk_samples(sites, tb.Config(precision="fp64", **base))
        g32 = bunny_mesh.walk_samples(sites, tb.Config(precision="mixed", **base))
        same = np.mean(g64["steps"] == g32["steps"])
        assert same > 0.5, same
        e64, _ = bunny_mesh.estimate(sites, tb.Config(precision="fp64", **base))
        e32, _ = bunny_mesh.estimate(sites, tb.Config(precision="mixed", **base))
    finally:
        bunny_mesh.set_tuning()
    z = (e32["score"] - e64["score"]) / np.sqrt(e32["score_se"] ** 2 + e64["score_se"] ** 2)
    assert np.max(np.abs(z)) < 3.0


# ---------------------------------------------------------------- vs reference outputs (independent streams)
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_reference_field_within_combined_error(tb, oracle_mod, precision, eval_points):
    V, F = oracle_mod.load_ascii_ply(GOLDEN / "stanford-bunny-watertight.ply.gz")
    ref = pd.read_csv(GOLDEN / "compiled_bunny" / "field-reference.csv")
    with tb.Mesh(V, F) as mesh:
        cfg = tb.Config(walks=2048, precision=precision, seed=12345, epsilon=5e-4, max_steps=512,
                        source=tb.sources.affine(0.65))
        est, summ = mesh.estimate(eval_points, cfg)
        if precision == "mixed":
            # The distance grid (on by default in the mixed form) takes shorter
            # steps far from the surface; the step count of the reference's
            # algorithm is the grid-off run's.
            assert summ["grid_steps"] > 0 and summ["steps"] / summ["paths"] > 17.7199
            mesh.set_tuning(grid_threshold=0)
            _, summ = mesh.estimate(eval_points, cfg)
            assert summ["grid_steps"] == 0
    z = (est["score"] - ref["score"].values) / np.sqrt(est["score_se"] ** 2 + ref["score_se"].values ** 2)
    assert np.max(np.abs(z)) < 4.5, np.max(np.abs(z))
    assert np.mean(np.abs(z) < 3.0) >= 0.95
    assert abs(np.mean(z)) < 0.35
    # Mean steps per path agree with the reference's 17.72 (summary.json:26) to 1%.
    assert abs(summ["steps"] / summ["paths"] - 17.7199) < 0.18


# ---------------------------------------------------------------- analytic unit ball
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_unit_ball_compliance_analytic(tb, precision):
    V, F = tb.geometry.icosphere(4)
    sites = tb.geometry.uniform_ball(64, 0.9, seed=0)
    with tb.Mesh(V, F) as mesh:
        cfg = tb.Config(walks=1024, precision=precision, seed=3, epsilon=1e-4, source=tb.sources.constant(1.0))
        est, _ = mesh.estimate(sites, cfg)
        smp = mesh.walk_samples(sites, cfg)
    u_exact = (1.0 - np.sum(sites ** 2, axis=1)) / 6.0
    se_u = smp["u"].std(axis=1, ddof=1) / np.sqrt(cfg.walks)
    # Inscribed polyhedron + epsilon shell bias, far below the MC error here.
    zu = (est["u"] - u_exact) / se_u
    zs = (est["score"] - u_exact ** 2) / est["score_se"]
    assert np.max(np.abs(zu)) < 4.5 and np.max(np.abs(zs)) < 4.5
    assert np.mean(np.abs(zu) < 3) >= 0.95


# ---------------------------------------------------------------- errors
def test_step_cap_is_runtime_error(tb, bunny_mesh, eval_points):
    cfg = tb.Config(walks=4, max_steps=1, precision="mixed")
    with pytest.raises(tb.TwosError) as e:
        bunny_mesh.estimate(eval_points[:4], cfg)
    assert e.value.code == 1 and "max-steps" in str(e.value)
    est, summ = bunny_mesh.estimate(eval_points[:4], cfg, raise_on_caps=False)
    assert summ["caps"] == 16 and np.all(est["caps"] == 4)


def test_far_site_is_query_failure(tb, bunny_mesh):
    cfg = tb.Config(walks=4, precision="fp64")
    with pytest.raises(tb.TwosError) as e:
        bunny_mesh.estimate(np.array([[50.0, 0.0, 0.0]]), cfg)
    assert e.value.code == 1 and "closest-point query failed" in str(e.value)


def test_usage_errors(tb, bunny_mesh):
    with pytest.raises(tb.TwosError) as e:
        bunny_mesh.estimate(np.zeros((1, 3)), tb.Config(walks=1))
    assert e.value.code == 2
    with pytest.raises(tb.TwosError) as e:
        bunny_mesh.estimate(np.zeros((1, 3)), tb.Config(walks=4, cavity_radius=0.0),
                            cavities=np.zeros((1, 3)))
    assert e.value.code == 2


# ---------------------------------------------------------------- device entry points
def test_estimate_device_matches_host(tb, bunny_mesh, eval_points):
    import torch
    cfg = tb.Config(walks=32, precision="mixed", seed=9)
    host, _ = bunny_mesh.estimate(eval_points, cfg)
    d_sites = torch.tensor(eval_points, dtype=torch.float64, device="cuda")
    d_out = torch.zeros((len(eval_points), 7), dtype=torch.float64, device="cuda")
    bunny_mesh.estimate_device(d_sites, len(eval_points), d_out, cfg)
    torch.cuda.synchronize()
    dev = d_out.cpu().numpy().copy().view(np.dtype(tb.SITE_DTYPE)).reshape(-1)
    for k in ("u", "score", "score_se", "steps"):
        np.testing.assert_array_equal(dev[k], host[k])


def test_topk_device(tb, bunny_mesh, oracle_mod):
    import torch
    rng = np.random.default_rng(4)
    keys = rng.normal(size=100_003)
    keys[17] = keys[99] = keys.max() + 1.0  # a tie broken by the lower index
    dk = torch.tensor(keys, device="cuda")
    idx = torch.zeros(64, dtype=torch.int32, device="cuda")
    bunny_mesh.topk_device(dk, len(keys), 64, idx)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(idx.cpu().numpy(), oracle_mod.topk_indices(keys, 64))


# ---------------------------------------------------------------- executables
def test_cli_twos_field_and_summary(tb, tmp_path, bunny1000):
    mesh = tmp_path / "bunny.ply"
    tb.geometry.write_ply(mesh, *bunny1000)
    field = tmp_path / "field.csv"
    summary = tmp_path / "summary.json"
    from twos_b200 import driver
    s = driver.run_cpp(None, mesh, GOLDEN / "compiled_bunny" / "evaluation-points.csv", field, summary, 32,
                       20260912 + 1800, 3, 8)
    ref = pd.read_csv(GOLDEN / "compiled_bunny" / "field-bunny-01000-faces.csv")
    out = pd.read_csv(field)
    assert list(out.columns) == list(ref.columns)
    np.testing.assert_array_equal(out[["x", "y", "z"]].values, ref[["x", "y", "z"]].values)
    refsum = json.loads((GOLDEN / "compiled_bunny" / "summary-bunny-01000-faces.json").read_text())
    assert set(refsum) - {"engine"} <= set(s)
    assert s["sites"] == 384 and s["walks_per_site"] == 32 and len(s["timings_seconds"]) == 3
    z = (out["score"] - ref["score"]) / np.sqrt(out["score_se"] ** 2 + ref["score_se"] ** 2)
    assert np.mean(np.abs(z) < 3) > 0.9


def test_cli_adjoint_serve_session(tb, tmp_path, housing):
    from twos_b200 import driver
    mesh = tmp_path / "housing.ply"
    tb.geometry.write_ply(mesh, *housing)
    src = GOLDEN / "distinct_adjoint" / "side1_seed2026091500_twos_sparse_round1_scout"
    a = json.loads((src / "argv.json").read_text())
    sess = driver.ServeSession()
    try:
        codes = []
        for hot, extra in [(0, []), (1, []), (0, ["--max-steps", "1"])]:
            out = tmp_path / f"f{hot}{len(extra)}.csv"
            args = ["--mesh", str(mesh), "--points", str(src / "points.csv"), "--cavities", str(src / "holes.csv"),
                    "--cavity-radius", a["--cavity-radius"], "--output", str(out), "--summary",
                    str(tmp_path / "k.json"), "--mode", "twos", "--source-mode", "housing", "--walks", a["--walks"],
                    "--seed", a["--seed"], "--threads", "8", "--repeats", "1", "--epsilon", a["--epsilon"],
                    "--max-steps", a["--max-steps"], "--sensor-side", a["--sensor-side"], "--hot-only", str(hot)]
            args += extra
            codes.append(sess.request(args))
            ref = pd.read_csv(src / "field.csv")
            got = pd.read_csv(out)
            assert list(got.columns) == list(ref.columns)
            assert len(got) == len(ref)
            if not extra:
                meta = json.loads((tmp_path / "k.json").read_text())
                assert {"total_seconds", "peak_rss_megabytes", "relative_residual", "steps", "caps"} <= set(meta)
        assert codes == [0, 0, 1]
        assert sess.close() == 1
    finally:
        if sess.proc.poll() is None:
            sess.proc.kill()
