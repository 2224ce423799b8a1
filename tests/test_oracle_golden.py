"""Pins the CPU oracle to the reference's own tracked outputs.

The oracle (oracle/twos_oracle.cpp) restates the reference backend; in its
reference-stream mode it uses the same per-walk std::mt19937_64 keying, the
same libstdc++ <random> and libm, so the integer step counts of the tracked
fixtures must reproduce exactly.  Values differ only by the reference's FP32
Embree query radius (wih_twos.cpp:344-348, 423-424: a candidate is accepted
when its FP64 distance is below the FP32-rounded current radius, so the
returned distance can differ from the exact minimum by one FP32 ulp of the
radius); the tolerances below bound that effect.
"""
import json

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN

COMP = GOLDEN / "compiled_bunny"
SEED = 20260912
# rtol for values: the FP32-radius acceptance moves each step's radius by at
# most ~1e-7 relative; accumulated over a walk and a site this stays < 2e-5.
U_RTOL, SCORE_RTOL, SE_RTOL = 2e-5, 5e-5, 2e-4


def _compliance(oracle_mod, mesh_file, points, walks, seed, sel=None, repeat=0):
    V, F = oracle_mod.load_ascii_ply(GOLDEN / mesh_file)
    m = oracle_mod.OracleMesh(V, F)
    ids = np.arange(len(points)) if sel is None else np.asarray(sel)
    est = m.estimate(points[ids], site_ids=ids, walks=walks, seed=seed, epsilon=5e-4, max_steps=512,
                     source=oracle_mod.affine_source(0.65), repeat=repeat)
    return est, ids


@pytest.mark.parametrize("faces", [1000, 4000])
def test_compliance_decimated_bunny_exact_steps(oracle_mod, eval_points, faces):
    # run_compiled_benchmark.py:754-760: 32 walks, seed + 1800, repeats 3, repeat 0 retained.
    est, _ = _compliance(oracle_mod, f"bunny-{faces:05d}-faces.ply.gz", eval_points, 32, SEED + 1800)
    ref = pd.read_csv(COMP / f"field-bunny-{faces:05d}-faces.csv")
    assert len(ref) == len(est) == 384
    np.testing.assert_array_equal(est["steps"], ref["steps"].values)
    np.testing.assert_array_equal(est["caps"], ref["limit_hits"].values)
    np.testing.assert_allclose(est["u"], ref["u"].values, rtol=U_RTOL)
    np.testing.assert_allclose(est["score"], ref["score"].values, rtol=SCORE_RTOL)
    np.testing.assert_allclose(est["score_se"], ref["score_se"].values, rtol=SE_RTOL)


def test_compliance_reference_field_subset(oracle_mod, eval_points):
    # field-reference.csv: 2,048 walks, seed + 720, 1 repeat (run_compiled_benchmark.py:676-680).
    sel = np.arange(0, 384, 48)
    est, ids = _compliance(oracle_mod, "stanford-bunny-watertight.ply.gz", eval_points, 2048, SEED + 720, sel)
    ref = pd.read_csv(COMP / "field-reference.csv").iloc[ids]
    np.testing.assert_array_equal(est["steps"], ref["steps"].values)
    np.testing.assert_allclose(est["u"], ref["u"].values, rtol=U_RTOL)
    np.testing.assert_allclose(est["score"], ref["score"].values, rtol=SCORE_RTOL)
    np.testing.assert_allclose(est["score_se"], ref["score_se"].values, rtol=SE_RTOL)


def test_compliance_walk_sweep_field(oracle_mod, eval_points):
    # field-twos-0016.csv: 16 walks, seed + 1000 + 16, repeat 0 retained.
    sel = np.arange(0, 384, 6)
    est, ids = _compliance(oracle_mod, "stanford-bunny-watertight.ply.gz", eval_points, 16, SEED + 1016, sel)
    ref = pd.read_csv(COMP / "field-twos-0016.csv").iloc[ids]
    np.testing.assert_array_equal(est["steps"], ref["steps"].values)
    np.testing.assert_allclose(est["u"], ref["u"].values, rtol=U_RTOL)


def _paired_cases():
    return json.loads((GOLDEN / "distinct_adjoint" / "index.json").read_text())


@pytest.mark.parametrize("tag", _paired_cases())
def test_paired_requests_exact_steps(oracle_mod, housing, tag):
    d = GOLDEN / "distinct_adjoint" / tag
    a = json.loads((d / "argv.json").read_text())
    pts = oracle_mod.read_points(d / "points.csv")
    try:
        holes = oracle_mod.read_points(d / "holes.csv")
    except RuntimeError:
        holes = np.zeros((0, 3))
    m = oracle_mod.OracleMesh(*housing)
    hot = int(a["--hot-only"])
    sel = np.arange(0, len(pts), max(1, len(pts) // 24))
    est = m.estimate(pts[sel], site_ids=sel, cavities=holes,
                     mode=oracle_mod.MODE_HOT if hot else oracle_mod.MODE_PAIRED,
                     walks=int(a["--walks"]), seed=int(a["--seed"]), epsilon=float(a["--epsilon"]),
                     max_steps=int(a["--max-steps"]), cavity_radius=float(a["--cavity-radius"]), green=True,
                     source=oracle_mod.housing_source(), adjoint=oracle_mod.sensor_source(int(a["--sensor-side"])))
    ref = pd.read_csv(d / "field.csv").iloc[sel]
    np.testing.assert_array_equal(est["steps"], ref["steps"].values)
    np.testing.assert_array_equal(est["caps"], ref["caps"].values)
    np.testing.assert_allclose(est["u"], ref["u"].values, rtol=1e-6, atol=1e-15)
    if not hot:
        np.testing.assert_allclose(est["p"], ref["p"].values, rtol=1e-6, atol=1e-12)
        np.testing.assert_allclose(est["score"], ref["score"].values, rtol=1e-5, atol=1e-12)
        np.testing.assert_allclose(est["same_index"], ref["same_index"].values, rtol=1e-5, atol=1e-12)
    else:
        np.testing.assert_allclose(est["score"], ref["u"].values, rtol=1e-6, atol=1e-15)


@pytest.mark.parametrize("tag", _paired_cases())
def test_paired_fixture_identity(tag):
    # distinct_adjoint/audit_benchmark.py:99-100: score == (n u p - same)/(n - 1).
    d = GOLDEN / "distinct_adjoint" / tag
    a = json.loads((d / "argv.json").read_text())
    if int(a["--hot-only"]):
        pytest.skip("hot requests report mean u")
    n = int(a["--walks"])
    ref = pd.read_csv(d / "field.csv", float_precision="round_trip")
    recon = (n * ref["u"] * ref["p"] - ref["same_index"]) / (n - 1)
    np.testing.assert_allclose(ref["score"], recon, rtol=1e-12, atol=1e-18)


def test_summary_fixture_queries_definition():
    # distance_queries_per_second = (steps + paths)/runtime (wih_twos.cpp:1779-1780).
    s = json.loads((COMP / "reference-summary.json").read_text())
    paths = s["sites"] * s["walks_per_site"]
    steps = s["mean_steps"] * paths
    assert abs((steps + paths) / s["runtime_seconds_median"] - s["distance_queries_per_second"]) < 1e-6 * s[
        "distance_queries_per_second"]
