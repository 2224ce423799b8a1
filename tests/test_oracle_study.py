"""Pins the oracle's paired/hot estimator to the study backend's tracked
requests (benchmarks/submission_study/pilot/pipeline/branch: wih_study,
study.cpp:80-120 paired_site with the config's sources and normalised sensor,
study.cpp:44-52).

The pilot requests were made with the branch config's two remote heat
sources; the third heat line of the tracked branch.txt (a bump at the sensor)
is not part of them.  Integer steps and caps must agree exactly; u, p, score
and same_index to the reference's FP32-query-radius residual (rtol 1e-6), and
exact zeros stay zeros."""
import json

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN

STUDY = GOLDEN / "submission_study"
CASES = ["paired-rescore", "paired-scout", "hot-refine"]


def study_request(oracle_mod, tag):
    d = STUDY / tag
    a = json.loads((d / "argv.json").read_text())
    sensor, heat = oracle_mod.load_study_config(STUDY / "branch.txt")
    R = sensor[3]
    sens = [oracle_mod.term(oracle_mod.TERM_BUMP, 1.0, div=32 * 3.141592653589793 * R ** 3 / 105,
                            c=tuple(sensor[:3]), w=(R, 0.0, 0.0))]
    pts = oracle_mod.read_points(d / "points.txt")
    holes = oracle_mod.read_points(d / "holes.txt") if a["has_cavities"] else np.zeros((0, 3))
    kw = dict(mode=2 if a["--hot-only"] == "1" else 1, walks=int(a["--walks"]), seed=int(a["--seed"]),
              epsilon=float(a["--epsilon"]), max_steps=int(a["--max-steps"]),
              cavity_radius=float(a["--cavity-radius"]), green=True, source=heat[:2], adjoint=sens,
              weight_order=1)
    return d, a, pts, holes, kw


@pytest.fixture(scope="module")
def branch(oracle_mod):
    V, F = oracle_mod.load_ascii_ply(GOLDEN / "branch.ply.gz")
    return oracle_mod.OracleMesh(V, F)


@pytest.mark.parametrize("tag", CASES)
def test_study_requests(oracle_mod, branch, tag):
    d, a, pts, holes, kw = study_request(oracle_mod, tag)
    est = branch.estimate(pts, cavities=holes, **kw)
    ref = pd.read_csv(d / "field.csv", float_precision="round_trip")
    np.testing.assert_array_equal(est["steps"], ref["steps"].values)
    np.testing.assert_array_equal(est["caps"], ref["caps"].values)
    assert int(est["steps"].sum()) == json.loads((d / "kernel.json").read_text())["steps"]
    for k in ("u", "p", "score", "same_index"):
        r = ref[k].values
        np.testing.assert_array_equal(est[k] == 0, r == 0, err_msg=k)
        np.testing.assert_allclose(est[k], r, rtol=1e-6, atol=0, err_msg=k)
