"""Pins the oracle's Differential-WoS restatement (evaluate_differential_site,
benchmarks/compiled_bunny/src/wih_twos.cpp:839-928, as built into
benchmarks/submission_study/study.cpp with WIH_ENCLOSURE_FALLBACK) to the
reference's tracked gradient requests of
benchmarks/submission_study/validation-v1-remote-sources/raw/.

The request totals of kernel.json -- steps (outer + nested walks), distance
queries and parity rays (study.cpp:8-16, 351) -- must reproduce exactly: they
fix every walk path, every cavity termination and every ray-parity decision.
The per-cavity derivative columns of field.csv must agree to round-off.

These "remote sources" requests were produced with the first two heat lines
of branch.txt (the compact sources away from the sensor); the third line, a
bump at the sensor, is not part of them -- exact agreement of every nonzero
derivative holds only without it.
"""
import json

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN

CASES = ["gradient-0.004-6", "gradient-0.008-0"]


@pytest.fixture(scope="module")
def branch(oracle_mod):
    V, F = oracle_mod.load_ascii_ply(GOLDEN / "branch.ply.gz")
    return oracle_mod.OracleMesh(V, F)


@pytest.mark.parametrize("tag", CASES)
def test_diffwos_totals_and_derivatives(oracle_mod, branch, tag):
    d = GOLDEN / "submission_study" / tag
    a = json.loads((d / "argv.json").read_text())
    _, heat = oracle_mod.load_study_config(GOLDEN / "submission_study" / "branch.txt")
    pts = oracle_mod.read_points(d / "points.txt")
    holes = oracle_mod.read_points(d / "holes.txt")
    out, stats, totals = branch.diffwos(
        pts, holes, float(a["--diff-offset"]), walks=int(a["--walks"]), seed=int(a["--seed"]),
        epsilon=float(a["--epsilon"]), max_steps=int(a["--max-steps"]), cavity_radius=float(a["--cavity-radius"]),
        green=a["--source-mode"] == "housing", source=heat[:2], weight_order=0)
    k = json.loads((d / "kernel.json").read_text())
    assert int(stats[:, 0].sum() + stats[:, 1].sum()) == k["steps"]
    assert int(totals[0]) == k["distance_queries"]
    assert int(totals[1]) == k["parity_rays"]
    assert int(stats[:, 6].sum()) == k["caps"] == 0
    assert int(stats[:, 5].sum()) == 0  # the request succeeded, so no unsafe offsets
    ref = pd.read_csv(d / "field.csv", float_precision="round_trip")
    cols = [c for c in ref.columns if c.startswith(("dc", "dR"))]
    assert len(cols) == 8 * len(holes)
    np.testing.assert_allclose(out.reshape(len(pts), -1), ref[cols].values, rtol=1e-12, atol=1e-18)
    np.testing.assert_array_equal(ref[["x", "y", "z"]].values, pts)
