"""Certified validation on the GPU (twos_validate, wih_twos --mode validate)
against the oracle and the reference's tracked validation attempts
(benchmarks/minimum_benefit/pilot-floor-policy).

Tolerances
* vs the oracle in the shared counter stream: steps, capped, clipped and
  containment identical; values to rtol 1e-10 (the device's sincospi against
  the host's cos/sin moves a direction by an ulp or so per step); the certified
  clearance bit-identical (no random draw involved).
* vs the reference (independent streams): the certified clearance
  bit-identical to validation.json; the exact FP64 centre distance to rtol
  1e-9; the n = 1024 stage means within 4 combined standard errors; the
  accept decision identical.
"""
import json
import subprocess

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN, PKG
from test_validation_cpu import CASES, MB, load_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.fixture(scope="module", params=list(CASES))
def case(request, tb, oracle_mod):
    tag = request.param
    kind, step, r, mesh, cfg, z, holes, samples, meta, decision = load_case(tag)
    V, F = oracle_mod.load_ascii_ply(GOLDEN / mesh)
    m = tb.Mesh(V, F)
    terms = tb.sources.affine(0.65) if kind == "bunny" else tb.sources.housing()
    yield tag, kind, step, r, cfg, z, holes, samples, meta, decision, V, F, m, terms
    m.close()


def _config(tb, kind, step, r, cfg, terms, walks):
    return tb.Config(walks=walks, precision="fp64", seed=cfg["seed"] + 100 * step + 2, stream=2,
                     epsilon=cfg["epsilon"], max_steps=cfg["max_steps"], cavity_radius=r,
                     green="green" if kind == "housing" else "center", source=terms)


def test_validate_equals_oracle_counter_stream(tb, oracle_mod, case):
    tag, kind, step, r, cfg, z, holes, samples, meta, decision, V, F, m, terms = case
    c = _config(tb, kind, step, r, cfg, terms, 512)
    s, st, summ = m.validate(z, c, cavities=holes, radius_cap=cfg["radius_cap"], value_cap=cfg["value_caps"][kind])
    o = oracle_mod.OracleMesh(V, F).validate(
        z, cfg["radius_cap"], cfg["value_caps"][kind], cavities=holes, rng=oracle_mod.RNG_COUNTER, stream=2,
        walks=512, seed=c.seed, epsilon=c.epsilon, max_steps=c.max_steps, cavity_radius=r,
        green=kind == "housing",
        source=[oracle_mod.term(t.kind, t.amp, t.axis, t.offset, t.div, tuple(t.c), tuple(t.w)) for t in terms])
    np.testing.assert_array_equal(s["steps"][0], o["steps"][0])
    np.testing.assert_array_equal(s["capped"][0].astype(bool), o["capped"][0])
    np.testing.assert_array_equal(s["clipped"][0].astype(bool), o["clipped"][0])
    assert s["contained"].all() and o["contained"].all() and summ["containment_failures"] == 0
    np.testing.assert_allclose(s["value"][0], o["value"][0], rtol=1e-10, atol=0)
    assert st["center_clearance_lower"][0, 0] == o["clearance"][0]
    assert summ["steps"] == int(s["steps"].sum())


def test_validate_stages_and_reference(tb, case):
    tag, kind, step, r, cfg, z, holes, samples, meta, decision, V, F, m, terms = case
    walks = 4096
    c = _config(tb, kind, step, r, cfg, terms, walks)
    s, st, summ = m.validate(z, c, cavities=holes, radius_cap=cfg["radius_cap"], value_cap=cfg["value_caps"][kind])
    assert list(st["n"][0]) == [1024, 4096]
    v = s["value"][0]
    for k, n in enumerate((1024, 4096)):
        acc = np.longdouble(0)
        for x in v[:n]:
            acc += np.longdouble(x)
        assert st["mean"][0, k] == float(acc / n)
        assert st["clipped"][0, k] == int(s["clipped"][0, :n].sum())
        assert st["path_caps"][0, k] == int(s["capped"][0, :n].sum())
    ref0 = meta["stages"][0]
    assert st["center_clearance_lower"][0, 0] == ref0["center_clearance_lower"]
    np.testing.assert_allclose(st["center_distance"][0, 0], ref0["embree_center_distance"], rtol=1e-9)
    ref_v = samples["value"].values[:1024]
    se = np.sqrt(v[:1024].var(ddof=1) / 1024 + ref_v.var(ddof=1) / 1024)
    assert abs(st["mean"][0, 0] - ref0["mean"]) < 4 * se
    # The host acceptance reaches the reference's decision on these samples.
    from twos_b200 import validation
    target = cfg["primary_target_fraction_of_fixed_scale"] * cfg["fixed_scales"][kind]
    stages = [dict(n=int(st["n"][0, k]), center_clearance_lower=float(st["center_clearance_lower"][0, k]))
              for k in range(st.shape[1])]
    accepted, records, best = validation.decide(v, stages, z[0], r, terms, cfg["value_caps"][kind],
                                                cfg["confidence_log_upper"], target)
    assert accepted == decision["accepted"]


def test_validate_errors(tb, case):
    tag, kind, step, r, cfg, z, holes, samples, meta, decision, V, F, m, terms = case
    c = _config(tb, kind, step, r, cfg, terms, 8)
    with pytest.raises(tb.TwosError, match="classified outside"):
        m.validate(V.max(0) + 1.0, c, cavities=holes, radius_cap=0.1, value_cap=0.1)
    if len(holes):
        with pytest.raises(tb.TwosError, match="classified outside"):
            m.validate(holes[:1], c, cavities=holes, radius_cap=0.1, value_cap=0.1)
    c.source = tb.sources.sensor(1)
    with pytest.raises(tb.TwosError, match="validation sources"):
        m.validate(z, c, cavities=holes, radius_cap=0.1, value_cap=0.1)


def test_cli_validate(tb, oracle_mod, tmp_path):
    tag = "bunny-00"
    kind, step, r, mesh, cfg, z, holes, samples, meta, decision = load_case(tag)
    import gzip
    import shutil
    with gzip.open(GOLDEN / mesh, "rb") as src, open(tmp_path / "m.ply", "wb") as dst:
        shutil.copyfileobj(src, dst)
    np.savetxt(tmp_path / "p.csv", z, delimiter=",", fmt="%.17g")
    argv = [str(PKG / "_build" / "wih_twos"), "--mode", "validate", "--mesh", str(tmp_path / "m.ply"), "--points",
            str(tmp_path / "p.csv"), "--output", str(tmp_path / "v.csv"), "--summary", str(tmp_path / "v.json"),
            "--walks", "2048", "--seed", str(cfg["seed"] + 2), "--repeats", "1", "--source-mode", "affine",
            "--source-y-slope", ".65", "--epsilon", str(cfg["epsilon"]), "--max-steps", str(cfg["max_steps"]),
            "--validation-radius-cap", str(cfg["radius_cap"]), "--validation-value-cap",
            str(cfg["value_caps"][kind])]
    res = subprocess.run(argv, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    got = pd.read_csv(tmp_path / "v.csv", float_precision="round_trip")
    assert list(got.columns) == ["site", "sample", "value", "steps", "capped", "clipped"] and len(got) == 2048
    js = json.loads((tmp_path / "v.json").read_text())
    assert js["distance_mode"] == "triangle_AABB_union_lower_bound" and js["containment_failures"] == 0
    assert [s["n"] for s in js["stages"]] == [1024, 2048]
    assert js["stages"][0]["center_clearance_lower"] == meta["stages"][0]["center_clearance_lower"]
    c = _config(tb, kind, 0, r, cfg, tb.sources.affine(0.65), 2048)
    with tb.Mesh(ply=tmp_path / "m.ply") as m:
        s, st, _ = m.validate(z, c, radius_cap=cfg["radius_cap"], value_cap=cfg["value_caps"][kind])
    np.testing.assert_array_equal(got["value"].values, s["value"][0])
    assert js["stages"][1]["mean"] == st["mean"][0, 1]
