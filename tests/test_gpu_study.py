"""The wih_study executable family and wih_twos --mode diffwos on the GPU,
through the same argv, files and --serve framing as the reference's study
driver (benchmarks/submission_study/run_study.py:19-38, study.cpp:273-379).

Tolerances
* FP64 form vs the oracle in the shared counter stream: identical steps and
  caps; u, p, score, same_index to rtol 1e-9 (sincospi vs cos/sin, a few ulp
  per step).
* vs the reference's tracked requests (independent streams): total steps
  within 3 % (1024 walks x 16 sites) and exact zeros where no walk can reach
  a source.
"""
import gzip
import json
import shutil
import subprocess

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN, PKG
from test_oracle_study import study_request

pytestmark = pytest.mark.gpu
STUDY = GOLDEN / "submission_study"
BIN = PKG / "_build"


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.fixture(scope="module")
def assets(tmp_path_factory, lib_built):
    """branch.ply (the tracked asset, decompressed) and the two-remote-source
    config the pilot requests used."""
    d = tmp_path_factory.mktemp("study_assets")
    with gzip.open(GOLDEN / "branch.ply.gz", "rb") as src, open(d / "branch.ply", "wb") as dst:
        shutil.copyfileobj(src, dst)
    lines = [ln for ln in (STUDY / "branch.txt").read_text().splitlines() if ln.strip()]
    (d / "branch.txt").write_text("\n".join(lines[:3]) + "\n")
    return d


def _argv(exe, assets, d, tag, a, out, extra=()):
    argv = [str(BIN / exe), "--mesh", str(assets / "branch.ply"), "--config", str(assets / "branch.txt"),
            "--points", str(STUDY / tag / "points.txt"),
            "--cavities", str(STUDY / tag / "holes.txt") if a["has_cavities"] else "",
            "--output", str(out / "field.csv"), "--summary", str(out / "kernel.json")]
    for k, v in a.items():
        if k.startswith("--"):
            argv += [k, v]
    return argv + list(extra)


def _oracle_counter(oracle_mod, kw, green=True):
    kw = dict(kw)
    kw.update(rng=oracle_mod.RNG_COUNTER, green=green)
    return kw


@pytest.mark.parametrize("tag", ["paired-rescore", "hot-refine"])
def test_wih_study_fp64_equals_oracle(oracle_mod, assets, tmp_path, tag):
    d, a, pts, holes, kw = study_request(oracle_mod, tag)
    r = subprocess.run(_argv("wih_study", assets, d, tag, a, tmp_path, ["--precision", "fp64"]),
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = pd.read_csv(tmp_path / "field.csv", float_precision="round_trip")
    assert list(got.columns) == ["site", "u", "p", "score", "same_index", "steps", "caps"]
    V, F = oracle_mod.load_ascii_ply(GOLDEN / "branch.ply.gz")
    want = oracle_mod.OracleMesh(V, F).estimate(pts, cavities=holes, **_oracle_counter(oracle_mod, kw))
    np.testing.assert_array_equal(got["steps"].values, want["steps"])
    for k in ("u", "p", "score", "same_index"):
        np.testing.assert_allclose(got[k].values, want[k], rtol=1e-9, atol=1e-300, err_msg=k)
    summary = json.loads((tmp_path / "kernel.json").read_text())
    for key in ("total_seconds", "peak_rss_megabytes", "distance_queries", "parity_rays", "enclosure_fallbacks",
                "relative_residual", "steps", "caps"):
        assert key in summary
    assert summary["steps"] == int(want["steps"].sum())
    n_walk_sites = len(pts) - sum(np.any(np.linalg.norm(p - holes, axis=1) <= kw["cavity_radius"]) for p in pts) \
        if len(holes) else len(pts)
    assert summary["distance_queries"] == summary["steps"] + n_walk_sites * kw["walks"]
    # The reference's own request, independent stream: same work, same zeros.
    ref = pd.read_csv(d / "field.csv")
    assert abs(got["steps"].sum() / ref["steps"].sum() - 1.0) < 0.03
    np.testing.assert_array_equal(got["p"].values == 0, ref["p"].values == 0)


def test_serve_session_and_errors(oracle_mod, tb, assets, tmp_path):
    """One session: a paired request, a hot one, then a refused --fd request
    that ends the session with DONE 1 (study.cpp:367-373)."""
    from twos_b200 import driver
    solver = driver.StudySolver(assets / "branch.ply", assets / "branch.txt", tmp_path / "serve")
    _, a, pts, holes, kw = study_request(oracle_mod, "paired-scout")
    df, meta = solver.call("scout", pts, holes, radius=kw["cavity_radius"], walks=48, seed=int(a["--seed"]))
    assert len(df) == len(pts) and meta["steps"] == int(df["steps"].sum()) and meta["caps"] == 0
    inside = np.array([np.any(np.linalg.norm(p - holes, axis=1) <= kw["cavity_radius"]) for p in pts])
    assert np.all(df["steps"].values[inside] == 0) and np.all(df["steps"].values[~inside] > 0)
    df2, _ = solver.call("hot", pts[:8], hot=True, walks=16, seed=3)
    assert np.all(df2["p"] == 0) and np.all(df2["same_index"] == 0)
    np.testing.assert_allclose(df2["score"], df2["u"], rtol=1e-12)
    with pytest.raises(RuntimeError, match="DONE 1"):
        solver.call("fd", pts[:2], fd=True, walks=4)
    assert solver.session is None
    solver.close()


def test_study_refusals(assets, tmp_path):
    tag = "paired-scout"
    a = json.loads((STUDY / tag / "argv.json").read_text())
    base = _argv("wih_study", assets, STUDY / tag, tag, a, tmp_path)
    r = subprocess.run(base + ["--fd", "1"], capture_output=True, text=True)
    assert r.returncode == 1 and "finite-difference" in r.stderr
    r = subprocess.run([x if x != "twos" else "mg" for x in base], capture_output=True, text=True)
    assert r.returncode == 1 and "mg" in r.stderr
    bad = [x if x != str(assets / "branch.txt") else str(tmp_path / "none.txt") for x in base]
    r = subprocess.run(bad, capture_output=True, text=True)
    assert r.returncode == 1 and "bad sensor config" in r.stderr
    r = subprocess.run(base + ["--walks", "1"], capture_output=True, text=True)
    assert r.returncode == 2


def test_wih_study_diff_matches_api(tb, assets, tmp_path):
    """--diff 1 writes the reference's differential CSV; its numbers are the
    library's twos_diffwos with the enclosure fallback on."""
    tag = "gradient-0.008-0"
    a = json.loads((STUDY / tag / "argv.json").read_text())
    a["has_cavities"] = True
    pts = np.loadtxt(STUDY / tag / "points.txt").reshape(-1, 3)[:32]
    np.savetxt(tmp_path / "pts.txt", pts, fmt="%.17g")
    argv = _argv("wih_study", assets, STUDY / tag, tag, a, tmp_path, ["--precision", "fp64", "--walks", "256"])
    argv[argv.index("--points") + 1] = str(tmp_path / "pts.txt")
    r = subprocess.run(argv, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = pd.read_csv(tmp_path / "field.csv", float_precision="round_trip")
    ref = pd.read_csv(STUDY / tag / "field.csv")
    assert list(got.columns) == list(ref.columns)
    summary = json.loads((tmp_path / "kernel.json").read_text())
    assert set(summary) == {"total_seconds", "steps", "caps", "peak_rss_megabytes", "distance_queries",
                            "parity_rays", "enclosure_fallbacks"}
    _, heat = tb.sources.load_study_config(assets / "branch.txt")
    holes = np.loadtxt(STUDY / tag / "holes.txt").reshape(-1, 3)
    cfg = tb.Config(walks=256, mode="compliance", precision="fp64", seed=int(a["--seed"]),
                    epsilon=float(a["--epsilon"]), max_steps=int(a["--max-steps"]),
                    cavity_radius=float(a["--cavity-radius"]), green="green", source=heat,
                    skip_cavity_sites=False)
    with tb.Mesh(ply=assets / "branch.ply") as mesh:
        rows, stats, s = mesh.diffwos(pts, cfg, holes, diff_offset=float(a["--diff-offset"]),
                                      enclosure_fallback=True)
    cols = [c for c in got.columns if c.startswith(("dc", "dR"))]
    flat = np.concatenate([rows["dc"], rows["dc_se"], rows["dR"][..., None], rows["dR_se"][..., None]], axis=-1)
    np.testing.assert_array_equal(got[cols].values, flat.reshape(len(pts), -1))
    assert summary["distance_queries"] == s["queries"] and summary["parity_rays"] == s["parity_rays"]


def test_wih_twos_diffwos_mode(tb, assets, tmp_path):
    tag = "gradient-0.008-0"
    pts = np.loadtxt(STUDY / tag / "points.txt").reshape(-1, 3)[:16]
    np.savetxt(tmp_path / "pts.txt", pts, fmt="%.17g")
    argv = [str(BIN / "wih_twos"), "--mode", "diffwos", "--mesh", str(assets / "branch.ply"), "--points",
            str(tmp_path / "pts.txt"), "--cavities", str(STUDY / tag / "holes.txt"), "--cavity-radius", "0.065",
            "--output", str(tmp_path / "f.csv"), "--summary", str(tmp_path / "s.json"), "--walks", "128",
            "--repeats", "2", "--epsilon", "2e-4", "--max-steps", "2048", "--diff-offset", "0.008",
            "--source-mode", "affine"]
    r = subprocess.run(argv, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = pd.read_csv(tmp_path / "f.csv")
    assert len(got) == 16 and got.columns[:4].tolist() == ["site", "x", "y", "z"]
    s = json.loads((tmp_path / "s.json").read_text())
    assert s["mode"] == "diffwos" and s["gradient_parameters"] == 4 * 6 and len(s["timings_seconds"]) == 2
    assert 0.0 <= s["unsafe_given_cavity_fraction"] <= 1.0
    r = subprocess.run([x for x in argv if x not in ("--cavities", str(STUDY / tag / "holes.txt"))],
                       capture_output=True, text=True)
    assert r.returncode == 2


@pytest.mark.parametrize("exe", ["wih_analytic_query", "wih_compliance_query"])
def test_analytic_executables_equal_oracle(oracle_mod, tb, assets, tmp_path, exe):
    tag = "paired-rescore"
    d, a, pts, holes, kw = study_request(oracle_mod, tag)
    r = subprocess.run(_argv(exe, assets, d, tag, a, tmp_path, ["--precision", "fp64"]), capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    got = pd.read_csv(tmp_path / "field.csv", float_precision="round_trip")
    if exe == "wih_compliance_query":
        f = [oracle_mod.term(oracle_mod.TERM_CONST, 1.0), oracle_mod.term(oracle_mod.TERM_LINEAR, 0.65, 1, 0.0)]
        kw.update(source=f, adjoint=f)
    else:
        sensor, _ = oracle_mod.load_study_config(STUDY / "branch.txt")
        R = sensor[3]
        kw.update(adjoint=[oracle_mod.term(oracle_mod.TERM_BUMP, 105 / (32 * 3.141592653589793 * R ** 3),
                                           c=tuple(sensor[:3]), w=(R, 0.0, 0.0))])
    V, F = oracle_mod.load_ascii_ply(GOLDEN / "branch.ply.gz")
    want = oracle_mod.OracleMesh(V, F).estimate(pts, cavities=holes, **_oracle_counter(oracle_mod, kw, green=2))
    np.testing.assert_array_equal(got["steps"].values, want["steps"])
    for k in ("u", "p", "score", "same_index"):
        np.testing.assert_allclose(got[k].values, want[k], rtol=1e-9, atol=1e-300, err_msg=k)
    if exe == "wih_compliance_query":
        np.testing.assert_array_equal(got["u"].values, got["p"].values)
    assert np.count_nonzero(got["u"].values) > 0


def test_integral_audit_executable(oracle_mod):
    from test_oracle_exact_source import audit_cases
    cases = audit_cases()
    text = "".join(" ".join(repr(float(v)) for v in c) + "\n" for c in cases)
    r = subprocess.run([str(BIN / "wih_analytic_integral_audit")], input=text, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    values = np.array([float(v) for v in r.stdout.split()])
    quad = np.array([oracle_mod.green_ball_quadrature(*c) for c in cases])
    err = np.abs(values - quad) / (cases[:, 3] * cases[:, 2] ** 2)
    assert len(values) == len(cases) and err.max() < 1e-9
