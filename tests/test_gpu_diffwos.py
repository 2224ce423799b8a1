"""GPU Differential WoS (twos_diffwos) against the oracle and the reference's
tracked gradient requests (benchmarks/submission_study/validation-v1-remote-
sources/raw/gradient-*: study.cpp --diff 1 on the branch geometry).

Tolerances
* FP64 form vs the oracle in the shared counter stream: every per-site count
  (outer and nested steps, cavity terminations, seam / segment / unsafe
  decisions, caps) and the request totals (distance queries, parity rays,
  enclosure fallbacks) identical; derivatives to rtol 1e-9 (the walks differ
  only by the device's sincospi against the host's cos/sin, a few ulp).
* Mixed form vs FP64 form (shared samples): the per-cavity derivative
  difference within 1.5 combined standard errors everywhere.
* Against the reference's field.csv (independent streams): z = difference /
  combined SE per derivative, |z| < 5 and the fraction with |z| < 3 >= 0.97.
"""
import json

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = ["gradient-0.004-6", "gradient-0.008-0"]
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


def _case(tb, tag, precision):
    d = STUDY / tag
    a = json.loads((d / "argv.json").read_text())
    _, heat = tb.sources.load_study_config(STUDY / "branch.txt")
    pts = np.loadtxt(d / "points.txt").reshape(-1, 3)
    holes = np.loadtxt(d / "holes.txt").reshape(-1, 3)
    # The tracked requests used the two remote heat sources (see the oracle's
    # golden test); the nested walks evaluate them at Green points.
    cfg = tb.Config(walks=int(a["--walks"]), mode="compliance", precision=precision, seed=int(a["--seed"]),
                    epsilon=float(a["--epsilon"]), max_steps=int(a["--max-steps"]),
                    cavity_radius=float(a["--cavity-radius"]), green=a["--source-mode"] == "housing",
                    source=heat[:2], skip_cavity_sites=False)
    return d, a, pts, holes, cfg


def _oracle_terms(oracle_mod, terms):
    return [oracle_mod.term(t.kind, t.amp, t.axis, t.offset, t.div, tuple(t.c), tuple(t.w)) for t in terms]


def _flat(rows):
    """[n_sites, n_cav] DIFF_DTYPE -> [n_sites, n_cav, 8] (dc, dc_se, dR, dR_se)."""
    return np.concatenate([rows["dc"], rows["dc_se"], rows["dR"][..., None], rows["dR_se"][..., None]], axis=-1)


@pytest.mark.parametrize("tag", CASES)
def test_fp64_equals_oracle_counter_stream(tb, oracle_mod, branch, branch_mesh, tag):
    d, a, pts, holes, cfg = _case(tb, tag, "fp64")
    off = float(a["--diff-offset"])
    rows, stats, summ = branch_mesh.diffwos(pts, cfg, holes, diff_offset=off, enclosure_fallback=True)
    om = oracle_mod.OracleMesh(*branch)
    out, ost, otot = om.diffwos(pts, holes, off, enclosure_fallback=True, rng=oracle_mod.RNG_COUNTER,
                                walks=cfg.walks, seed=cfg.seed, epsilon=cfg.epsilon, max_steps=cfg.max_steps,
                                cavity_radius=cfg.cavity_radius, green=cfg.green,
                                source=_oracle_terms(oracle_mod, cfg.source), threads=0)
    names = ["outer_steps", "nested_steps", "cavity_terminations", "near_seam", "segment_unsafe", "unsafe_offset",
             "limits"]
    for k, name in enumerate(names):
        np.testing.assert_array_equal(stats[name], ost[:, k], err_msg=name)
    assert summ["queries"] == int(otot[0])
    assert summ["parity_rays"] == int(otot[1])
    assert summ["enclosure_fallbacks"] == int(otot[2])
    assert summ["steps"] == int(ost[:, 0].sum() + ost[:, 1].sum())
    assert stats["cavity_terminations"].sum() > 0
    np.testing.assert_allclose(_flat(rows), out, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("tag", CASES)
def test_reference_gradients_within_combined_error(tb, branch_mesh, tag):
    d, a, pts, holes, cfg = _case(tb, tag, "fp64")
    rows, stats, summ = branch_mesh.diffwos(pts, cfg, holes, diff_offset=float(a["--diff-offset"]),
                                            enclosure_fallback=True)
    k = json.loads((d / "kernel.json").read_text())
    # Same estimator, independent stream: totals agree statistically.
    assert abs(summ["steps"] / k["steps"] - 1.0) < 0.02
    assert abs(summ["queries"] / k["distance_queries"] - 1.0) < 0.02
    assert abs(summ["parity_rays"] / max(k["parity_rays"], 1) - 1.0) < 0.1
    ref = pd.read_csv(d / "field.csv", float_precision="round_trip")
    cols = [c for c in ref.columns if c.startswith(("dc", "dR"))]
    want = ref[cols].values.reshape(len(pts), len(holes), 8)
    got = _flat(rows)
    zs = []
    for mean, se in [(0, 3), (1, 4), (2, 5), (6, 7)]:
        s = np.sqrt(got[..., se] ** 2 + want[..., se] ** 2)
        ok = s > 0
        zs.append((got[..., mean][ok] - want[..., mean][ok]) / s[ok])
        # Where neither estimator saw a sample spread the derivative is the
        # same constant (zero when no walk ended on that cavity).
        np.testing.assert_array_equal(got[..., mean][~ok], want[..., mean][~ok])
    z = np.concatenate(zs)
    assert len(z) > 0
    assert np.max(np.abs(z)) < 5.0, np.max(np.abs(z))
    assert np.mean(np.abs(z) < 3.0) >= 0.97


def test_mixed_shares_samples_with_fp64(tb, branch_mesh):
    d, a, pts, holes, cfg = _case(tb, CASES[0], "fp64")
    pts = pts[:96]
    off = float(a["--diff-offset"])
    r64, s64, _ = branch_mesh.diffwos(pts, cfg, holes, diff_offset=off, enclosure_fallback=True)
    cfg.precision = "mixed"
    # Distance grid off: the FP32 query alone keeps the FP64 form's paths.
    branch_mesh.set_tuning(grid_threshold=0)
    try:
        r32, s32, summ = branch_mesh.diffwos(pts, cfg, holes, diff_offset=off, enclosure_fallback=True)
    finally:
        branch_mesh.set_tuning()
    assert summ["launches"] == 4
    # Most walks take the same path; the termination counts nearly agree.
    t64, t32 = s64["cavity_terminations"].sum(), s32["cavity_terminations"].sum()
    assert abs(int(t64) - int(t32)) <= 0.02 * t64 + 5
    g64, g32 = _flat(r64), _flat(r32)
    for mean, se in [(0, 3), (1, 4), (2, 5), (6, 7)]:
        s = np.sqrt(g64[..., se] ** 2 + g32[..., se] ** 2)
        diff = np.abs(g64[..., mean] - g32[..., mean])
        assert np.all(diff <= 2.0 * s + 1e-12), np.max(diff / np.maximum(s, 1e-300))
    # With the grid (the default) the mixed walks are other samples of the same
    # estimator: agreement within the combined Monte Carlo error.
    rg, _, _ = branch_mesh.diffwos(pts, cfg, holes, diff_offset=off, enclosure_fallback=True)
    gg = _flat(rg)
    for mean, se in [(0, 3), (1, 4), (2, 5), (6, 7)]:
        s = np.sqrt(g64[..., se] ** 2 + gg[..., se] ** 2)
        diff = np.abs(g64[..., mean] - gg[..., mean])
        assert np.all(diff <= 4.5 * s + 1e-12), np.max(diff / np.maximum(s, 1e-300))


def test_unsafe_offsets_are_reported(tb, oracle_mod):
    """Two overlapping cavities in the unit ball: walks that end near their
    seam circle are unsafe; the call fails as study.cpp:309-310 does and the
    rows and statistics still come back, equal to the oracle's."""
    V, F = tb.geometry.icosphere(3)
    R = 0.2
    pair = np.array([[-0.6 * R, 0.0, 0.0], [0.6 * R, 0.0, 0.0]])
    # 0.05 outside both spheres, 0.06 from their seam circle (radius 0.8 R).
    sites = np.array([[0.0, 0.22, 0.0], [0.0, 0.0, 0.22], [0.0, -0.22, 0.0], [0.0, 0.0, -0.22]])
    cfg = tb.Config(walks=256, precision="fp64", seed=5, epsilon=1e-4, max_steps=2048, cavity_radius=R,
                    source=tb.sources.constant(1.0), skip_cavity_sites=False)
    with tb.Mesh(V, F) as mesh:
        with pytest.raises(tb.TwosError, match="unsafe"):
            mesh.diffwos(sites, cfg, pair, diff_offset=0.02)
        rows, stats, summ = mesh.diffwos(sites, cfg, pair, diff_offset=0.02, strict=False)
    assert summ["error"] and stats["near_seam"].sum() > 0
    om = oracle_mod.OracleMesh(V, F)
    out, ost, otot = om.diffwos(sites, pair, 0.02, enclosure_fallback=False, rng=oracle_mod.RNG_COUNTER,
                                walks=cfg.walks, seed=cfg.seed, epsilon=cfg.epsilon, max_steps=cfg.max_steps,
                                cavity_radius=R, green=False, source=_oracle_terms(oracle_mod, cfg.source),
                                threads=0)
    for k, name in enumerate(["outer_steps", "nested_steps", "cavity_terminations", "near_seam",
                              "segment_unsafe", "unsafe_offset", "limits"]):
        np.testing.assert_array_equal(stats[name], ost[:, k], err_msg=name)
    assert summ["queries"] == int(otot[0]) and summ["parity_rays"] == int(otot[1])
    np.testing.assert_allclose(_flat(rows), out, rtol=1e-9, atol=1e-12)


def test_usage_errors(tb, branch_mesh):
    d, a, pts, holes, cfg = _case(tb, CASES[0], "mixed")
    with pytest.raises(tb.TwosError, match="cavities"):
        branch_mesh.diffwos(pts[:2], cfg, np.zeros((0, 3)))
    with pytest.raises(tb.TwosError, match="diff_offset"):
        branch_mesh.diffwos(pts[:2], cfg, holes, diff_offset=cfg.epsilon)
    cfg.mode = "paired"
    with pytest.raises(tb.TwosError, match="one source"):
        branch_mesh.diffwos(pts[:2], cfg, holes)
