"""Design loop on the device (twos_design_loop): scout -> top-k -> fresh
validation -> lower-bound argmax -> accept/insert, captured as a CUDA graph.

* FP64 form vs the oracle's FP64 restatement on the same counter-stream
  samples: identical chosen candidates, accept decisions and cavities (bit
  exact); scores to rtol 1e-9.
* Graph replay vs plain launches: identical histories.
* Mixed vs FP64 form under shared samples, distance grid off (the FP32 query
  alone only perturbs the FP64 path by its rounding): identical decisions
  wherever the FP64 lower bounds of the best two shortlist entries differ by
  more than the mixed form's perturbation.
* Mixed form with the distance grid (its walks take other radii, so its
  samples are no longer the FP64 ones): the first iteration's chosen lower
  bound agrees with the FP64 one within 4 combined standard errors.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


def _setup(tb):
    V, F = tb.geometry.icosphere(3)
    cand = tb.geometry.uniform_ball(1500, 0.85, seed=1)
    return V, F, cand


KW = dict(iterations=6, shortlist=16, cavity_radius=0.05, z=1.96, accept_threshold=0.02, outer_clearance=0.02,
          pair_gap=0.01)


def _configs(tb, precision):
    scout = tb.Config(walks=64, precision=precision, seed=31, stream=0, epsilon=1e-4, max_steps=1024,
                      source=tb.sources.constant(1.0))
    val = tb.Config(walks=256, precision=precision, seed=31, stream=1, epsilon=1e-4, max_steps=1024,
                    source=tb.sources.constant(1.0))
    return scout, val


def test_fp64_design_loop_matches_oracle(tb, oracle_mod):
    V, F, cand = _setup(tb)
    scout, val = _configs(tb, "fp64")
    with tb.Mesh(V, F) as mesh:
        hist, cav, summ = mesh.design_loop(cand, scout, val, use_graph=True, **KW)
    om = oracle_mod.OracleMesh(V, F)
    ref, ref_cav = oracle_mod.design_loop(
        om, cand, dict(walks=64, seed=31, stream=0, epsilon=1e-4, max_steps=1024,
                       source=[oracle_mod.term(oracle_mod.TERM_CONST, 1.0)]),
        dict(walks=256, seed=31, stream=1, epsilon=1e-4, max_steps=1024,
             source=[oracle_mod.term(oracle_mod.TERM_CONST, 1.0)]),
        KW["iterations"], KW["shortlist"], KW["cavity_radius"], KW["z"], KW["accept_threshold"],
        KW["outer_clearance"], KW["pair_gap"])
    assert [int(h["chosen"]) for h in hist] == [r["chosen"] for r in ref]
    assert [bool(h["accepted"]) for h in hist] == [r["accepted"] for r in ref]
    assert any(r["accepted"] for r in ref) and not all(r["accepted"] for r in ref)
    np.testing.assert_array_equal(cav, ref_cav)
    for k in ("scout_score", "score", "score_se", "lower"):
        np.testing.assert_allclose(hist[k], [r[k] for r in ref], rtol=1e-9, err_msg=k)
    assert summ["caps"] == 0


def test_graph_replay_equals_plain_launches(tb):
    V, F, cand = _setup(tb)
    scout, val = _configs(tb, "mixed")
    with tb.Mesh(V, F) as mesh:
        h1, c1, _ = mesh.design_loop(cand, scout, val, use_graph=True, **KW)
        h0, c0, _ = mesh.design_loop(cand, scout, val, use_graph=False, **KW)
    np.testing.assert_array_equal(h1, h0)
    np.testing.assert_array_equal(c1, c0)


def test_mixed_decisions_match_fp64(tb):
    V, F, cand = _setup(tb)
    with tb.Mesh(V, F) as mesh:
        mesh.set_tuning(grid_threshold=0)
        h64, c64, _ = mesh.design_loop(cand, *_configs(tb, "fp64"), **KW)
        h32, c32, _ = mesh.design_loop(cand, *_configs(tb, "mixed"), **KW)
    for it in range(KW["iterations"]):
        if h64["chosen"][it] != h32["chosen"][it]:
            # Only a near tie may flip the choice; after it the paths diverge.
            assert abs(h64["lower"][it] - h32["lower"][it]) < 0.05 * abs(h64["lower"][it])
            break
        assert h64["accepted"][it] == h32["accepted"][it]
    assert h64["chosen"][0] == h32["chosen"][0]


def test_mixed_grid_design_loop_agrees_with_fp64(tb):
    V, F, cand = _setup(tb)
    with tb.Mesh(V, F) as mesh:
        h64, _, _ = mesh.design_loop(cand, *_configs(tb, "fp64"), **KW)
        h32, _, summ = mesh.design_loop(cand, *_configs(tb, "mixed"), **KW)
    assert summ["grid_steps"] > 0 and summ["caps"] == 0
    se = np.hypot(h64["score_se"][0], h32["score_se"][0])
    assert abs(h64["lower"][0] - h32["lower"][0]) < 4 * se


def _replay_validation(tb, mesh, cand, cav, h, it, precision):
    """The validation estimate of iteration `it`'s chosen candidate, replayed
    as a one-site estimate with the loop's keys: stream 1, repeat = it, site
    index = the choice's shortlist slot, the cavities present then."""
    _, val = _configs(tb, precision)
    val.repeat = it
    val.site_offset = int(h["slot"][it])
    val.cavity_radius = KW["cavity_radius"]
    c = cav[: int(h["n_cavities"][it])]
    rows, _ = mesh.estimate(cand[int(h["chosen"][it])][None, :], val, cavities=c if len(c) else None)
    return rows[0]


def test_accept_decisions_identical_given_chosen(tb):
    """The scout keeps the mixed form's distance grid, so the two forms may
    choose different candidates; the validation stage runs without it, so
    for the candidate the mixed loop chose, the FP64 form's validation of the
    same candidate uses the same samples and reaches the same accept bit."""
    V, F, cand = _setup(tb)
    with tb.Mesh(V, F) as mesh:
        h32, cav32, summ = mesh.design_loop(cand, *_configs(tb, "mixed"), **KW)
        assert summ["grid_steps"] > 0
        mesh.set_tuning(grid_threshold=0)
        checked = 0
        for it in range(KW["iterations"]):
            if h32["chosen"][it] == 0xFFFFFFFF:
                continue
            same = _replay_validation(tb, mesh, cand, cav32, h32, it, "mixed")
            assert same["score"] == h32["score"][it] and same["score_se"] == h32["score_se"][it]
            r64 = _replay_validation(tb, mesh, cand, cav32, h32, it, "fp64")
            lower64 = r64["score"] - KW["z"] * r64["score_se"]
            assert abs(lower64 - h32["lower"][it]) < 1e-3 * abs(h32["lower"][it])
            if abs(lower64 - KW["accept_threshold"]) > 1e-3 * KW["accept_threshold"]:
                assert bool(lower64 > KW["accept_threshold"]) == bool(h32["accepted"][it])
                checked += 1
    assert checked >= KW["iterations"] - 1
