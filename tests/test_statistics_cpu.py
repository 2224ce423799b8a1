"""The oracle's statistics against the reference's own definitions and its
tracked seeded experiment.

* crossfit_square (benchmarks/stanford_bunny/run_bunny_benchmark.py:257-269,
  the vectorised form of evaluate_site, benchmarks/compiled_bunny/src/
  wih_twos.cpp:686-715) and crossfit_product (experiments/
  run_controlled_experiments.py:79-87, sign included) against brute-force
  double loops over i != j and explicit leave-one-out recomputation;
* the seeded cross-fit bias experiment (run_controlled_experiments.py:
  250-321) against its tracked output experiments/output/crossfit_bias.csv
  (a committed fixture): identical to the last bit, and the summary's claim
  that the cross-fit bias at correlation 0.9 stays within 0.004
  (:757-760) with the tracked value.
"""
import csv
import itertools
import json

import numpy as np

from conftest import GOLDEN

FIX = GOLDEN / "controlled_experiments"


def _brute_square(x):
    n = len(x)
    est = sum(x[i] * x[j] for i, j in itertools.permutations(range(n), 2)) / (n * (n - 1))
    leave = []
    for k in range(n):
        y = [x[i] for i in range(n) if i != k]
        m = len(y)
        leave.append(sum(y[i] * y[j] for i, j in itertools.permutations(range(m), 2)) / (m * (m - 1)))
    lm = sum(leave) / n
    se = np.sqrt((n - 1) / n * sum((v - lm) ** 2 for v in leave))
    return est, se


def test_crossfit_square_matches_its_definition(oracle_mod):
    rng = np.random.default_rng(7)
    x = rng.lognormal(size=(5, 9))
    est, se = oracle_mod.crossfit_square(x)
    for s in range(len(x)):
        e, sd = _brute_square(list(x[s]))
        assert abs(est[s] - e) <= 1e-13 * abs(e)
        assert abs(se[s] - sd) <= 1e-11 * sd


def test_crossfit_product_matches_its_definition(oracle_mod):
    rng = np.random.default_rng(8)
    a = rng.normal(1.0, 0.5, size=(4, 11))
    b = 0.3 * a + rng.normal(0.6, 0.4, size=(4, 11))
    got = oracle_mod.crossfit_product(a, b)
    n = a.shape[1]
    for s in range(len(a)):
        off = sum(a[s, i] * b[s, j] for i, j in itertools.permutations(range(n), 2)) / (n * (n - 1))
        assert abs(got[s] + off) <= 1e-13 * abs(off)  # the reference returns minus the off-diagonal mean
    se = oracle_mod.cross_jackknife_se(a, b)
    for s in range(len(a)):
        leave = []
        for k in range(n):
            keep = [i for i in range(n) if i != k]
            leave.append(-oracle_mod.crossfit_product(a[s, keep], b[s, keep]))
        lm = np.mean(leave)
        assert abs(se[s] - np.sqrt((n - 1) / n * np.sum((np.array(leave) - lm) ** 2))) <= 1e-11 * se[s]


def test_seeded_crossfit_experiment_reproduces_tracked_rows(oracle_mod):
    rows = oracle_mod.crossfit_experiment()
    ref = list(csv.DictReader(open(FIX / "crossfit_bias.csv")))
    assert len(rows) == len(ref) == 40
    for r, q in zip(rows, ref):
        assert r["method"] == q["method"] and abs(r["correlation"] - float(q["correlation"])) < 1e-15
        for k in ("mean_estimate", "bias", "bias_se", "rmse"):
            assert r[k] == float(q[k]), (r["method"], r["correlation"], k)


def test_seeded_crossfit_claims(oracle_mod):
    summary = json.loads((FIX / "summary.json").read_text())["crossfit"]
    rows = [r for r in oracle_mod.crossfit_experiment() if abs(r["correlation"] - 0.9) < 1e-12]
    by = {r["method"]: r["bias"] for r in rows}
    assert abs(by["Cross-fit TWoS"]) <= 0.004  # run_controlled_experiments.py:757-760
    assert by["Cross-fit TWoS"] == summary["crossfit_bias_at_corr_0.9"]
    assert by["Same-seed product"] == summary["same_seed_bias_at_corr_0.9"]
    # The same-seed product's bias is -cov = -0.9 * 0.5 * 0.6 within its noise.
    assert abs(by["Same-seed product"] + 0.27) < 0.003
