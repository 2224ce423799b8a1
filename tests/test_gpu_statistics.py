"""Known-answer tests of the device reduction (finalize_kernel, through the
C ABI twos_finalize_samples) on identical host-generated samples.

* Compliance rows against the oracle's crossfit_square (benchmarks/
  stanford_bunny/run_bunny_benchmark.py:257-269; evaluate_site, benchmarks/
  compiled_bunny/src/wih_twos.cpp:686-715): estimate and jackknife SE.
* Paired rows against crossfit_product (experiments/
  run_controlled_experiments.py:79-87, which returns minus the off-diagonal
  mean) and its leave-one-out jackknife SE, on the seeded cross-fit
  experiment's own samples (run_controlled_experiments.py:250-271, 30,000
  replicates x 32 pairs per correlation).
* The experiment rerun with the device reduction as its cross-fit estimator
  reproduces the tracked per-correlation rows (experiments/output/
  crossfit_bias.csv) and the claim that the bias at correlation 0.9 stays
  within 0.004 (:757-760).

Tolerances: the device sums in a fixed warp-shuffle order, the oracle in
numpy's pairwise order, both in FP64.  Estimates agree to 1e-14 of the
scale sum|a| sum|b| / (n (n - 1)) (the sums' rounding, no cancellation beyond
that), means to 1e-13 relative (n terms summed in another order), SEs to
1e-10 relative (the leave-one-out values differ from their mean
by ~1/n of their size, which amplifies the rounding of the sums).  Mixed
precision rounds the samples to float first; the oracle gets the same
rounded samples.
"""
import csv

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mesh(lib_built, bunny1000):
    import twos_b200 as tb
    m = tb.Mesh(*bunny1000)
    yield m
    m.close()


def _scale(a, b):
    n = a.shape[1]
    return np.abs(a).sum(1) * np.abs(b).sum(1) / (n * (n - 1))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_compliance_reduction_matches_crossfit_square(mesh, oracle_mod, precision):
    rng = np.random.default_rng(11)
    # Walk-like payoffs: heavy-tailed, a few near zero, several walk counts.
    for n_sites, walks in [(257, 4), (300, 33), (64, 1024), (7, 4096)]:
        x = rng.lognormal(-3.0, 1.0, size=(n_sites, walks))
        x[:, ::7] *= 1e-3
        if precision == "mixed":
            x = x.astype(np.float32).astype(np.float64)
        steps = rng.integers(1, 60, size=x.shape, dtype=np.uint32)
        rows = mesh.finalize_samples(x, steps=steps, mode="compliance", precision=precision)
        est, se = oracle_mod.crossfit_square(x)
        assert np.all(np.abs(rows["score"] - est) <= 1e-14 * _scale(x, x)), (n_sites, walks)
        np.testing.assert_allclose(rows["score_se"], se, rtol=1e-10, atol=0)
        np.testing.assert_allclose(rows["u"], x.mean(1), rtol=1e-13, atol=0)
        np.testing.assert_allclose(rows["same_index"], (x * x).mean(1), rtol=1e-13, atol=0)
        np.testing.assert_array_equal(rows["steps"], steps.sum(1, dtype=np.uint64))
        assert np.all(rows["caps"] == 0)


def test_caps_are_counted(mesh):
    x = np.ones((3, 8))
    steps = np.full((3, 8), 5, dtype=np.uint32)
    steps[1, 2] |= np.uint32(0x80000000)
    rows = mesh.finalize_samples(x, steps=steps)
    assert rows["caps"].tolist() == [0, 1, 0]
    assert rows["steps"].tolist() == [40, 40, 40]


def test_paired_reduction_matches_crossfit_product_on_the_seeded_experiment(mesh, oracle_mod):
    rng = np.random.default_rng(np.random.SeedSequence(oracle_mod.CROSSFIT_SEED).spawn(5)[2])
    for correlation in np.linspace(-0.9, 0.9, 10):
        a, b, _ = oracle_mod.crossfit_experiment_draws(correlation, rng)
        if abs(correlation) < 0.5:
            continue  # keep the test short; the draws still advance as in the reference
        rows = mesh.finalize_samples(a, b, mode="paired")
        ref = -oracle_mod.crossfit_product(a, b)
        assert np.all(np.abs(rows["score"] - ref) <= 1e-14 * _scale(a, b)), correlation
        np.testing.assert_allclose(rows["score_se"], oracle_mod.cross_jackknife_se(a, b), rtol=1e-10, atol=0)
        np.testing.assert_allclose(rows["same_index"], np.mean(a * b, axis=1), rtol=1e-13, atol=0)
        np.testing.assert_allclose(rows["u"], a.mean(1), rtol=1e-13, atol=0)
        np.testing.assert_allclose(rows["p"], b.mean(1), rtol=1e-13, atol=0)


def test_seeded_experiment_with_the_device_reduction(mesh, oracle_mod):
    def device(a, b):
        return -mesh.finalize_samples(a, b, mode="paired")["score"]

    rows = oracle_mod.crossfit_experiment(estimator=device)
    ref = list(csv.DictReader(open(GOLDEN / "controlled_experiments" / "crossfit_bias.csv")))
    for r, q in zip(rows, ref):
        assert r["method"] == q["method"]
        for k in ("mean_estimate", "bias"):
            assert abs(r[k] - float(q[k])) <= 1e-13, (r["method"], r["correlation"], k)
        assert abs(r["bias_se"] - float(q["bias_se"])) <= 1e-9 * float(q["bias_se"])
    at09 = {r["method"]: r["bias"] for r in rows if abs(r["correlation"] - 0.9) < 1e-12}
    assert abs(at09["Cross-fit TWoS"]) <= 0.004
    assert at09["Same-seed product"] < -0.26  # the i = j term's bias, -cov


def test_hot_reduction_is_the_mean(mesh):
    rng = np.random.default_rng(3)
    x = rng.normal(size=(50, 100))
    rows = mesh.finalize_samples(x, mode="hot")
    np.testing.assert_allclose(rows["score"], x.mean(1), rtol=1e-13, atol=1e-16)
    loo = (x.sum(1, keepdims=True) - x) / 99.0
    se = np.sqrt(99.0 / 100.0 * np.sum((loo - loo.mean(1, keepdims=True)) ** 2, axis=1))
    np.testing.assert_allclose(rows["score_se"], se, rtol=1e-10)


def test_usage_errors(mesh):
    import twos_b200 as tb
    with pytest.raises(tb.TwosError):
        mesh.finalize_samples(np.ones((2, 1)))
    with pytest.raises(tb.TwosError):
        mesh.finalize_samples(np.ones((2, 4)), mode="paired")
