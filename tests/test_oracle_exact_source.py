"""Pins the oracle's exact ball integral of a bump source (exact_bump_green,
benchmarks/submission_study/study.cpp:53-77, the analytic study source) to an
independent Green-volume quadrature, as the reference's own check does
(benchmarks/matched_accuracy/check_integral.py: 300 seeded cases plus edge
cases, error normalised by A R^2 below 1e-9).

The cases are drawn here with the same generator and seed as that check; the
quadrature is oracle.green_ball_quadrature (scipy)."""
import numpy as np
import pytest

EDGE = [(0, .001), (0, .3), (0, 1), (0, 2), (1, 1e-4), (2, 1), (2, 1 + 1e-8), (1, 2), (1e-14, .5), (.5, .5),
        # small offsets where P(d + r) - P(|d - r|) cancels
        (1e-9, .5), (1e-7, .3), (.999, 1e-6)]


def audit_cases():
    rng = np.random.default_rng(17092026)
    cases = []
    for _ in range(300):
        R = 10 ** rng.uniform(-2, 0)
        A = 10 ** rng.uniform(-1, 2)
        cases.append((rng.uniform(0, 3) * R, 10 ** rng.uniform(-3, .7) * R, R, A))
    cases += [(d, r, 1.0, 1.0) for d, r in EDGE]
    return np.array(cases)


@pytest.fixture(scope="module")
def quadrature(oracle_mod):
    c = audit_cases()
    return c, np.array([oracle_mod.green_ball_quadrature(*x) for x in c])


def test_closed_form_matches_quadrature(oracle_mod, quadrature):
    cases, ref = quadrature
    got = oracle_mod.exact_bump_green(cases)
    err = np.abs(got - ref) / (cases[:, 3] * cases[:, 2] ** 2)
    assert err.max() < 1e-9, (err.max(), cases[err.argmax()])
    assert got.min() >= 0.0


def test_closed_form_limits(oracle_mod):
    # Support inside the ball (d + R <= r): N(d) - M / (4 pi r); disjoint: 0.
    R, A = 0.2, 3.0
    d, r = 0.1, 0.5
    mass_over_4pi = A * R ** 3 * 8 / 105
    t = d / R
    n_at = A * R * R * (1 / 6 - t ** 2 / 6 + t ** 4 / 10 - t ** 6 / 42)
    got = oracle_mod.exact_bump_green([[d, r, R, A], [1.0, 0.5, 0.2, 1.0]])
    np.testing.assert_allclose(got[0], n_at - mass_over_4pi / r, rtol=1e-14)
    assert got[1] == 0.0
