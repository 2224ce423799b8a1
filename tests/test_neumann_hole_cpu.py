"""Finite-hole check of the Neumann-cavity topological derivative that the
gradient form's TD is assembled from (D_T = 3/2 grad u . grad p - q u - f p),
in exact rational arithmetic (oracle/neumann_hole.py, modelled on the
reference's Dirichlet audit benchmarks/exact_cavity_audit/audit.py:11-27).

The data make every term of the formula nonzero at the hole centre: Dirichlet
modes of degree 0, 1 and 2, a constant source f0 and an objective density q
with modes of degree 0, 1 and 2.  At radii 1e-1, 1e-2, 1e-3 and 1e-4 the exact
(J(a) - J(0)) / |B_a| approaches D_T with an error that falls as a^2, while a
polarization of 1 or 3 instead of 3/2, a flipped sign of q u, or a missing f p
term leaves a finite error."""
from fractions import Fraction as Fr

import pytest

import neumann_hole as nh

DATA = nh.Data(f0=Fr(7, 5), a0=Fr(3, 4), a1=Fr(-5, 3), a2=Fr(2, 7), c0=Fr(6, 5), c1=Fr(9, 4), c2=Fr(-3, 2))
RADII = [Fr(1, 10), Fr(1, 100), Fr(1, 1000), Fr(1, 10000)]


def test_every_term_is_nonzero_at_the_centre():
    u, grad_dot, q, p = nh.centre_fields(DATA)
    assert u != 0 and grad_dot != 0 and q != 0 and p != 0 and DATA.f0 != 0


def test_finite_hole_ratio_converges_to_the_formula_as_a_squared():
    rows = nh.check(DATA, RADII)
    errs = [abs(r["error"]) for r in rows]
    for a, e in zip(RADII, errs):
        # O(a^2): the next terms of every mode are a^5 / a^3.
        assert e <= 4 * a ** 2, (a, float(e))
    for e0, e1 in zip(errs, errs[1:]):
        assert e1 * 50 < e0  # one decade in a: two decades in the error
    assert float(abs(rows[-1]["error"] / rows[-1]["td"])) < 1e-7


def test_the_unperturbed_objective_matches_direct_integration():
    # J(0)/(4 pi) = c0 * int r^2 U0 + c1/3 * int r^3 (a1 r) + c2/5 * int r^4 (a2 r^2), U0 = -f0 r^2/6 + a0 + f0/6.
    d = DATA
    direct = d.c0 * (-d.f0 / 30 + (d.a0 + d.f0 / 6) / 3) + d.c1 * d.a1 / 15 + d.c2 * d.a2 / 35
    assert nh.objective(d, Fr(0)) == direct


@pytest.mark.parametrize("polarization,q_sign,with_f", [(Fr(1), -1, True), (Fr(3), -1, True), (Fr(3, 2), 1, True),
                                                         (Fr(3, 2), -1, False)])
def test_wrong_formulas_do_not_converge(polarization, q_sign, with_f):
    a = RADII[-1]
    wrong = nh.topological_derivative(DATA, polarization, q_sign)
    if not with_f:
        u, grad_dot, q, p = nh.centre_fields(DATA)
        wrong = wrong + DATA.f0 * p
    assert abs(nh.ratio(DATA, a) - wrong) > Fr(1, 100)


def test_harmonic_config_reduces_to_the_estimators_formula():
    """With f = 0 (the plain method's harmonic u) the formula is the one the
    gradient form's TD uses, 3/2 grad u . grad p - q u."""
    d = nh.Data(f0=Fr(0), a0=Fr(1, 2), a1=Fr(1, 2), a2=Fr(1), c0=Fr(2), c1=Fr(-1), c2=Fr(0))
    u, grad_dot, q, _ = nh.centre_fields(d)
    rows = nh.check(d, RADII)
    assert rows[0]["td"] == Fr(3, 2) * grad_dot - q * u
    assert abs(rows[-1]["error"]) <= 4 * RADII[-1] ** 2
