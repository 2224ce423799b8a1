"""TEST INFRASTRUCTURE: exact finite-hole check of the Neumann-cavity
topological derivative, in rational arithmetic.

The reference implements only Dirichlet cavities; its exact cavity audit
(benchmarks/exact_cavity_audit/audit.py:11-27) checks the Dirichlet formula
on a concentric hole of the unit ball with Fractions.  This module does the
same for the Neumann hole that the gradient form's topological derivative
assumes, so the formula

    D_T = (3/2) grad u . grad p - q u - f p      (at the hole centre)

is checked by solving the finite-hole problem exactly, not by Monte Carlo.

Problem on Omega_a = {a < r < 1} (unit ball minus a concentric ball B_a):
    -Lap u = f0            in Omega_a
          u = g             on r = 1,   g = a0 + a1 z + a2 P2-term
      du/dn = 0             on r = a    (the Neumann hole)
    J(a)  = int_{Omega_a} q u dx,       q = c0 + c1 z + c2 r^2 P2(cos t)
Adjoint on the unperturbed ball: -Lap p = q, p = 0 on r = 1.

Separation of variables in Legendre modes l = 0, 1, 2 (u_l = A r^l + B r^-(l+1)
plus the particular radial part of the source) gives u on the annulus in
closed form; J is then an integral of Laurent polynomials in r times the
orthogonality constants 4 pi / (2l + 1).  Everything below omits the common
factor 4 pi, as the reference's audit does, so every quantity is a Fraction.

As a -> 0, (J(a) - J(0)) / |B_a| -> D_T with an error O(a^2); `check`
returns the ratio, D_T and the error at each radius.
"""
from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction as Fr


@dataclass(frozen=True)
class Data:
    """Source f0, Dirichlet modes (a0, a1, a2) of g on r = 1 and the modes
    (c0, c1, c2) of the objective's density q."""
    f0: Fr
    a0: Fr
    a1: Fr
    a2: Fr
    c0: Fr
    c1: Fr
    c2: Fr


def annulus_modes(d: Data, a: Fr):
    """Coefficients of u on a < r < 1 for a Neumann hole of radius a (a = 0:
    the unperturbed ball).  Mode 0: -f0 r^2/6 + A0 + B0/r; mode 1: (A1 r +
    B1 r^-2) P1; mode 2: (A2 r^2 + B2 r^-3) P2.  The Neumann condition at
    r = a gives B0 = -f0 a^3/3, B1 = A1 a^3/2, B2 = 2 A2 a^5/3; the Dirichlet
    data at r = 1 fixes the A's."""
    B0 = -d.f0 * a ** 3 / 3
    A0 = d.a0 + d.f0 / 6 - B0
    A1 = d.a1 / (1 + a ** 3 / 2)
    B1 = A1 * a ** 3 / 2
    A2 = d.a2 / (1 + 2 * a ** 5 / 3)
    B2 = 2 * A2 * a ** 5 / 3
    return A0, B0, A1, B1, A2, B2


def objective(d: Data, a: Fr) -> Fr:
    """J(a) / (4 pi): sum over modes of (angular constant) x int_a^1 r^2 Q_l U_l dr,
    with angular constants 1, 1/3, 1/5 and Q_0 = c0, Q_1 = c1 r, Q_2 = c2 r^2."""
    A0, B0, A1, B1, A2, B2 = annulus_modes(d, a)
    one = Fr(1)
    # int_a^1 r^2 (-f0 r^2/6 + A0 + B0/r) dr
    m0 = -d.f0 * (one - a ** 5) / 30 + A0 * (one - a ** 3) / 3 + B0 * (one - a ** 2) / 2
    # int_a^1 r^3 (A1 r + B1 r^-2) dr
    m1 = A1 * (one - a ** 5) / 5 + B1 * (one - a ** 2) / 2
    # int_a^1 r^4 (A2 r^2 + B2 r^-3) dr
    m2 = A2 * (one - a ** 7) / 7 + B2 * (one - a ** 2) / 2
    return d.c0 * m0 + d.c1 * m1 / 3 + d.c2 * m2 / 5


def centre_fields(d: Data):
    """u, grad u . grad p, q and p at the hole centre for the unperturbed
    problem.  u0 = -f0 r^2/6 + a0 + f0/6 + a1 z + a2 r^2 P2, so u(0) = a0 + f0/6
    and grad u(0) = (0, 0, a1).  The adjoint p = c0 (1 - r^2)/6 + c1 z (1 - r^2)/10
    + c2 r^2 P2 (1 - r^2)/14 (Lap(h r^2) = (6 + 4l) h for a degree-l harmonic h),
    so p(0) = c0/6 and grad p(0) = (0, 0, c1/10)."""
    u = d.a0 + d.f0 / 6
    grad_dot = d.a1 * d.c1 / 10
    return u, grad_dot, d.c0, d.c0 / 6


def topological_derivative(d: Data, polarization: Fr = Fr(3, 2), q_sign: int = -1) -> Fr:
    """D_T = polarization * grad u . grad p + q_sign * q u - f p at the centre.
    The defaults are the formula under test; other values let a test show
    that a wrong coefficient or sign does not converge."""
    u, grad_dot, q, p = centre_fields(d)
    return polarization * grad_dot + q_sign * q * u - d.f0 * p


def ratio(d: Data, a: Fr) -> Fr:
    """(J(a) - J(0)) / |B_a|, with |B_a| / (4 pi) = a^3 / 3."""
    return (objective(d, a) - objective(d, Fr(0))) / (a ** 3 / 3)


def check(d: Data, radii) -> list[dict]:
    """Exact ratio, the formula and their difference at each radius."""
    dt = topological_derivative(d)
    return [{"radius": a, "ratio": ratio(d, a), "td": dt, "error": ratio(d, a) - dt} for a in radii]
