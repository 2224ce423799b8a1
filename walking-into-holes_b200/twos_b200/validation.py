"""Host-side acceptance of a certified validation (the exact half of the
minimum-benefit protocol, benchmarks/minimum_benefit/
run_application_validation.py:41-140 and 231-248).

The device half is ``Mesh.validate`` (twos_validate): certified fresh samples
and their stage statistics.  This module turns them into a decision with the
reference's arithmetic: every bound is rounded one ulp toward the safe side
after rounding to nearest, sums of samples are exact (rationals), pi comes
from Machin's formula from below, and the candidate's membership is decided
by exact rational ray parity.

* ``exact_inside``     -- rational positive-axis ray parity (41-70).
* ``source_bounds``    -- outward bounds of f over the box z +- R for a source
                          given as terms (a leading constant, then linear or
                          Gaussian terms; 83-101).
* ``floor_benefit``    -- the temperature-floor certificate over a grid of
                          radii R in (r, clearance) (103-127).
* ``average_benefit``  -- the average-trace certificate (129-140).
* ``stage_record`` / ``decide`` -- the Hoeffding margin C sqrt(log/(2n)),
                          the state lower bound, the benefit lower bound per
                          stage and the accept decision (231-254).

These need only numpy and the standard library (fractions, math).
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

from ._abi import TERM_CONST, TERM_GAUSS, TERM_LINEAR


def _dn(x: float) -> float:
    return math.nextafter(float(x), -math.inf)


def _up(x: float) -> float:
    return math.nextafter(float(x), math.inf)


# ------------------------------------------------------------------ membership
def _orient(a, b, c):
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def exact_inside(point, V, F):
    """Whether ``point`` is inside the closed triangle mesh (V, F), by exact
    rational parity of the ray from the point along +axis: triangles whose
    projection strictly contains the point's projection are crossed at the
    rational height of the plane; an edge, vertex or coplanar hit makes the
    axis degenerate and the next axis is tried; a hit at the point itself
    means the point is on the surface (not inside).  Returns (inside, info);
    raises when all three axes are degenerate."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F)
    p = [Fraction(float(x)) for x in point]
    tri = V[F]
    for axis in range(3):
        u, v = [a for a in range(3) if a != axis]
        lo = tri[:, :, [u, v]].min(axis=1)
        hi = tri[:, :, [u, v]].max(axis=1)
        q2 = np.array([float(point[u]), float(point[v])])
        candidates = np.flatnonzero(np.all((lo <= q2) & (hi >= q2), axis=1))
        q = (p[u], p[v])
        crossings = 0
        degenerate = False
        for t in candidates:
            verts = [[Fraction(float(x)) for x in tri[t, k]] for k in range(3)]
            a, b, c = [(w[u], w[v]) for w in verts]
            area = _orient(a, b, c)
            if area == 0:
                if _orient(a, b, q) == 0 and _orient(a, c, q) == 0:
                    degenerate = True
                    break
                continue
            w = [_orient(q, b, c), _orient(a, q, c), _orient(a, b, q)]
            sign = 1 if area > 0 else -1
            if any(x * sign < 0 for x in w):
                continue
            if any(x == 0 for x in w):
                degenerate = True
                break
            height = sum(wk * vk[axis] for wk, vk in zip(w, verts)) / area
            if height == p[axis]:
                return False, {"axis": axis, "boundary": True}
            crossings += height > p[axis]
        if not degenerate:
            return bool(crossings % 2), {"axis": axis, "intersections": int(crossings), "rational_predicates": True}
    raise RuntimeError("all axis rays degenerate; no certified classification")


# ------------------------------------------------------------------ source bounds
def exp_lower(t: float) -> float:
    """(1 - t/1024)^1024 <= exp(-t), rounded down at every step."""
    a = max(0.0, _dn(1.0 - _up(t / 1024.0)))
    for _ in range(10):
        a = max(0.0, _dn(a * a))
    return a


def exp_upper(t: float) -> float:
    """1 / (1 + t/1024)^1024 >= exp(-t), the power rounded down, then the
    reciprocal rounded up."""
    a = _dn(1.0 + max(0.0, _dn(t / 1024.0)))
    for _ in range(10):
        a = _dn(a * a)
    return _up(1.0 / a)


def is_harmonic(terms) -> bool:
    """Only constant and linear terms (f harmonic, so its ball mean is its
    centre value)."""
    return all(t.kind in (TERM_CONST, TERM_LINEAR) for t in terms)


def source_bounds(z, R: float, terms):
    """(lower, upper) of the source over the box z +- R (outward rounding):
    a leading constant, then each linear term's range and each Gaussian's
    exp bounds from the nearest / farthest box coordinates."""
    terms = list(terms)
    lo = hi = 0.0
    start = 0
    if terms and terms[0].kind == TERM_CONST:
        lo = hi = float(terms[0].amp)
        start = 1
    for t in terms[start:]:
        if t.kind == TERM_LINEAR:
            k, a, o = int(t.axis), float(t.amp), float(t.offset)
            lo = _dn(lo + _dn(a * _dn(_dn(float(z[k]) - R) + o)))
            hi = _up(hi + _up(a * _up(_up(float(z[k]) + R) + o)))
        elif t.kind == TERM_GAUSS:
            upper = lower = 0.0
            for axis in range(3):
                d = abs(float(z[axis]) - float(t.c[axis]))
                far = _up(_up(_up(d) + R) / float(t.w[axis]))
                near = max(0.0, _dn(_dn(d) - R))
                near = max(0.0, _dn(near / float(t.w[axis])))
                upper = _up(upper + _up(far * far))
                lower = max(0.0, _dn(lower + max(0.0, _dn(near * near))))
            lo = _dn(lo + _dn(float(t.amp) * exp_lower(upper)))
            hi = _up(hi + _up(float(t.amp) * exp_upper(lower)))
        elif t.kind == TERM_CONST:
            lo = _dn(lo + float(t.amp))
            hi = _up(hi + float(t.amp))
        else:
            raise ValueError("certified source bounds take constant, linear and Gaussian terms")
    return max(0.0, lo), hi


def pi_lower() -> float:
    """pi from below: Machin's formula 16 atan(1/5) - 4 atan(1/239) with the
    alternating series summed exactly (12 and 5 terms), rounded down."""
    a = sum((Fraction((-1) ** k, (2 * k + 1) * 5 ** (2 * k + 1)) for k in range(12)), Fraction(0))
    b = sum((Fraction((-1) ** k, (2 * k + 1) * 239 ** (2 * k + 1)) for k in range(5)), Fraction(0))
    return _dn(float(16 * a - 4 * b))


# ------------------------------------------------------------------ certificates
def floor_benefit(L: float, z, r: float, clearance: float, terms):
    """The temperature-floor certificate: over 128 radii R in (r, 0.99
    clearance), the floor m = q_lo + c (L - q_hi)_+ of the trace on the
    cavity, with q the source's ball integral bounds and c = (1 - t)/(1 + t)^2,
    t = r/R; bound 4 pi r m^2.  Returns (best bound, geometry) with the
    first radius that attains it; (0, None) when clearance <= r."""
    if clearance <= r:
        return 0.0, None
    radii = np.linspace(np.nextafter(r, np.inf), 0.99 * clearance, 128)
    pi_lo = pi_lower()
    best = (-1.0, None)
    for R in radii:
        R = float(R)
        if not r < R < clearance:
            continue
        flo, fhi = source_bounds(z, R, terms)
        diff = max(0.0, _dn(_dn(R * R) - _up(r * r)))
        qlo = max(0.0, _dn(_dn(flo * diff) / 6))
        qhi = _up(_up(fhi * _up(R * R)) / 6)
        t = _up(r / R)
        den = _up(_up(1 + t) ** 2)
        c = max(0.0, _dn(_dn(1 - t) / den))
        h = max(0.0, _dn(L - qhi))
        m = max(0.0, _dn(qlo + max(0.0, _dn(c * h))))
        b = max(0.0, _dn(_dn(_dn(4 * pi_lo) * r) * max(0.0, _dn(m * m))))
        if b > best[0]:
            best = (b, dict(R=R, f_lower=flo, f_upper=fhi, temperature_floor=m))
    return best


def average_benefit(L: float, z, r: float, clearance: float, terms):
    """The average-trace certificate: the trace mean over the cavity sphere is
    at least L minus the source's ball integral (bounded above with f's upper
    bound over the ball, or its centre value when f is harmonic); bound
    4 pi r (trace lower)^2."""
    if not r < clearance:
        return 0.0, None
    _, fhi = source_bounds(z, 0.0 if is_harmonic(terms) else r, terms)
    ihi = _up(_up(fhi * _up(r * r)) / 6)
    trace_lower = max(0.0, _dn(L - ihi))
    bound = max(0.0, _dn(_dn(_dn(4 * pi_lower()) * r) * max(0.0, _dn(trace_lower * trace_lower))))
    return bound, dict(source_integral_upper=ihi, source_upper=fhi, trace_mean_lower=trace_lower)


def sampling_margin(value_cap: float, n: int, confidence_log_upper: float) -> float:
    """Hoeffding half-width C sqrt(log(1/delta) / (2 n)) for samples in
    [0, C], rounded up."""
    return _up(value_cap * _up(math.sqrt(_up(confidence_log_upper / (2 * n)))))


def exact_mean_lower(values, n: int) -> float:
    """The mean of the first n binary64 samples, summed exactly, rounded down."""
    s = sum((Fraction(float(v)) for v in np.asarray(values)[:n]), Fraction(0))
    return _dn(float(s / n))


def stage_record(values, n: int, clearance: float, z, r: float, terms, value_cap: float,
                 confidence_log_upper: float, target: float) -> dict:
    """One stage of the decision (run_application_validation.py:235-247)."""
    margin = sampling_margin(value_cap, n, confidence_log_upper)
    L = max(0.0, _dn(exact_mean_lower(values, n) - margin))
    floor_bound, geometry = floor_benefit(L, z, r, clearance, terms)
    avg_bound, avg_geometry = average_benefit(L, z, r, clearance, terms)
    bound = max(floor_bound, avg_bound)
    source_only, _ = floor_benefit(0.0, z, r, clearance, terms)
    return dict(n=int(n), sampling_margin=margin, state_lower=L, benefit_lower=bound, source_only_lower=source_only,
                floor_bound=floor_bound, average_bound=avg_bound, average_geometry=avg_geometry, geometry=geometry,
                passes=bool(bound >= target))


def decide(values, stages, z, r: float, terms, value_cap: float, confidence_log_upper: float, target: float):
    """Accept when the best stage's benefit lower bound reaches the target.
    ``values`` are one site's samples in order, ``stages`` its stage records
    (n and center_clearance_lower).  The samples must lie in [0, value_cap]
    and the record must have no containment failure (checked by the caller's
    device call).  Returns (accepted, stage records, best record)."""
    v = np.asarray(values, dtype=np.float64)
    if not np.all((v >= 0) & (v <= value_cap)):
        raise ValueError("samples outside [0, value_cap]")
    records = [stage_record(v, int(st["n"]), float(st["center_clearance_lower"]), z, r, terms, value_cap,
                            confidence_log_upper, target) for st in stages]
    best = max(records, key=lambda x: x["benefit_lower"])
    return bool(best["benefit_lower"] >= target), records, best
