"""Source terms of the reference's walks, as twos_source_term lists.

A source is the ordered sum of its terms, evaluated exactly in that order so
the FP64 form reproduces the reference's arithmetic.
"""
from __future__ import annotations

import math

from ._abi import (SourceTerm, TERM_BALL, TERM_BOX, TERM_BUMP, TERM_CONST, TERM_GAUSS, TERM_LINEAR, TERM_QUAD)


def term(kind, amp=1.0, axis=0, offset=0.0, div=1.0, c=(0.0, 0.0, 0.0), w=(1.0, 1.0, 1.0)) -> SourceTerm:
    t = SourceTerm()
    t.kind, t.axis, t.amp, t.offset, t.div = int(kind), int(axis), float(amp), float(offset), float(div)
    t.c[:] = [float(v) for v in c]
    t.w[:] = [float(v) for v in w]
    return t


def constant(value=1.0):
    """f = value (the uniform Poisson source f = 1)."""
    return [term(TERM_CONST, value)]


def affine(slope=0.65):
    """f = 1 + slope*(y + 0.5) (benchmarks/compiled_bunny/src/wih_twos.cpp:550-552)."""
    return [term(TERM_CONST, 1.0), term(TERM_LINEAR, slope, axis=1, offset=0.5)]


def housing():
    """0.08 + 5.2 chip_a + 4.6 chip_b + 2.0 regulator (wih_twos.cpp:553-565)."""
    return [
        term(TERM_CONST, 0.08),
        term(TERM_GAUSS, 5.2, c=(-0.48, -0.18, -0.08), w=(0.24, 0.22, 0.16)),
        term(TERM_GAUSS, 4.6, c=(0.43, 0.19, -0.07), w=(0.21, 0.20, 0.15)),
        term(TERM_GAUSS, 2.0, c=(0.02, -0.31, -0.02), w=(0.30, 0.16, 0.19)),
    ]


def sensor(side=1, radius=0.13):
    """Sensor bump (1 - |x-c|^2/R^2)_+^2 about (0.55 s, 0.18 s, -0.03)
    (benchmarks/distinct_adjoint/adjoint.cpp:11-15, 98-102)."""
    return [term(TERM_BUMP, 1.0, c=(0.55 * side, 0.18 * side, -0.03), w=(radius, 0.0, 0.0))]


def normalized_sensor(center, radius=0.13):
    """Bump divided by its integral 32 pi R^3/105
    (benchmarks/submission_study/study.cpp:45-47)."""
    return [term(TERM_BUMP, 1.0, div=32 * 3.141592653589793 * radius ** 3 / 105, c=center, w=(radius, 0, 0))]


def box_indicator(lo, hi, amp=1.0):
    """amp on the box lo <= x <= hi (infinite bounds allowed)."""
    return [term(TERM_BOX, amp, c=lo, w=hi)]


def ball_indicator(center, radius, amp=1.0):
    """amp on the ball |x - c| <= r."""
    return [term(TERM_BALL, amp, c=center, w=(radius, 0.0, 0.0))]


def ball_mean_density(center, radius):
    """1_{|x-c|<r} / |B_r|: the density of a mean over a ball."""
    return ball_indicator(center, radius, amp=1.0 / (4.0 / 3.0 * math.pi * radius ** 3))


def study_heat(rows):
    """Heat lines (x, y, z, r, A) of a study configuration as the source
    sum of A (1 - |x-c|^2/r^2)_+^2 in file order
    (benchmarks/submission_study/study.cpp:27-35)."""
    return [term(TERM_BUMP, r[4], c=tuple(r[:3]), w=(r[3], 0.0, 0.0)) for r in rows]


def load_study_config(path):
    """A study configuration file (benchmarks/submission_study/study.cpp:37-42):
    a sensor "x y z r", then heat records "x y z r A", read as one stream of
    numbers (line breaks do not matter; reading stops at the first token that
    is not a number or at an incomplete record).  Returns ((x, y, z, r), heat
    terms).  Raises ValueError on a bad sensor or without heat records."""
    values = []
    with open(path) as f:
        for tok in f.read().split():
            try:
                values.append(float(tok))
            except ValueError:
                break
    if len(values) < 4:
        raise ValueError(f"{path}: bad sensor config")
    rest = values[4:]
    heat = [rest[i:i + 5] for i in range(0, len(rest) - 4, 5)]
    if not heat:
        raise ValueError(f"{path}: missing compact heat sources")
    return tuple(values[:4]), study_heat(heat)


def quadratic(weights, amp=1.0, center=(0.0, 0.0, 0.0)):
    """amp * sum_k weights_k (x_k - c_k)^2 (harmonic when the weights sum to
    zero), e.g. boundary data x0^2 - x1^2 = quadratic((1, -1, 0))."""
    return [term(TERM_QUAD, amp, c=center, w=tuple(weights))]


def linear(slope, axis, offset=0.0):
    """slope * (x[axis] + offset)."""
    return [term(TERM_LINEAR, slope, axis=axis, offset=offset)]
