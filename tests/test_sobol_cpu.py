"""The Sobol' sequence of twos_rqmc's SOBOL method (Sobol-over-steps RQMC,
benchmarks/critical_baselines/sampling.py:49-60 in 3D), on the host:

* the library's direction numbers (twos_sobol_directions: primitivity by the
  factors of 2^s - 1, Sobol's recurrence on the m_k) equal the oracle's
  (primitivity by counting the order of x, the recurrence on the fixed-point
  V_k), bit for bit;
* dimensions 0 and 1 are the canonical ones: the first 2^m points equal
  scipy's unscrambled Sobol' points (the reference study's generator);
* every one-dimensional projection of the first 2^m points, plain or
  scrambled as the method scrambles, is a (0, m, 1)-net;
* in the reference's own 2D study (the oracle's restatement, one coordinate
  per step) the sequence cuts the TD mean-square error like the study's scipy
  Sobol' does."""
import numpy as np
import pytest

import oracle
import sampling2d


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


def test_library_directions_equal_the_oracle(tb):
    for dims, bits in ((512, 10), (5000, 16), (3, 32)):
        np.testing.assert_array_equal(tb.sobol_directions(dims, bits), oracle.sobol_directions(dims, bits))


def test_usage_errors(tb):
    for dims, bits in ((0, 10), (10, 0), (10, 33), (70000, 10)):
        with pytest.raises(tb.TwosError) as e:
            tb.sobol_directions(dims, bits)
        assert e.value.code == 2


def _points(v, n):
    """Unscrambled points 0..n-1 from direction numbers v [dims, bits]."""
    x = np.zeros((n, v.shape[0]), dtype=np.uint64)
    idx = np.arange(n)
    for b in range(v.shape[1]):
        x[(idx >> b) & 1 == 1] ^= v[:, b].astype(np.uint64)
    return x


def test_first_two_dimensions_are_scipys():
    from scipy.stats import qmc
    m = 10
    ours = _points(oracle.sobol_directions(2, 32), 1 << m).astype(np.float64) / 2.0 ** 32
    theirs = qmc.Sobol(2, scramble=False).random_base2(m)
    key = lambda a: np.lexsort((a[:, 1], a[:, 0]))  # noqa: E731 -- the same point sets, in any order
    np.testing.assert_array_equal(ours[key(ours)], theirs[key(theirs)])


@pytest.mark.parametrize("scrambled", [False, True])
def test_every_coordinate_is_a_0m1_net(scrambled):
    m, dims = 10, 512
    if scrambled:
        u = sampling2d.own_sobol_points(1 << m, dims, np.random.default_rng(5))
        assert u.min() > 0.0 and u.max() < 1.0
        cells = np.floor(u * (1 << m)).astype(np.int64)
    else:
        cells = (_points(oracle.sobol_directions(dims, m), 1 << m) >> np.uint64(32 - m)).astype(np.int64)
    # Each of the 2^m cells of width 2^-m holds exactly one point, in every coordinate.
    assert all(np.array_equal(np.sort(cells[:, d]), np.arange(1 << m)) for d in range(dims))


def test_own_sequence_in_the_reference_2d_study():
    """Disk, 25 sites, 256 walks, 4 batches, 6 repetitions: MC, the study's
    scipy Sobol-over-steps and the same method on this sequence."""
    sites = sampling2d.study_sites()
    u, p = sampling2d.harmonic_fields(sites)
    exact = -u * p
    mse = {m: np.mean([np.mean((sampling2d.td_estimate(0, "disk", 256, rep, m) - exact) ** 2) for rep in range(6)])
           for m in ("mc", "rqmc", "sobol_own")}
    assert mse["sobol_own"] < 0.5 * mse["mc"], mse
    assert mse["sobol_own"] < 2.0 * mse["rqmc"], mse
