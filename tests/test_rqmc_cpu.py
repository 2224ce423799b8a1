"""Array-RQMC restated in the oracle (the 3D form of benchmarks/
critical_baselines/sampling.py:49-88) without a GPU.

* The Hilbert key: on every corner cube of side 2, 4, 8, 16 the keys are
  exactly 0 .. side^3 - 1 and consecutive keys are face neighbours (what a
  Hilbert curve is; the reference checks its 2D key against a library).
* On the unit ball with harmonic Dirichlet data for u and p the batch
  cross-fit estimates -u p; Array-RQMC (Hilbert order, Korobov lattice)
  lowers its mean-square error against the exact value well below matched
  Monte Carlo (the reference's finding in 2D).
"""
import numpy as np

HARMONIC = dict(u=[(0, .28, 0, (1, 1, 1)), (1, .58, 0, (1, 1, 1)), (1, -.30, 1, (1, 1, 1)), (6, .22, 0, (1, -1, 0))],
                p=[(0, .46, 0, (1, 1, 1)), (1, -.38, 0, (1, 1, 1)), (1, .34, 1, (1, 1, 1)), (6, .40, 0, (0, 1, -1))])


def fields(sites):
    x, y, z = sites.T
    return .28 + .58 * x - .30 * y + .22 * (x * x - y * y), .46 - .38 * x + .34 * y + .40 * (y * y - z * z)


def grid_sites(k=5):
    g = np.linspace(-.55, .55, k)
    return np.array([[a, b, 0.1] for a in g for b in g])


def terms(make, spec):
    return [make(kind, amp, axis=axis, w=w) for kind, amp, axis, w in spec]


def test_hilbert_key_is_a_hilbert_curve(oracle_mod):
    L = oracle_mod.lib()
    for side in (2, 4, 8, 16):
        cells = [(x, y, z) for x in range(side) for y in range(side) for z in range(side)]
        keys = [L.oracle_hilbert_key(*c) for c in cells]
        assert sorted(keys) == list(range(side ** 3))
        order = [c for _, c in sorted(zip(keys, cells))]
        assert all(sum(abs(a - b) for a, b in zip(order[i], order[i + 1])) == 1 for i in range(len(order) - 1))


def test_array_rqmc_beats_mc(oracle_mod, lib_built):
    from twos_b200 import geometry
    V, F = geometry.icosphere(3)
    om = oracle_mod.OracleMesh(V, F)
    sites = grid_sites(3)
    u, p = fields(sites)
    exact = -u * p
    ub, pb = terms(oracle_mod.term, HARMONIC["u"]), terms(oracle_mod.term, HARMONIC["p"])
    mse = {}
    for method in (0, 1):
        errs = []
        for rep in range(8):
            bu, bp, _, caps = om.rqmc(sites, method, 4, 13, ub, pb, rng=oracle_mod.RNG_COUNTER, walks=256,
                                      seed=100 + rep, epsilon=1e-5, max_steps=4096, source=[])
            assert caps == 0
            R = 4
            td = -(bu.sum(0) * bp.sum(0) - (bu * bp).sum(0)) / (R * (R - 1))
            errs.append(np.mean((td - exact) ** 2))
        mse[method] = np.mean(errs)
    assert mse[1] < 0.5 * mse[0], mse
