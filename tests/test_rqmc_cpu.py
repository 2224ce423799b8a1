"""Array-RQMC restated in the oracle (the 3D form of benchmarks/
critical_baselines/sampling.py:49-88) without a GPU.

* The Hilbert key: on every corner cube of side 2, 4, 8, 16 the keys are
  exactly 0 .. side^3 - 1 and consecutive keys are face neighbours (what a
  Hilbert curve is; the reference checks its 2D key against a library).
* On the unit ball with harmonic Dirichlet data for u and p the batch
  cross-fit estimates -u p; Array-RQMC (Hilbert order, Korobov lattice)
  lowers its mean-square error against the exact value well below matched
  Monte Carlo (the reference's finding in 2D).
* Neighbour reuse (reused_means, sampling.py:76-88, in 3D): the oracle's
  pooled means equal a numpy restatement on a random record; a lone site
  keeps its plain mean; a site on the boundary (first radius 0) lends no
  walks.
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


def reused_means_3d(sites, first, wu, wp, radius):
    """reused_means (sampling.py:76-88) with the 3D Poisson kernel ratio
    r (r^2 - |x-y|^2) / |x-z|^3 and weight (1-a)^4 / (1+a)^2 for one batch:
    first [n_sites, walks, 3], wu / wp [n_sites, walks], radius [n_sites]."""
    out = np.full((len(sites), 2), np.nan)
    with np.errstate(divide="ignore", invalid="ignore"):
        for k, x in enumerate(sites):
            a = np.linalg.norm(x - sites, axis=1) / radius
            valid = a < 1 - 1e-12
            if not valid.any():
                continue
            a, rv = a[valid], radius[valid]
            w = (1 - a) ** 4 / (1 + a) ** 2
            rho2 = np.sum((x - sites[valid]) ** 2, axis=1)
            kernel = rv[:, None] * (rv[:, None] ** 2 - rho2[:, None]) / np.linalg.norm(x - first[valid], axis=2) ** 3
            out[k, 0] = np.sum(w * np.mean(kernel * wu[valid], axis=1)) / w.sum()
            out[k, 1] = np.sum(w * np.mean(kernel * wp[valid], axis=1)) / w.sum()
    return out


def test_neighbour_means_match_numpy(oracle_mod):
    rng = np.random.default_rng(3)
    n_sites, walks, batches = 12, 40, 2
    sites = rng.uniform(-.5, .5, (n_sites, 3))
    radius = rng.uniform(.05, .6, n_sites)
    radius[3] = 0.0  # a site on the boundary: its walks stopped at once
    sites[3] = (5.0, 5.0, 5.0)  # ... and inside no other site's first ball
    d = rng.normal(size=(batches, n_sites, walks, 3))
    first = sites[None, :, None, :] + radius[None, :, None, None] * d / np.linalg.norm(d, axis=3, keepdims=True)
    wu, wp = rng.normal(size=(2, batches, n_sites, walks))
    plain_u, plain_p = wu.mean(2), wp.mean(2)
    bu, bp = plain_u.copy(), plain_p.copy()
    oracle_mod.lib().oracle_neighbour_means(*[oracle_mod._ptr(np.ascontiguousarray(v)) if isinstance(v, np.ndarray)
                                              else v for v in (sites, n_sites, batches, walks, first, wu, wp, radius,
                                                               bu, bp)])
    for b in range(batches):
        ref = reused_means_3d(sites, first[b], wu[b], wp[b], radius)
        lone = np.isnan(ref[:, 0])
        assert lone[3] and lone.sum() < n_sites - 1
        np.testing.assert_allclose(bu[b][~lone], ref[~lone, 0], rtol=1e-12)
        np.testing.assert_allclose(bp[b][~lone], ref[~lone, 1], rtol=1e-12)
        np.testing.assert_array_equal(bu[b][lone], plain_u[b][lone])
        np.testing.assert_array_equal(bp[b][lone], plain_p[b][lone])


def test_neighbour_reuse_lone_site_keeps_plain_mean(oracle_mod, lib_built):
    from twos_b200 import geometry
    V, F = geometry.icosphere(3)
    om = oracle_mod.OracleMesh(V, F)
    ub, pb = terms(oracle_mod.term, HARMONIC["u"]), terms(oracle_mod.term, HARMONIC["p"])
    kw = dict(rng=oracle_mod.RNG_COUNTER, walks=64, seed=5, epsilon=1e-5, max_steps=4096, source=[])
    site = np.array([[0.1, 0.2, 0.05]])
    bu0, bp0, steps0, _ = om.rqmc(site, 0, 2, 5, ub, pb, **kw)
    bu2, bp2, steps2, _, rec = om.rqmc(site, 2, 2, 5, ub, pb, record=True, **kw)
    assert steps0 == steps2
    # The kernel ratio of the site's own walks is r^3 / |x - z|^3 = 1 up to rounding.
    np.testing.assert_allclose(bu2, bu0, rtol=1e-12)
    np.testing.assert_allclose(bp2, bp0, rtol=1e-12)
    np.testing.assert_allclose(np.linalg.norm(rec["walk_first"] - site, axis=-1), rec["site_radius"][0], rtol=1e-12)
    np.testing.assert_allclose(rec["walk_u"].mean(-1), bu0, rtol=1e-12)
