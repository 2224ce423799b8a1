"""The oracle's gradient form against the analytic fields of the plain
method (the unit-sphere workload; see tests/test_gpu_gradient.py for the
fields).
No reference output exists for a Neumann cavity (the reference implements
only Dirichlet cavities), so this pins the restatement to the analytic
u = g, grad u . grad p and their standard errors."""
import numpy as np

from test_gpu_gradient import analytic


def test_oracle_gradient_config1(oracle_mod):
    import sys
    from conftest import PKG
    sys.path.insert(0, str(PKG))
    from twos_b200 import geometry
    V, F = geometry.icosphere(4)
    rng = np.random.default_rng(0)
    d = rng.normal(size=(64, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    sites = d * (0.9 * rng.random(64) ** (1 / 3))[:, None]
    T = oracle_mod.term
    boundary = [T(6, 1.0, w=(1.0, -1.0, 0.0)), T(oracle_mod.TERM_LINEAR, 0.5, axis=2)]
    q = [T(oracle_mod.TERM_BALL, 1.0 / (4 / 3 * np.pi * 0.5 ** 3), c=(0, 0, 0), w=(0.5, 0, 0))]
    o = oracle_mod.OracleMesh(V, F).estimate_gradient(
        sites, rng=oracle_mod.RNG_COUNTER, mode=1, walks=1024, seed=5, epsilon=1e-4, max_steps=4096, green=True,
        source=[], adjoint=q, boundary=boundary)
    g, grad_g, grad_p, _ = analytic(sites)
    assert int(o["caps"].sum()) == 0
    assert np.mean(np.abs(o["u"] - g)) < 0.03
    z = (o["cross"] - np.sum(grad_g * grad_p, axis=1)) / o["cross_se"]
    assert np.max(np.abs(z)) < 4.5 and np.mean(np.abs(z) < 3) >= 0.95 and abs(np.mean(z)) < 0.6
