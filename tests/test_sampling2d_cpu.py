"""The oracle's restatement of the reference's 2D sampling study
(oracle/sampling2d.py; benchmarks/critical_baselines/sampling.py) against the
study's own tracked per-site TD estimates (output/sampling_fields.csv, a
committed subset: repetition 0 at 64 walks and repetition 1 at 256 walks,
disk and square, every method): MC, Sobol-over-steps RQMC, Array-RQMC
(Hilbert order, shifted Korobov lattice) and neighbour reuse, each cross-fit
over 4 batches.  These are the estimators twos_rqmc runs in 3D; the random
draws follow the study's order, so the estimates reproduce to rounding."""
import numpy as np
import pandas as pd
import pytest

import sampling2d
from conftest import GOLDEN

FIELDS = pd.read_csv(GOLDEN / "critical_baselines" / "sampling_fields_subset.csv")


@pytest.mark.parametrize("domain_id,domain", [(0, "disk"), (1, "square")])
@pytest.mark.parametrize("method", ["mc", "rqmc", "array", "neighbors"])
def test_2d_study_estimates_reproduce(domain_id, domain, method):
    for n, rep in ((64, 0), (256, 1)):
        ref = FIELDS[(FIELDS.domain == domain) & (FIELDS.method == method) & (FIELDS.n == n) &
                     (FIELDS.rep == rep)].sort_values("site")
        assert len(ref) == 25
        td = sampling2d.td_estimate(domain_id, domain, n, rep, method)
        np.testing.assert_allclose(td, ref.estimate.values, rtol=0, atol=1e-14)
        sites = sampling2d.study_sites()
        np.testing.assert_allclose(sites.real, ref.x.values, atol=1e-15)
        u, p = sampling2d.harmonic_fields(sites)
        np.testing.assert_allclose(-u * p, ref.exact.values, rtol=1e-14)


def test_hilbert_order_is_a_bijection_on_a_small_grid():
    bits = 3
    g = (np.arange(8) + 0.5) / 8 * 2 - 1
    z = (g[:, None] + 1j * g[None, :]).ravel()
    h = sampling2d.hilbert2(z, bits=bits)
    assert sorted(h.tolist()) == list(range(64))
    # Consecutive indices are neighbouring cells.
    cells = np.stack([np.floor((z.real + 1) * 4), np.floor((z.imag + 1) * 4)], 1)[np.argsort(h)]
    assert np.all(np.abs(np.diff(cells, axis=0)).sum(1) == 1)
