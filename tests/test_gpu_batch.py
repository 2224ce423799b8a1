"""Batched multi-geometry launch (twos_estimate_batch): uneven meshes, site
counts and walk counts in one persistent launch give exactly the rows of one
twos_estimate call per job (same counter-stream samples, same fixed-order
FP64 reductions), in both precisions; step caps and usage errors keep the
single-call behaviour."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


def _jobs(tb):
    meshes, sites, walks = [], [], []
    for k, (level, seed) in enumerate([(2, 2), (3, 3), (4, 4), (3, 5)]):
        V, F = tb.geometry.noise_sphere(level, seed)
        meshes.append(tb.Mesh(V, F))
        sites.append(tb.geometry.uniform_ball([37, 5, 120, 64][k], 0.5, seed=k))
        walks.append([64, 300, 16, 128][k])
    return meshes, sites, walks


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_equals_individual_calls(tb, precision):
    meshes, sites, walks = _jobs(tb)
    try:
        cfgs = [tb.Config(walks=w, precision=precision, seed=100 + j, epsilon=1e-4, source=tb.sources.constant(1.0))
                for j, w in enumerate(walks)]
        outs, summ = tb.estimate_batch(meshes, sites, cfgs)
        total_steps = 0
        for m, s, c, o in zip(meshes, sites, cfgs, outs):
            ref, rs = m.estimate(s, c)
            total_steps += rs["steps"]
            for k in ("u", "p", "score", "score_se", "same_index", "steps", "caps"):
                np.testing.assert_array_equal(o[k], ref[k], err_msg=k)
        assert summ["steps"] == total_steps
        assert summ["paths"] == sum(len(s) * w for s, w in zip(sites, walks))
        assert summ["launches"] == 3  # site pre-pass, walk kernel, finalize
    finally:
        for m in meshes:
            m.close()


def test_batch_paired_with_cavities(tb):
    meshes, sites, walks = _jobs(tb)
    try:
        cav = [np.array([[0.1, 0.0, 0.0]]), None, np.array([[0.0, 0.1, 0.0], [-0.2, 0.0, 0.0]]), None]
        cfgs = [tb.Config(walks=w, mode="paired", precision="mixed", seed=7, epsilon=1e-4, green=True,
                          cavity_radius=0.05, source=tb.sources.constant(1.0),
                          adjoint=tb.sources.ball_indicator((0, 0, 0), 0.5)) for w in walks]
        outs, _ = tb.estimate_batch(meshes, sites, cfgs, cav)
        for m, s, c, cv, o in zip(meshes, sites, cfgs, cav, outs):
            ref, _ = m.estimate(s, c, cavities=cv)
            for k in ("u", "p", "score", "score_se", "steps"):
                np.testing.assert_array_equal(o[k], ref[k], err_msg=k)
    finally:
        for m in meshes:
            m.close()


def test_batch_usage_errors(tb):
    meshes, sites, walks = _jobs(tb)
    try:
        cfgs = [tb.Config(walks=w, precision="mixed") for w in walks]
        cfgs[1].precision = "fp64"
        with pytest.raises(tb.TwosError) as e:
            tb.estimate_batch(meshes, sites, cfgs)
        assert e.value.code == 2
    finally:
        for m in meshes:
            m.close()


def test_batch_splits_launches_to_keep_tables_in_shared_memory(tb):
    """Twelve jobs on twelve meshes: their job and geometry descriptors
    exceed the walk kernel's shared-memory table budget, so the batch runs
    as several launches (three kernels each) with the same rows as one call
    per job."""
    meshes, sites, cfgs = [], [], []
    try:
        for j in range(12):
            V, F = tb.geometry.noise_sphere(1 + j % 2, 50 + j)
            meshes.append(tb.Mesh(V, F))
            sites.append(tb.geometry.uniform_ball(9 + j, 0.4, seed=200 + j))
            cfgs.append(tb.Config(walks=32, precision="mixed", seed=300 + j, epsilon=1e-4,
                                  source=tb.sources.constant(1.0)))
        outs, summ = tb.estimate_batch(meshes, sites, cfgs)
        assert summ["launches"] > 3 and summ["launches"] % 3 == 0
        for m, s, c, o in zip(meshes, sites, cfgs, outs):
            ref, _ = m.estimate(s, c)
            for k in ("u", "score", "score_se", "steps"):
                np.testing.assert_array_equal(o[k], ref[k], err_msg=k)
    finally:
        for m in meshes:
            m.close()
