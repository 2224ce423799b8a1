"""Launch tuning (twos_mesh_set_tuning) and the autotuner: results are a pure
function of the request and the samples, so every block size, refill
threshold, step threshold, occupancy cap, traversal-unit count and the
entry-node start give bit-identical rows (the distance-grid threshold changes
the walks' radii and is held fixed)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tb(lib_built):
    import twos_b200
    return twos_b200


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_every_tuning_gives_identical_rows(tb, bunny1000, eval_points, precision):
    cfg = tb.Config(walks=96, precision=precision, seed=3, source=tb.sources.affine(0.65))
    with tb.Mesh(*bunny1000) as mesh:
        ref, _ = mesh.estimate(eval_points, cfg)
        for block, refill, step, bps in [(256, 1, 1, 0), (512, 1, 1, 0), (128, 8, 8, 0), (128, 32, 32, 2),
                                         (256, 4, 16, 1)]:
            mesh.set_tuning(block=block, refill=refill, step_threshold=step, blocks_per_sm=bps)
            assert mesh.get_tuning() == {"block": block, "refill": refill, "step_threshold": step,
                                         "blocks_per_sm": bps, "grid_threshold": 0.1, "units": 8, "entry": 1,
                                         "grid_fp64": 0, "bvh_width": 2, "lane_walks": 1, "wavefront": 0}
            out, _ = mesh.estimate(eval_points, cfg)
            for k in ("u", "score", "score_se", "steps"):
                np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{k} {block} {refill} {step} {bps}")
        for units in (1, 3, 64):
            mesh.set_tuning(units=units)
            out, _ = mesh.estimate(eval_points, cfg)
            for k in ("u", "score", "score_se", "steps"):
                np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{k} units={units}")
        # The entry-node start and the BVH width change how a query's
        # traversal runs, never its minimum; walks per lane only which lane
        # runs a walk.
        for variant in (dict(entry=0), dict(bvh_width=4), dict(bvh_width=4, entry=0), dict(bvh_width=4, units=3),
                        dict(lane_walks=2), dict(lane_walks=4, refill=8), dict(lane_walks=64, block=512),
                        dict(lane_walks=3, block=256), dict(wavefront=1 << 20), dict(wavefront=512, units=1),
                        dict(wavefront=4096, entry=0, units=3), dict(wavefront=256, units=2)):
            mesh.set_tuning(**variant)
            out, _ = mesh.estimate(eval_points, cfg)
            for k in ("u", "score", "score_se", "steps"):
                np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{k} {variant}")


@pytest.mark.parametrize("mode", ["paired", "hot"])
def test_wavefront_form_gives_identical_rows_in_every_mode(tb, bunny1000, eval_points, mode):
    """The wavefront form runs the persistent kernel's walks: the same rows
    in the paired and hot modes too (the compliance mode is covered above),
    with cavities and their skipped sites."""
    cfg = tb.Config(walks=64, precision="mixed", seed=5, mode=mode, source=tb.sources.affine(0.65),
                    adjoint=tb.sources.constant(1.0), cavity_radius=0.02, skip_cavity_sites=True)
    cav = eval_points[:2] + 0.01
    with tb.Mesh(*bunny1000) as mesh:
        ref, _ = mesh.estimate(eval_points, cfg, cavities=cav)
        for slots in (256, 1 << 16):
            mesh.set_tuning(wavefront=slots)
            out, _ = mesh.estimate(eval_points, cfg, cavities=cav)
            for k in ref.dtype.names:
                np.testing.assert_array_equal(out[k], ref[k], err_msg=f"{k} {mode} {slots}")
        mesh.set_tuning()


def test_invalid_tuning_is_usage_error(tb, bunny1000):
    with tb.Mesh(*bunny1000) as mesh:
        for bad in [dict(block=96), dict(refill=0), dict(step_threshold=33), dict(blocks_per_sm=-1),
                    dict(grid_threshold=0.05), dict(grid_threshold=-1.0), dict(grid_threshold=float("nan")),
                    dict(units=0), dict(units=65), dict(entry=2), dict(grid_fp64=3),
                    dict(bvh_width=3), dict(lane_walks=0), dict(lane_walks=65), dict(lane_walks=2, bvh_width=4),
                    dict(wavefront=100),
                    dict(wavefront=-256), dict(wavefront=1 << 27)]:
            with pytest.raises(tb.TwosError) as e:
                mesh.set_tuning(**bad)
            assert e.value.code == 2


def test_autotuner_picks_a_grid_point(tb, bunny1000, eval_points, tmp_path):
    from twos_b200.autotune import autotune, DEFAULT_GRID
    cfg = tb.Config(walks=256, precision="mixed", seed=1, source=tb.sources.affine(0.65))
    cache = tmp_path / "tuning.json"
    with tb.Mesh(*bunny1000) as mesh:
        best, results = autotune(mesh, eval_points, cfg, calib_sites=256, calib_walks=64, repeats=1, cache=cache)
        assert mesh.get_tuning() == best
        # The default grid is swept whole, each valid setting once (walk
        # claims with the four-wide BVH are refused).
        import itertools
        names = list(DEFAULT_GRID)
        valid = [c for c in itertools.product(*DEFAULT_GRID.values())
                 if not (dict(zip(names, c))["bvh_width"] == 4 and dict(zip(names, c))["lane_walks"] > 1)]
        assert len({tuple(sorted(t.items())) for t, _ in results}) == len(results) == len(valid)
        assert all(best[k] in v for k, v in DEFAULT_GRID.items())
        assert all(t > 0 for _, t in results)
        again, cached = autotune(mesh, eval_points, cfg, cache=cache)
        assert again == best and cached == []
