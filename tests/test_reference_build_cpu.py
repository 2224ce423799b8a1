"""The reference's own compiled backend (benchmarks/compiled_bunny/src/
wih_twos.cpp, built unchanged against the project's Embree/Eigen shim
headers by `make -C oracle ref`) against its own tracked outputs: the field
of the 1,000- and 4,000-face bunnies (benchmarks/compiled_bunny/output/
field-bunny-0*-faces.csv; 32 walks, seed 20260912 + 1800, 3 repeats with
repeat 0 retained, eps 5e-4, max-steps 512, affine source of slope 0.65;
run_compiled_benchmark.py:754-760).  Integer step counts must reproduce
exactly; values differ only where Embree's FP32 query radius and the shim's
traversal order break a tie differently (the oracle's tolerances)."""
import gzip
import shutil

import numpy as np
import pandas as pd
import pytest

from conftest import GOLDEN

import ref_runner

pytestmark = pytest.mark.skipif(not ref_runner.available(), reason="oracle/_ref/wih_twos is not built")


@pytest.mark.parametrize("faces", [1000, 4000])
def test_reference_binary_reproduces_tracked_field(tmp_path, eval_points, faces):
    ply = tmp_path / "mesh.ply"
    with gzip.open(GOLDEN / f"bunny-{faces:05d}-faces.ply.gz", "rb") as f, open(ply, "wb") as g:
        shutil.copyfileobj(f, g)
    rows, summary, _ = ref_runner.run_compliance(ply, eval_points, walks=32, seed=20260912 + 1800, epsilon=5e-4,
                                                 max_steps=512, slope=0.65, repeats=3, workdir=tmp_path)
    ref = pd.read_csv(GOLDEN / "compiled_bunny" / f"field-bunny-{faces:05d}-faces.csv")
    np.testing.assert_array_equal(rows["steps"].astype(np.int64), ref["steps"].values)
    np.testing.assert_array_equal(rows["limit_hits"].astype(np.int64), ref["limit_hits"].values)
    np.testing.assert_allclose(rows["u"], ref["u"].values, rtol=2e-5)
    np.testing.assert_allclose(rows["score"], ref["score"].values, rtol=5e-5)
    np.testing.assert_allclose(rows["score_se"], ref["score_se"].values, rtol=2e-4)
    assert summary["faces"] == faces and summary["sites"] == 384 and summary["walks_per_site"] == 32
