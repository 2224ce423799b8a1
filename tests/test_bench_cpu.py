"""bench.py's reference arm on the host cores (no GPU): one JSON line with the
contract's keys, the reference arm's marker, a bounded CPU sample of the
reference's own compiled backend (oracle/_ref/wih_twos; the oracle port when
it is not built), and the same workload keys as the GPU arm reports."""
import contextlib
import io
import json


def test_reference_arm_prints_the_contract_line(lib_built):
    import bench
    import ref_runner
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.main(["--impl", "reference", "--steps", "2", "--warmup", "1", "--walks", "64", "--ref-sites", "6"])
    lines = [l for l in buf.getvalue().splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 2
    assert d["cpu_baseline"]["kind"] == ("reference" if ref_runner.available() else "port")
    assert d["cpu_baseline"]["cores"] >= 1 and d["cpu_baseline"]["cpu_model"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    V, F, grid = bench.workload(64)
    assert d["config"] == bench.workload_config(len(bench.workload_sites(grid)), 64)


def test_reference_subset_is_fixed():
    import bench
    a = bench.reference_subset(122000, 1024)
    assert len(a) == 1024 and len(set(a.tolist())) == 1024
    assert (a == bench.reference_subset(122000, 1024)).all()
