"""Extract the golden fixtures used by the parity tests from the reference tree.

Run once in a container where the reference checkout is mounted:

    python tests/golden/make_fixtures.py /path/to/walking-into-holes

It copies (meshes gzip-compressed) the reference's own tracked inputs and
outputs for the TWoS backend:

* compliance fields of benchmarks/compiled_bunny/output/ (wih_twos --mode twos,
  affine source, eps 5e-4, max-steps 512, slope 0.65; argv from
  run_compiled_benchmark.py:133-159, seeds from :676-760);
* paired primal/adjoint requests of
  benchmarks/distinct_adjoint/persistent_output/ (wih_adjoint, housing
  source, sensor bump, Green-point sampling), with each request's argv.

The fixtures are committed, so tests never read the reference at run time.
"""
from __future__ import annotations

import gzip
import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

COMPLIANCE_FILES = [
    "evaluation-points.csv",
    "field-bunny-01000-faces.csv",
    "field-bunny-04000-faces.csv",
    "field-reference.csv",
    "field-twos-0016.csv",
    "reference-summary.json",
    "summary-bunny-01000-faces.json",
]
MESHES = {
    "benchmarks/compiled_bunny/output/bunny-01000-faces.ply": "bunny-01000-faces.ply.gz",
    "benchmarks/compiled_bunny/output/bunny-04000-faces.ply": "bunny-04000-faces.ply.gz",
    "benchmarks/stanford_bunny/output/stanford-bunny-watertight.ply": "stanford-bunny-watertight.ply.gz",
    "benchmarks/engineering_housing/assets/stylized-finned-housing.ply": "stylized-finned-housing.ply.gz",
}
MESHES["benchmarks/submission_study/assets/branch.ply"] = "branch.ply.gz"
# Differential-WoS requests of the study backend (wih_study --diff 1): argv in
# request.json, totals in kernel.json, per-cavity derivatives in field.csv.
GRADIENT = [
    "gradient-0.004-6",
    "gradient-0.008-0",
]
PAIRED = [
    "side1/seed2026091500/twos_sparse/round1/scout",
    "side1/seed2026091500/twos_dense/round2/rescore",
    "side1/seed2026091500/wos_hot/round3/scout",
    "side-1/seed2026091500/twos_sparse/round4/rescore",
]


def main(reference: Path) -> None:
    out = HERE
    for src, dst in MESHES.items():
        with open(reference / src, "rb") as fh, gzip.GzipFile(out / dst, "wb", compresslevel=9, mtime=0) as gz:
            shutil.copyfileobj(fh, gz)
    comp = out / "compiled_bunny"
    comp.mkdir(exist_ok=True)
    for name in COMPLIANCE_FILES:
        shutil.copyfile(reference / "benchmarks/compiled_bunny/output" / name, comp / name)
    paired = out / "distinct_adjoint"
    paired.mkdir(exist_ok=True)
    base = reference / "benchmarks/distinct_adjoint/persistent_output"
    index = []
    for rel in PAIRED:
        src = base / rel
        tag = rel.replace("/", "_")
        dst = paired / tag
        dst.mkdir(exist_ok=True)
        for name in ("points.csv", "holes.csv", "field.csv"):
            if (src / name).exists():
                shutil.copyfile(src / name, dst / name)
        summary = json.loads((src / "summary.json").read_text())
        argv = summary["command"][1:]
        # Paths in the recorded argv are remapped to the fixture's own files.
        keep = {}
        for key, value in zip(argv[0::2], argv[1::2]):
            if key in ("--mesh", "--points", "--output", "--summary", "--cavities"):
                continue
            keep[key] = value
        (dst / "argv.json").write_text(json.dumps(keep, indent=1, sort_keys=True) + "\n")
        index.append(tag)
    (paired / "index.json").write_text(json.dumps(index, indent=1) + "\n")
    grad = out / "submission_study"
    grad.mkdir(exist_ok=True)
    shutil.copyfile(reference / "benchmarks/submission_study/assets/branch.txt", grad / "branch.txt")
    gbase = reference / "benchmarks/submission_study/validation-v1-remote-sources/raw"
    for tag in GRADIENT:
        dst = grad / tag
        dst.mkdir(exist_ok=True)
        for name in ("points.txt", "holes.txt", "field.csv", "kernel.json"):
            shutil.copyfile(gbase / tag / name, dst / name)
        argv = json.loads((gbase / tag / "request.json").read_text())[1:]
        keep = {k: v for k, v in zip(argv[0::2], argv[1::2])
                if k not in ("--mesh", "--config", "--points", "--cavities", "--output", "--summary")}
        (dst / "argv.json").write_text(json.dumps(keep, indent=1, sort_keys=True) + "\n")
    # Paired and hot requests of the study's pilot pipeline (wih_study, the
    # branch geometry, the config's two remote heat sources).
    sbase = reference / "benchmarks/submission_study"
    for tag, rel in STUDY_REQUESTS.items():
        src = sbase / rel
        dst = grad / tag
        dst.mkdir(exist_ok=True)
        for name in ("points.txt", "holes.txt", "field.csv", "kernel.json"):
            shutil.copyfile(src / name, dst / name)
        argv = json.loads((src / "request.json").read_text())[1:]
        keep = {k: v for k, v in zip(argv[0::2], argv[1::2])
                if k not in ("--mesh", "--config", "--points", "--cavities", "--output", "--summary")}
        keep["has_cavities"] = bool(dict(zip(argv[0::2], argv[1::2])).get("--cavities"))
        (dst / "argv.json").write_text(json.dumps(keep, indent=1, sort_keys=True) + "\n")
    minimum_benefit(reference, out)
    controlled_experiments(reference, out)
    sampling_study(reference, out)


def sampling_study(reference: Path, out: Path) -> None:
    """Per-site TD estimates of the 2D sampling study (benchmarks/
    critical_baselines/sampling.py; output/sampling_fields.csv): repetition
    0 at 64 walks and repetition 1 at 256 walks, both domains, every method."""
    import csv
    dst = out / "critical_baselines"
    dst.mkdir(exist_ok=True)
    src = reference / "benchmarks/critical_baselines/output/sampling_fields.csv"
    with open(src) as f, open(dst / "sampling_fields_subset.csv", "w", newline="") as g:
        rows = csv.DictReader(f)
        w = csv.DictWriter(g, fieldnames=rows.fieldnames)
        w.writeheader()
        for row in rows:
            if (row["n"], row["rep"]) in (("64", "0"), ("256", "1")):
                w.writerow(row)
    shutil.copyfile(reference / "benchmarks/critical_baselines/output/sampling_manifest.json",
                    dst / "sampling_manifest.json")


def controlled_experiments(reference: Path, out: Path) -> None:
    """The seeded cross-fit bias experiment of experiments/
    run_controlled_experiments.py:250-321 (its tracked per-correlation rows
    and the summary's claims), which pins the statistics the device
    reduction computes."""
    dst = out / "controlled_experiments"
    dst.mkdir(exist_ok=True)
    shutil.copyfile(reference / "experiments/output/crossfit_bias.csv", dst / "crossfit_bias.csv")
    shutil.copyfile(reference / "experiments/output/summary.json", dst / "summary.json")


def minimum_benefit(reference: Path, out: Path) -> None:
    """Certified validation attempts of benchmarks/minimum_benefit/
    pilot-floor-policy: the finalist, the retained cavities, the stage JSON,
    the decision record and the first 4,096 of the 65,536 samples (enough
    for the n = 1024 and n = 4096 stages, which use a prefix)."""
    import gzip
    base = reference / "benchmarks/minimum_benefit/pilot-floor-policy"
    dst_root = out / "minimum_benefit"
    dst_root.mkdir(exist_ok=True)
    shutil.copyfile(base / "configuration.json", dst_root / "configuration.json")
    for tag, (kind, attempt) in MIN_BENEFIT.items():
        src = base / kind / attempt
        dst = dst_root / tag
        dst.mkdir(exist_ok=True)
        for name in ("validation-points.csv", "validation-holes.csv", "validation.json", "decision.json"):
            shutil.copyfile(src / name, dst / name)
        with open(src / "validation.csv") as f:
            head = [next(f) for _ in range(4097)]
        with gzip.open(dst / "validation-head.csv.gz", "wt") as g:
            g.writelines(head)


MIN_BENEFIT = {"bunny-00": ("bunny", "attempt-00"), "housing-01": ("housing", "attempt-01")}

STUDY_REQUESTS = {
    "paired-rescore": "pilot/pipeline/branch/twos-1611/raw/round2-rescore",
    "paired-scout": "pilot/pipeline/branch/twos-1611/raw/round3-scout",
    "hot-refine": "pilot/pipeline/branch/hot-1611/refine-raw/r0-trial1",
}


if __name__ == "__main__":
    main(Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
