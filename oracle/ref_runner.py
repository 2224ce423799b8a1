"""TEST INFRASTRUCTURE and CPU baseline: runs the reference's own compiled
backend (benchmarks/compiled_bunny/src/wih_twos.cpp, built unchanged into
oracle/_ref/wih_twos against the project's Embree/Eigen shim headers by
`make -C oracle ref`) through its own interface: an ASCII PLY mesh and a
points CSV in, the field CSV and summary JSON out (wih_twos.cpp:1715-1792),
argv as run_cpp passes it (benchmarks/compiled_bunny/
run_compiled_benchmark.py:133-159).

The reference's compliance source is f = 1 + slope * (y + 0.5)
(wih_twos.cpp:546-549); slope 0 gives the uniform source f = 1.
"""
from __future__ import annotations

import json
import os
import platform
import subprocess
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BINARY = HERE / "_ref" / "wih_twos"


def available() -> bool:
    return BINARY.exists() and os.access(BINARY, os.X_OK)


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def write_ply(path: Path, V: np.ndarray, F: np.ndarray) -> None:
    """ASCII triangle PLY with 17 significant digits (the reader takes doubles)."""
    V = np.asarray(V, dtype=np.float64)
    F = np.asarray(F, dtype=np.int64)
    with open(path, "w") as f:
        f.write(f"ply\nformat ascii 1.0\nelement vertex {len(V)}\nproperty double x\nproperty double y\n"
                f"property double z\nelement face {len(F)}\nproperty list uchar int vertex_indices\nend_header\n")
        np.savetxt(f, V, fmt="%.17g")
        np.savetxt(f, np.c_[np.full(len(F), 3), F], fmt="%d")


def write_points(path: Path, P: np.ndarray) -> None:
    np.savetxt(path, np.asarray(P, dtype=np.float64), fmt="%.17g", delimiter=",", header="x,y,z", comments="")


def run_compliance(mesh_ply: Path, sites: np.ndarray, walks: int, seed: int, epsilon: float, max_steps: int,
                   slope: float = 0.0, threads: int | None = None, repeats: int = 1, workdir: Path | None = None):
    """One `wih_twos --mode twos` request.  Returns the field rows (u, score,
    score_se, steps, limit_hits as arrays), the summary JSON and the wall
    time of the process.  Raises on a nonzero exit."""
    if not available():
        raise FileNotFoundError(f"{BINARY} is not built (make -C oracle ref)")
    threads = threads or host_threads()
    tmp = tempfile.TemporaryDirectory() if workdir is None else None
    wd = Path(tmp.name) if tmp else Path(workdir)
    try:
        pts, out, summ = wd / "points.csv", wd / "field.csv", wd / "summary.json"
        write_points(pts, sites)
        argv = [str(BINARY), "--mode", "twos", "--mesh", str(mesh_ply), "--points", str(pts), "--output", str(out),
                "--summary", str(summ), "--walks", str(walks), "--seed", str(seed), "--epsilon", repr(epsilon),
                "--max-steps", str(max_steps), "--source-mode", "affine", "--source-y-slope", repr(slope),
                "--repeats", str(repeats), "--threads", str(threads)]
        env = dict(os.environ, OMP_PROC_BIND="true", OMP_NUM_THREADS=str(threads))
        t0 = time.perf_counter()
        r = subprocess.run(argv, capture_output=True, text=True, env=env)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"wih_twos exited {r.returncode}: {r.stderr.strip()[-400:]}")
        data = np.genfromtxt(out, delimiter=",", names=True)
        rows = {k: np.atleast_1d(data[k]) for k in ("u", "score", "score_se", "steps", "limit_hits")}
        return rows, json.loads(summ.read_text()), wall
    finally:
        if tmp:
            tmp.cleanup()
