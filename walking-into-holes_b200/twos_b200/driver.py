"""Reference-compatible Python entry points over the wih_* executables.

The reference's Python drivers reach its compiled backend by argv and files
(benchmarks/compiled_bunny/run_compiled_benchmark.py:133-159 ``run_cpp``) or
through a persistent ``--serve`` child (benchmarks/distinct_adjoint/
run_persistent.py:106-124, benchmarks/submission_study/run_study.py:19-38).
These helpers keep the same signatures and return values and point them at
this package's executables, so a driver switches backend by swapping the
binary path.
"""
from __future__ import annotations

import json
import os
import subprocess
from pathlib import Path

from ._abi import BIN_DIR

WIH_TWOS = BIN_DIR / "wih_twos"
WIH_ADJOINT = BIN_DIR / "wih_adjoint"


def run_cpp(executable, mesh, points, output, summary, walks: int, seed: int, repeats: int, threads: int,
            trace=None, trace_sites: int = 0, precision: str | None = None, device: int | None = None) -> dict:
    """Same argv and return value as run_compiled_benchmark.py:133-159."""
    command = [
        str(executable or WIH_TWOS), "--mesh", str(mesh), "--points", str(points),
        "--output", str(output), "--summary", str(summary),
        "--walks", str(walks), "--seed", str(seed),
        "--repeats", str(repeats), "--threads", str(threads),
        "--epsilon", "0.0005", "--max-steps", "512",
        "--source-y-slope", "0.65",
    ]
    if trace is not None:
        command += ["--trace-output", str(trace), "--trace-sites", str(trace_sites)]
    if precision is not None:
        command += ["--precision", precision]
    if device is not None:
        command += ["--device", str(device)]
    environment = dict(os.environ)
    environment["OMP_NUM_THREADS"] = str(threads)
    subprocess.run(command, check=True, env=environment)
    return json.loads(Path(summary).read_text())


class ServeSession:
    """A persistent ``--serve`` child speaking the reference's framing:
    "<argc>\\n" then argc lines (argv[0] first), answered by "DONE <code>"."""

    def __init__(self, executable=None, log=None):
        self.executable = str(executable or WIH_ADJOINT)
        self._log = open(log, "w") if log else subprocess.DEVNULL
        self.proc = subprocess.Popen([self.executable, "--serve"], stdin=subprocess.PIPE, stdout=subprocess.PIPE,
                                     stderr=self._log, text=True, bufsize=1)

    def request(self, args: list[str]) -> int:
        argv = [self.executable] + [str(a) for a in args]
        self.proc.stdin.write(str(len(argv)) + "\n" + "\n".join(argv) + "\n")
        self.proc.stdin.flush()
        line = self.proc.stdout.readline().strip()
        if not line.startswith("DONE "):
            raise RuntimeError(f"serve session ended: {line!r}")
        return int(line.split()[1])

    def close(self) -> int:
        if self.proc.stdin:
            self.proc.stdin.close()
        code = self.proc.wait()
        if self._log not in (None, subprocess.DEVNULL):
            self._log.close()
        return code


WIH_STUDY = BIN_DIR / "wih_study"
WIH_ANALYTIC_QUERY = BIN_DIR / "wih_analytic_query"
WIH_COMPLIANCE_QUERY = BIN_DIR / "wih_compliance_query"


class StudySolver:
    """The study driver's solver (submission_study/run_study.py:19-38
    ``Solver.call``) over a ``--serve`` child of a wih_study executable: the
    same argv per request, the same files (points.txt, holes.txt, field.csv,
    kernel.json, request.json) under ``folder/tag``, and the same return
    value (field DataFrame, summary dict with request_wall_seconds)."""

    def __init__(self, mesh, config, folder, executable=None):
        self.mesh, self.config, self.folder = Path(mesh), Path(config), Path(folder)
        self.executable = str(executable or WIH_STUDY)
        self.session = None
        self.calls = []

    def call(self, tag, points, holes=(), radius=.065, mode="twos", walks=128, seed=7, hot=False, fd=False,
             diff=False, epsilon=.0002, offset=.004, precision=None):
        import time

        import numpy as np
        import pandas as pd
        d = self.folder / tag
        d.mkdir(parents=True, exist_ok=True)
        holes = np.asarray(holes).reshape(-1, 3)
        points = np.asarray(points).reshape(-1, 3)
        np.savetxt(d / "points.txt", points, fmt="%.17g")
        np.savetxt(d / "holes.txt", holes, fmt="%.17g")
        args = ["--mesh", str(self.mesh), "--config", str(self.config), "--points", str(d / "points.txt"),
                "--cavities", str(d / "holes.txt") if len(holes) else "", "--cavity-radius", str(radius),
                "--output", str(d / "field.csv"), "--summary", str(d / "kernel.json"), "--mode", mode,
                "--source-mode", "housing", "--walks", str(walks), "--repeats", "1", "--seed", str(seed),
                "--threads", "4", "--max-steps", "2048", "--epsilon", str(epsilon), "--hot-only", str(int(hot)),
                "--fd", str(int(fd)), "--diff", str(int(diff)), "--diff-offset", str(offset)]
        if precision is not None:
            args += ["--precision", precision]
        (d / "request.json").write_text(json.dumps([self.executable] + args, indent=2))
        if self.session is None:
            self.folder.mkdir(parents=True, exist_ok=True)
            self.session = ServeSession(self.executable, log=self.folder / "server.log")
        start = time.perf_counter()
        code = self.session.request(args)
        if code != 0:
            # The server stops after a failed request (study.cpp:373).
            self.close()
            raise RuntimeError(f"{d}: DONE {code} " + (self.folder / "server.log").read_text())
        meta = json.loads((d / "kernel.json").read_text())
        meta["request_wall_seconds"] = time.perf_counter() - start
        (d / "kernel.json").write_text(json.dumps(meta, indent=2))
        self.calls.append(meta)
        return pd.read_csv(d / "field.csv"), meta

    def close(self):
        if self.session is not None:
            self.session.close()
            self.session = None
