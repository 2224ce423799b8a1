#!/usr/bin/env python
"""Benchmark: TD site-estimates/s at equal 95% CI (mixed vs FP64 GPU, vs host CPU).

Workload (one "step"): the compliance TWoS estimator over every interior
site of the noise-displaced icosphere -- subdivision 7 (327,680 triangles),
vertices scaled radially by 1 + 0.15 * (8 random real spherical harmonics of
degree <= 6, seed 1), Poisson f = 1 with u = 0 on the surface, sites = the
64^3 cell centres of the bounding box inside the displaced sphere (kept when
|x| < r(x/|x|) (1 - 2e-4), which keeps them inside the inscribed mesh too),
4,096 walks per site, epsilon = 1e-4, max 1,024 steps.  Synthetic inputs,
generated here from seeds.

value    mixed form (FP32 query/position, FP64 accumulation) site-estimates/s,
         sites resident in HBM, scaled to the FP64 form's 95% CI half-width:
         rate * (h_mixed / h_fp64)^2, h = median over sites of 1.96 * SE.
e2e      the same metric through the host-buffer C-ABI call (twos_estimate):
         pinned host sites in, pinned host rows out, copies inside the timed
         region.
fp64     the plain all-FP64 GPU form at the same N (the target comparison);
         beside it the FP64 form given the mixed form's distance grid and
         entry nodes (fp64_with_grid: the precision change alone).
accuracy mixed against FP64 per site (z of the TD difference over every
         site), and on the unit ball (closed-form TD u^2 = ((1-|x|^2)/6)^2)
         the ratio of the mixed form's RMS error to the FP64 form's.
cpu_baseline  the reference's own compiled backend (wih_twos.cpp built
         unchanged against the project's Embree/Eigen shims, oracle/_ref),
         OpenMP over all host cores, on a fixed random subset of the sites.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--shard sites|replicas]

For N > 1 (torchrun) the sites are split into contiguous blocks of equal
predicted cost, one per rank, each keyed by its global site index (so the
gathered rows equal a one-GPU run's), and the rows are gathered once; time
= max over ranks.  --shard replicas runs the full workload on every rank
with its own seed instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "walking-into-holes_b200"))

METRIC = "TD site-estimates/s at equal 95% CI: mixed vs FP64 GPU, vs host CPU"
UNIT = "site-estimates/s"
WORKLOAD = ("noise-displaced icosphere L7 (327,680 tris, SH seed 1), Poisson f=1 u=0, 64^3 grid clipped to "
            "interior, 4096 walks/site, eps=1e-4")
L2_POLICY = "GPU arms: 256 MiB write between timed steps (L2 flush)"
# Canonical algorithmic bytes per closest-point query on this workload:
# 32 B per AABB test + 36 B per triangle test of the canonical binary SAH
# traversal, counted at the workload's own walk positions by
# `python oracle/canonical_bytes.py` (96 sites x 64 walks).
CANONICAL_BYTES_PER_QUERY = 38530.8  # 546.3 AABB + 584.7 triangle tests per query
CANONICAL_SOURCE = "oracle/canonical_bytes.py --sites 96 --walks 64"
SITE_MARGIN = 2e-4  # relative radial margin inside the displaced sphere (the mesh's chords lie within 4.5e-5)
REF_SUBSET = 1024   # fixed random subset of sites timed on the host cores
REF_SUBSET_SEED = 1234

# The walk kernel's counters from one `ncu --set full` capture of the medium
# case (the command and the rest of the metrics are in the profiles folder's
# summary of the walk kernel); they change only with the kernel.
NCU_WALK_KERNEL = {
    "case": "bench.py --walks 256 --grid 24 --steps 1 --warmup 1 --no-cpu --no-fp64 --no-ablation --no-accuracy "
            "--no-autotune",
    "lts__throughput_pct": 13.3,
    "smsp__thread_inst_executed_per_inst_executed": 7.90,
    "smsp__issue_active_pct": 70.3,
    "sm__warps_active_pct": 48.2,
    "lts__t_sector_hit_rate_pct": 73.6,
    "wavefront_split": {"step_kernel_threads_per_inst": 24.1, "query_kernel_threads_per_inst": 8.4,
                        "issue_active_pct": 38},
}


def dram_traffic_per_launch(walks: int) -> float:
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one walk-
    kernel launch, from one single-pass ncu capture of the full workload
    (default launch tuning): 691.7 GB read + 8.1 GB written for 502,403,072
    walks, 1,393 B per walk.  With the 2^28-vertex grid (4 GB of cell
    records, entry nodes included) the touched cells no longer fit the 126 MB
    L2: the reads are grid records; the writes are the per-walk samples.
    Scaled to the walks of the launch."""
    return 1392.83 * walks


EPSILON = 1e-4
MAX_STEPS = 1024
SEED = 20260912


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--shard", choices=["sites", "replicas"], default="sites",
                    help="N > 1: split the sites over the ranks (default) or run a full replica per rank")
    ap.add_argument("--walks", type=int, default=4096)
    ap.add_argument("--grid", type=int, default=64)
    ap.add_argument("--fp64-steps", type=int, default=1)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the unit-ball error-ratio leg")
    ap.add_argument("--no-autotune", action="store_true", help="keep the session's default launch tuning")
    ap.add_argument("--no-ablation", action="store_true",
                    help="skip the one-step mixed-form run with the distance grid off")
    ap.add_argument("--cpu-sites", type=int, default=0,
                    help="sites of the fixed subset timed on the host cores in this arm's cpu_baseline "
                         "(0: 8 per host thread, as one reference-arm step)")
    ap.add_argument("--ref-sites", type=int, default=REF_SUBSET,
                    help="--impl reference: sites of the fixed subset (split over the steps)")
    ap.add_argument("--housing-ref-sites", type=int, default=256, help="housing workload: FP64 reference sites")
    ap.add_argument("--workload", choices=["noise-sphere", "housing", "batch", "design", "unit-sphere"],
                    default="noise-sphere",
                    help="housing: the box-minus-cylinders epsilon sweep; batch: 32 uneven meshes in one launch; design: the graph-captured design loop; unit-sphere: the plain method's Neumann-cavity TD (separate JSON lines)")
    ap.add_argument("--sites", type=int, default=1_000_000, help="housing workload sites")
    return ap.parse_args(argv)


# ---------------------------------------------------------------- workload
def workload(grid_n):
    from twos_b200 import geometry
    V, F = geometry.noise_sphere(7, 1)
    grid = geometry.grid_points(V.min(0), V.max(0), grid_n)
    return V, F, grid


def workload_sites(grid):
    """Grid points inside the displaced sphere by the analytic radius with a
    relative margin: the same sites for every arm, inside the mesh as well."""
    from twos_b200 import geometry
    r = np.linalg.norm(grid, axis=1)
    keep = r > 1e-12
    g = grid[keep]
    rad = 1.0 + 0.15 * geometry.sh_field(g / r[keep][:, None], 1)
    return g[r[keep] < rad * (1.0 - SITE_MARGIN)]


def reference_subset(n: int, count: int) -> np.ndarray:
    """Indices of the fixed random subset of sites timed on the host cores."""
    rng = np.random.default_rng(REF_SUBSET_SEED)
    return np.sort(rng.choice(n, size=min(n, count), replace=False))


def source_terms():
    from twos_b200 import sources
    return sources.constant(1.0)


def workload_config(n_sites: int, walks: int) -> dict:
    """The workload keys both arms report identically."""
    return {"workload": WORKLOAD, "sites": int(n_sites), "walks": int(walks), "epsilon": EPSILON,
            "max_steps": MAX_STEPS, "mesh_triangles": 327680, "source": "f = 1, u = 0 on the surface",
            "l2": L2_POLICY}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------- ranks
def max_over_ranks(value: float, dist=None, device: str = "cpu") -> float:
    """Max of a per-rank time over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank: int) -> int:
    """In the replica mode each rank's copy of the workload draws an independent stream."""
    return SEED + rank


# ---------------------------------------------------------------- host CPU legs
def cpu_reference_leg(V, F, sites, walks, threads=None, workdir=None, repeat_tag=0):
    """Times the reference's own compiled backend (oracle/_ref/wih_twos, its
    `--mode twos` compliance path with f = 1 + 0 * (y + 0.5) = 1) on `sites`
    with every host thread: its own timed region (runtime_seconds_median of
    its summary: the site loop, not the mesh load or BVH build).  Falls back
    to the oracle port (the same algorithm and mt19937_64 stream) when the
    binary is missing.  Returns the rate and the per-site half-widths."""
    sys.path.insert(0, str(REPO / "oracle"))
    import ref_runner
    threads = threads or ref_runner.host_threads()
    if ref_runner.available():
        wd = Path(workdir) if workdir else Path(tempfile.mkdtemp(prefix="twos_ref_"))
        ply = wd / "mesh.ply"
        if not ply.exists():
            ref_runner.write_ply(ply, V, F)
        rows, summ, wall = ref_runner.run_compliance(ply, sites, walks=walks, seed=SEED + repeat_tag,
                                                     epsilon=EPSILON, max_steps=MAX_STEPS, slope=0.0,
                                                     threads=threads, repeats=1, workdir=wd)
        seconds = float(summ["runtime_seconds_median"])
        return {"sites": len(sites), "seconds": seconds, "wall": wall, "rate": len(sites) / seconds,
                "threads": int(summ["threads"]), "h": 1.96 * rows["score_se"], "kind": "reference",
                "engine": "reference wih_twos.cpp (unchanged) + project BVH shim in place of Embree 4",
                "queries_per_second": float(summ["distance_queries_per_second"]),
                "mean_steps": float(summ["mean_steps"])}
    import oracle
    oracle.build()
    om = oracle.OracleMesh(V, F)
    t = time.perf_counter()
    est = om.estimate(sites, walks=walks, seed=SEED + repeat_tag, epsilon=EPSILON, max_steps=MAX_STEPS,
                      source=[oracle.term(oracle.TERM_CONST, 1.0)], weight_order=0, threads=threads)
    dt = time.perf_counter() - t
    return {"sites": len(sites), "seconds": dt, "wall": dt, "rate": len(sites) / dt, "threads": threads,
            "h": 1.96 * est["score_se"], "kind": "port",
            "engine": "oracle restatement of wih_twos.cpp (reference algorithm + mt19937_64 stream)"}


def cpu_step_sites() -> int:
    """Sites of one host-CPU sample: 8 per host thread, so the reference's
    `schedule(dynamic, 4)` site loop (wih_twos.cpp:1825-1841) deals every
    thread two chunks and no thread idles for want of sites."""
    sys.path.insert(0, str(REPO / "oracle"))
    import ref_runner
    return 8 * ref_runner.host_threads()


def cpu_model() -> str:
    sys.path.insert(0, str(REPO / "oracle"))
    import ref_runner
    return ref_runner.cpu_model()


# ---------------------------------------------------------------- accuracy legs
def unit_ball_error_ratio(tb, walks: int, n_sites: int = 4096):
    """Compliance on the unit sphere (icosphere L7, f = 1, u = 0, eps 1e-4):
    the closed-form TD is u^2 = ((1 - |x|^2)/6)^2 (the reference's
    paper/sections/03_problem.tex:5).  RMS error of each form's estimate
    against it over n_sites sites uniform in r < 0.9, and their ratio
    (mixed / FP64).  The mixed form runs with its distance grid."""
    V, F = tb.geometry.icosphere(7)
    sites = tb.geometry.uniform_ball(n_sites, 0.9, seed=2)
    exact = ((1.0 - np.sum(sites ** 2, axis=1)) / 6.0) ** 2
    out = {"workload": f"unit sphere (icosphere L7), compliance f=1 u=0, {n_sites} sites in r<0.9 x {walks} walks, "
                       "eps 1e-4, exact TD ((1-|x|^2)/6)^2"}
    with tb.Mesh(V, F) as mesh:
        for prec in ("fp64", "mixed"):
            cfg = tb.Config(walks=walks, precision=prec, seed=SEED + 7, epsilon=EPSILON, max_steps=MAX_STEPS,
                            source=source_terms())
            rows, summ = mesh.estimate(sites, cfg)
            err = rows["score"] - exact
            z = err / rows["score_se"]
            out[prec] = {"rms_error": float(np.sqrt(np.mean(err ** 2))), "mean_error": float(np.mean(err)),
                         "median_abs_z": float(np.median(np.abs(z))),
                         "share_abs_z_below_3": float(np.mean(np.abs(z) < 3)),
                         "grid_steps_share": summ["grid_steps"] / max(1, summ["steps"])}
    out["error_ratio"] = out["mixed"]["rms_error"] / out["fp64"]["rms_error"]
    out["target"] = "<= 1.1"
    return out


def mixed_vs_fp64(rows_mixed, rows64):
    """Per-site z of the mixed form's TD against the FP64 form's over the
    same sites (independent samples: the grid changes the mixed radii)."""
    z = (rows_mixed["score"] - rows64["score"]) / np.hypot(rows_mixed["score_se"], rows64["score_se"])
    return {"sites": int(len(z)), "max_abs_z": float(np.max(np.abs(z))),
            "share_abs_z_below_3": float(np.mean(np.abs(z) < 3)), "mean_z": float(np.mean(z)),
            "median_abs_z": float(np.median(np.abs(z)))}


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import twos_b200 as tb
    from twos_b200 import shard

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    V, F, grid = workload(args.grid)
    sites_all = workload_sites(grid)
    n_all = len(sites_all)
    mesh = tb.Mesh(V, F, device=local)
    info = mesh.info()
    sharded = world > 1 and args.shard == "sites"
    if sharded:
        # Contiguous blocks of equal predicted cost; every rank computes the
        # same split from the same distances.
        d = mesh.closest_point(sites_all, precision="mixed", with_points=False)
        bounds = shard.partition(shard.site_cost(d, args.walks, EPSILON), world)
        lo, hi = int(bounds[rank]), int(bounds[rank + 1])
        seed = SEED
    else:
        bounds = np.array([0, n_all])
        lo, hi = 0, n_all
        seed = replica_seed(rank) if world > 1 else SEED
    sites = sites_all[lo:hi]
    n = len(sites)
    counts = np.diff(bounds) if sharded else [n]
    stream = torch.cuda.Stream()
    mesh.set_stream(stream)
    d_sites = torch.tensor(sites, dtype=torch.float64, device="cuda")
    d_out = torch.zeros((max(n, 1), 7), dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2
    base = dict(walks=args.walks, mode="compliance", seed=seed, epsilon=EPSILON, max_steps=MAX_STEPS,
                source=source_terms(), query_radius=4.0, site_offset=lo)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(cfg, steps, warmup, host=None):
        for w in range(warmup):
            cfg.repeat = 1000 + w
            if host is None:
                mesh.estimate_device(d_sites, n, d_out, cfg)
            else:
                mesh.estimate(host[0], cfg, out=host[1])
        ms, summs = [], []
        barrier()
        for k in range(steps):
            cfg.repeat = k
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if host is None:
                    summs.append(mesh.estimate_device(d_sites, n, d_out, cfg))
                else:
                    summs.append(mesh.estimate(host[0], cfg, out=host[1])[1])
                e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        barrier()
        total = max_over_ranks(sum(ms), dist, "cuda")
        return total, ms, summs

    def rows_now():
        local_rows = d_out[:n].cpu().numpy().copy().view(np.dtype(tb.SITE_DTYPE)).reshape(-1)
        return shard.gather_rows(local_rows, counts, dist, "cuda") if sharded else local_rows

    tuning = mesh.get_tuning()
    if not args.no_autotune:
        # The product's autotuner on a calibration subset, before any timing:
        # every rank tunes its own session the same way.
        from twos_b200.autotune import autotune
        tuning, _ = autotune(mesh, sites_all, tb.Config(precision="mixed", **dict(base, site_offset=0)),
                             calib_sites=4096, calib_walks=128, repeats=2, seed=rank, refine=8)
    clocks = ClockSampler(local)
    clocks.start()
    cfg_mixed = tb.Config(precision="mixed", **base)
    t_mixed, ms_mixed, s_mixed = timed(cfg_mixed, args.steps, args.warmup)
    clock_info = clocks.stop()
    rows_mixed = rows_now()
    h_mixed = float(np.median(1.96 * rows_mixed["score_se"]))

    # e2e: host-buffer entry point, pinned host memory, copies inside the timed region.
    h_sites = torch.from_numpy(np.ascontiguousarray(sites)).pin_memory()
    h_out = torch.zeros((n, 7), dtype=torch.float64).pin_memory()
    host = (h_sites.numpy(), h_out.numpy().view(np.dtype(tb.SITE_DTYPE)).reshape(-1))
    t_e2e, ms_e2e, s_e2e = timed(tb.Config(precision="mixed", **base), args.steps, 1, host=host)

    units = n_all if sharded else world * n_all
    fp64 = None
    rows64 = None
    if not args.no_fp64:
        t64, ms64, s64 = timed(tb.Config(precision="fp64", **base), args.fp64_steps, 1)
        rows64 = rows_now()
        h64 = float(np.median(1.96 * rows64["score_se"]))
        fp64 = {"rate": units * len(ms64) / (t64 / 1e3), "ms_per_step": t64 / len(ms64), "steps": len(ms64),
                "h_median": h64, "walk_seconds": float(np.mean([s["walk_seconds"] for s in s64]))}
    fp64_grid = None
    if fp64 is not None and not args.no_ablation:
        # The FP64 form with the mixed form's grid steps and entry nodes: the
        # like-for-like denominator of the precision change alone.
        mesh.set_tuning(**dict(tuning, grid_fp64=1))
        t_g, ms_g, s_g = timed(tb.Config(precision="fp64", **base), 1, 1)
        rows_g = rows_now()
        mesh.set_tuning(**tuning)
        fp64_grid = {"rate_unscaled": units / (t_g / 1e3), "ms_per_step": t_g,
                     "h_median": float(np.median(1.96 * rows_g["score_se"])),
                     "walk_seconds": s_g[0]["walk_seconds"],
                     "steps_per_walk": s_g[0]["steps"] / max(1, s_g[0]["paths"]),
                     "grid_steps_share": s_g[0]["grid_steps"] / max(1, s_g[0]["steps"])}
    no_grid = None
    if not args.no_ablation:
        mesh.set_tuning(**dict(tuning, grid_threshold=0))
        t_ng, ms_ng, s_ng = timed(tb.Config(precision="mixed", **base), 1, 1)
        rows_ng = rows_now()
        mesh.set_tuning(**tuning)
        no_grid = {"rate_unscaled": units / (t_ng / 1e3), "ms_per_step": t_ng,
                   "h_median": float(np.median(1.96 * rows_ng["score_se"])),
                   "walk_seconds": s_ng[0]["walk_seconds"],
                   "steps_per_walk": s_ng[0]["steps"] / max(1, s_ng[0]["paths"])}
    h_ref = fp64["h_median"] if fp64 else h_mixed
    if fp64_grid:
        fp64_grid["rate"] = fp64_grid["rate_unscaled"] * (fp64_grid["h_median"] / h_ref) ** 2
    if no_grid:
        no_grid["rate"] = no_grid["rate_unscaled"] * (no_grid["h_median"] / h_ref) ** 2
        if fp64:
            no_grid["over_fp64"] = no_grid["rate"] / fp64["rate"]
    scale = (h_mixed / h_ref) ** 2
    rate_mixed = units * args.steps / (t_mixed / 1e3)
    value = rate_mixed * scale
    rate_e2e = units * args.steps / (t_e2e / 1e3) * scale

    out = None
    if rank == 0:
        queries = np.mean([s["queries"] for s in s_mixed])
        grid_steps = np.mean([s["grid_steps"] for s in s_mixed])
        steps = np.mean([s["steps"] for s in s_mixed])
        walk_s = float(np.mean([s["walk_seconds"] for s in s_mixed]))
        nodes = np.mean([s["node_tests"] for s in s_mixed])
        planes = np.mean([s["plane_tests"] for s in s_mixed])
        tris = np.mean([s["triangle_tests"] for s in s_mixed])
        walks_launch = n * args.walks
        # Bytes the walk kernel must fetch: 96 B per node visit (two child
        # boxes + normal slabs + child words; 192 B for a four-wide node),
        # 32 B per triangle plane test
        # (plane slab + first vertex), 32 B more per full closest-point test
        # (the other two vertices), counted on the device; four 32 B sectors
        # per distance-grid lookup (the cell's eight corners lie in four
        # (i, j) rows; one lookup after every step).
        grid_lookups = steps if info["grid_dims"][0] else 0.0
        node_bytes = 192.0 if tuning.get("bvh_width", 2) == 4 else 96.0
        fetched = node_bytes * nodes + 32.0 * planes + 32.0 * tris + 32.0 * grid_lookups
        bvh_queries = queries - grid_steps
        hbm_peak, hbm_kind = measured_peaks()
        l2_peak = tb.l2_read_gbs(local)
        ach = fetched / walk_s / 1e9
        traffic = dram_traffic_per_launch(walks_launch)
        roof = {"bound": "l2", "achieved": ach, "peak": l2_peak, "unit": "GB/s", "frac": ach / l2_peak,
                "traffic": traffic,
                "peak_source": "measured in this run: twos_l2_read_gbs, 32-byte loads from every SM over a "
                               "64 MiB L2-resident buffer (the walk kernel's load form)",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one full-workload walk-kernel "
                                  "launch, 1,393 B per walk (grid records read from HBM, per-walk samples "
                                  "written), scaled to this launch's walks",
                "hbm": {"peak": hbm_peak, "peak_source": hbm_kind + " hbm_gbs",
                        "traffic_gbs": traffic / walk_s / 1e9, "frac": traffic / walk_s / 1e9 / hbm_peak},
                "ncu_walk_kernel": NCU_WALK_KERNEL,
                "bytes_per_walk": float(fetched / walks_launch),
                "bytes_definition": "device-counted: 96 B/node visit (192 B four-wide) + 32 B/plane test + 32 B/full "
                                    "triangle test + 32 B/distance-grid lookup (one 16-byte cell record, one sector; "
                                    "one per step)",
                "distance_evaluations_per_launch": float(queries), "grid_steps_per_launch": float(grid_steps),
                "bvh_queries_per_launch": float(bvh_queries), "walk_kernel_seconds": walk_s,
                "bvh_queries_per_second": float(bvh_queries / walk_s),
                "steps_per_walk": float(steps / walks_launch),
                "node_tests_per_bvh_query": float(nodes / bvh_queries),
                "plane_tests_per_bvh_query": float(planes / bvh_queries),
                "triangle_tests_per_bvh_query": float(tris / bvh_queries),
                "canonical": {"bytes_per_query": CANONICAL_BYTES_PER_QUERY, "source": CANONICAL_SOURCE,
                              "effective_gbs": CANONICAL_BYTES_PER_QUERY * bvh_queries / walk_s / 1e9,
                              "note": "bytes of a plain binary-SAH traversal per BVH query; this traversal "
                                      "fetches ~18x fewer and the grid skips most queries, so it is not a roof"}}
        accuracy = {}
        if rows64 is not None:
            accuracy["mixed_vs_fp64_z"] = mixed_vs_fp64(rows_mixed, rows64)
        if not args.no_accuracy and world == 1:
            accuracy["error_ratio_vs_oracle"] = unit_ball_error_ratio(tb, args.walks)
        cpu = None
        if not args.no_cpu and world == 1:
            idx = reference_subset(n_all, REF_SUBSET)[: args.cpu_sites or cpu_step_sites()]
            c = cpu_reference_leg(V, F, sites_all[idx], args.walks)
            h_cpu = float(np.median(c["h"]))
            h_gpu = float(np.median(1.96 * rows64["score_se"][idx])) if rows64 is not None else h_cpu
            cpu = {"value": c["rate"] * (h_cpu / h_gpu) ** 2, "unit": UNIT, "cores": c["threads"], "kind": c["kind"],
                   "cpu_model": cpu_model(), "rate_unscaled": c["rate"],
                   "sample": f"the first {c['sites']} sites of the fixed {REF_SUBSET}-site random subset (seed "
                             f"{REF_SUBSET_SEED}) x {args.walks} walks, {c['engine']}, OpenMP {c['threads']} threads, "
                             f"OMP_PROC_BIND=true, {c['seconds']:.1f} s in its timed site loop; scaled to the FP64 "
                             "GPU form's half-width on the same sites"}
        launches = int(sum(s["launches"] for s in s_mixed))
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_mixed / args.steps, "higher_is_better": True,
            "scaling": "strong" if sharded else "weak", "vs_baseline": None,
            "dtype": "f32 query/position, f64 accumulation", "data": "synthetic",
            "config": workload_config(n_all, args.walks),
            "parallelism": (f"sites sharded over {world} GPUs (contiguous equal-cost blocks, one row gather)"
                            if sharded else (f"replicas x{world}" if world > 1 else "1 GPU")),
            "implementation": {"bvh_nodes": int(info["bvh_nodes"]), "mixed_delta": info["mixed_delta"],
                               "distance_grid": {"dims": info["grid_dims"], "spacing": info["grid_spacing"],
                                                 "build_seconds_with_bvh": info["build_seconds"]},
                               "tuning": tuning},
            "ci": {"h_mixed_median": h_mixed, "h_fp64_median": h_ref, "scale": scale,
                   "rate_mixed_unscaled": rate_mixed},
            "fp64_form": fp64,
            "mixed_over_fp64": (value / fp64["rate"]) if fp64 else None,
            "mixed_without_grid": no_grid,
            "fp64_with_grid": fp64_grid,
            "mixed_over_fp64_with_grid": (value / fp64_grid["rate"]) if fp64_grid else None,
            "accuracy": accuracy,
            "e2e": {"value": rate_e2e, "unit": UNIT, "h2d_bytes_per_step": int(n * 24),
                    "d2h_bytes_per_step": int(n * 56), "ms_per_step": t_e2e / args.steps},
            "roofline": roof,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clock_info,
        }
        if cpu:
            out["gpu_over_cpu"] = value / cpu["value"]
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    mesh.close()
    return out


def run_reference(args):
    """The reference's own compiled backend on the host cores: wih_twos.cpp
    built unchanged (oracle/_ref/wih_twos, with the project's shim headers in
    place of Embree 4 and Eigen), OpenMP over every host thread with
    OMP_PROC_BIND=true, on the same workload and sites.  Each of the K timed
    steps is one process over the next 8-per-thread slice of the fixed
    --ref-sites random subset (cycling through it), timed by the reference's
    own site loop; warm-up steps run one thread's worth of sites each."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    V, F, grid = workload(args.grid)
    sites_all = workload_sites(grid)
    idx = reference_subset(len(sites_all), args.ref_sites)
    wd = Path(tempfile.mkdtemp(prefix="twos_ref_"))
    per = min(len(idx), cpu_step_sites())
    for w in range(args.warmup):
        cpu_reference_leg(V, F, sites_all[idx[:max(1, per // 8)]], args.walks, workdir=wd, repeat_tag=100 + w)
    runs = []
    for k in range(args.steps):
        take = np.take(idx, np.arange(k * per, (k + 1) * per), mode="wrap")
        runs.append(cpu_reference_leg(V, F, sites_all[take], args.walks, workdir=wd, repeat_tag=k))
    total_sites = sum(c["sites"] for c in runs)
    total_s = sum(c["seconds"] for c in runs)
    value = total_sites / total_s
    threads = runs[0]["threads"]
    h = np.concatenate([c["h"] for c in runs])
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / max(1, len(runs)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(len(sites_all), args.walks),
        "parallelism": f"OpenMP x{threads} host threads",
        "ci": {"h_median": float(np.median(h)),
               "scale": 1.0, "note": "the reference is the FP64 algorithm at the same N: its half-width is the "
                                     "FP64 GPU form's, so the equal-CI scale is 1"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": runs[0]["kind"],
                         "cpu_model": cpu_model(),
                         "sample": f"{total_sites} sites over {len(runs)} steps ({per} per step, cycling through the "
                                   f"fixed {len(idx)}-site random subset, seed {REF_SUBSET_SEED}, of the "
                                   f"{len(sites_all)} sites) x {args.walks} walks, "
                                   f"{runs[0]['engine']}, OMP_PROC_BIND=true; rate = sites / the reference's own "
                                   "timed site loop"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_housing_box(args):
    """Housing-like workload (not the headline line): box 4 x 2 x 1 minus 6
    through-cylinders of radius 0.15 (centres from seed 34), 529,608
    triangles; f = 1 on x0 < 1, adjoint q = 1_{x0 > 3} / |{x0 > 3}|; paired
    walks with a Green point per step; mixed form at eps in {1e-3, 1e-4,
    1e-5}: site-estimates/s over `--sites` sites x `--walks` walks, and the
    error of the cross-index TD against the FP64 form with 16x the walks on
    the first `--housing-ref-sites` sites (RMS error, and z = error / combined
    standard error), also with the distance grid off."""
    import torch
    import twos_b200 as tb
    from twos_b200 import geometry, sources
    V, F, centres = geometry.box_minus_cylinders(0.0115, 34)
    big = 1e30
    f = sources.box_indicator((-big, -big, -big), (1.0, big, big))
    vol = geometry.box_region_volume(centres, 0.15, 3.0, right=True)
    q = sources.box_indicator((3.0, -big, -big), (big, big, big), amp=1.0 / vol)
    sites = geometry.box_interior_points(args.sites, centres, 0.15, seed=35)
    mesh = tb.Mesh(V, F)
    n = len(sites)
    d_sites = torch.from_numpy(np.ascontiguousarray(sites)).cuda()
    d_out = torch.zeros((n, 7), dtype=torch.float64, device="cuda")
    rows = []
    for eps in (1e-3, 1e-4, 1e-5):
        base = dict(mode="paired", seed=SEED, epsilon=eps, max_steps=1 << 16, green=True, source=f, adjoint=q)
        cfg = tb.Config(walks=args.walks, precision="mixed", **base)
        mesh.estimate_device(d_sites, min(n, 16384), d_out, cfg)  # warm-up on a prefix
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        summ = mesh.estimate_device(d_sites, n, d_out, cfg)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        est = d_out.cpu().numpy().copy().view(np.dtype(tb.SITE_DTYPE)).reshape(-1)
        m = args.housing_ref_sites
        ref, _ = mesh.estimate(sites[:m], tb.Config(walks=16 * args.walks, precision="fp64", **dict(base, seed=SEED + 1)))
        # The same sites in the mixed form with the distance grid off: the
        # grid's share of the error, if any.
        mesh.set_tuning(grid_threshold=0)
        off, _ = mesh.estimate(sites[:m], cfg)
        mesh.set_tuning()

        def errors(e):
            err = e["score"] - ref["score"]
            comb = np.hypot(e["score_se"], ref["score_se"])
            ok = comb > 0  # sites where some walk pair saw both sources
            z = err[ok] / comb[ok]
            return float(np.sqrt(np.mean(err ** 2))), float(np.median(np.abs(z))), float(np.mean(np.abs(z) < 3))

        rms, zmed, z3 = errors(est[:m])
        rms_off, zmed_off, z3_off = errors(off)
        rows.append({"epsilon": eps, "site_estimates_per_s": n / dt, "seconds": dt,
                     "mean_steps_per_walk": summ["steps"] / summ["paths"],
                     "grid_steps_share": summ["grid_steps"] / max(1, summ["steps"]),
                     "td_rms_error_vs_fp64_16x": rms, "td_median_abs_z": zmed, "td_share_abs_z_below_3": z3,
                     "grid_off": {"td_rms_error_vs_fp64_16x": rms_off, "td_median_abs_z": zmed_off,
                                  "td_share_abs_z_below_3": z3_off},
                     "td_rms": float(np.sqrt(np.mean(ref["score"] ** 2)))})
    mesh.close()
    return {"workload": "housing-like box 4x2x1 minus 6 cylinders, 529,608 triangles, 1M sites", "triangles": int(len(F)),
            "sites": n, "walks": args.walks, "reference": f"FP64 form, {16 * args.walks} walks, {args.housing_ref_sites} sites",
            "dtype": "f32 query/position, f64 accumulation", "data": "synthetic", "per_epsilon": rows}


def run_batch(args):
    """Batched uneven workload (not the headline line): 32 noise-displaced
    icospheres (seeds 2-33, subdivision levels uniform in 3..7), site counts
    log-uniform in [100, 50000] (uniform in the ball r < 0.5, kept when
    inside), walks per site log-uniform in [256, 8192]; compliance, f = 1,
    eps = 1e-4, mixed form.  Times all 32 jobs in one persistent launch
    (twos_estimate_batch: one device work queue over every job) against one
    twos_estimate call per job, and reports the autotuner's pick for the
    largest job."""
    import torch  # noqa: F401  (initialises the device the library shares)
    import twos_b200 as tb
    from twos_b200 import autotune, geometry, sources
    rng = np.random.default_rng(3)
    meshes, sites, cfgs, info = [], [], [], []
    for j in range(32):
        level = int(rng.integers(3, 8))
        V, F = geometry.noise_sphere(level, 2 + j)
        m = tb.Mesh(V, F)
        n = int(round(np.exp(rng.uniform(np.log(100), np.log(50000)))))
        w = int(round(np.exp(rng.uniform(np.log(256), np.log(8192)))))
        pts = geometry.uniform_ball(2 * n, 0.5, seed=100 + j)
        pts = pts[m.inside(pts)][:n]
        meshes.append(m)
        sites.append(pts)
        cfgs.append(tb.Config(walks=w, precision="mixed", seed=SEED + j, epsilon=EPSILON, max_steps=MAX_STEPS,
                              source=sources.constant(1.0)))
        info.append({"level": level, "triangles": int(len(F)), "sites": int(len(pts)), "walks": w})
    total_sites = sum(len(s) for s in sites)
    total_walks = sum(len(s) * c.walks for s, c in zip(sites, cfgs))
    # Warm-ups of both paths, then three timed rounds of each, alternating;
    # the medians are reported.
    tb.estimate_batch(meshes, sites, cfgs)
    for m, s, c in zip(meshes, sites, cfgs):
        m.estimate(s, c)
    batch_times, seq_times = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        _, summ = tb.estimate_batch(meshes, sites, cfgs)
        batch_times.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        for m, s, c in zip(meshes, sites, cfgs):
            m.estimate(s, c)
        seq_times.append(time.perf_counter() - t0)
    t_batch = float(np.median(batch_times))
    t_seq = float(np.median(seq_times))
    big = int(np.argmax([len(s) * c.walks for s, c in zip(sites, cfgs)]))
    best, table = autotune.autotune(meshes[big], sites[big], cfgs[big], refine=4)
    n_ref = min(4, len(table) // 2)  # the refine stage's re-timings close the list
    for m in meshes:
        m.close()
    return {"workload": "32 uneven noise spheres (levels 3-7) in one launch", "jobs": info,
            "sites": total_sites, "walks": int(total_walks), "dtype": "f32 query/position, f64 accumulation",
            "data": "synthetic",
            "batched": {"seconds": t_batch, "site_estimates_per_s": total_sites / t_batch,
                        "walks_per_s": total_walks / t_batch, "launches": summ["launches"],
                        "rounds_seconds": batch_times},
            "one_call_per_job": {"seconds": t_seq, "site_estimates_per_s": total_sites / t_seq,
                                 "walks_per_s": total_walks / t_seq, "rounds_seconds": seq_times},
            "autotune_largest_job": {"pick": best,
                                     "sweep_seconds_per_walk": {json.dumps(t): s for t, s in table[:-n_ref]},
                                     "refined_seconds_per_walk": {json.dumps(t): s for t, s in table[-n_ref:]}}}


def run_design(args):
    """Design-loop workload (not the headline line): the design loop captured as
    a CUDA graph on the unit icosphere L4.  Each of 20
    iterations scouts 100,000 candidates (uniform in r < 0.85) with 2,048
    walks, takes the top 64, validates them with 4,096 fresh walks (stream
    1), takes the best lower bound score - 1.96 SE and inserts a ball cavity
    of radius 0.03 when it clears the threshold; compliance, f = 1, eps 1e-4.
    Reports iterations/s of the mixed and the FP64 form, whether their
    chosen candidates and accept decisions agree, and -- since the scout's
    distance grid lets the two forms choose different (near-tied)
    candidates -- whether the FP64 form, validating the mixed form's own
    choice with the same samples (the validation stage runs without the
    grid), reaches the same accept bit at every iteration."""
    import torch  # noqa: F401
    import twos_b200 as tb
    from twos_b200 import geometry, sources
    V, F = geometry.icosphere(4)
    cand = geometry.uniform_ball(100_000, 0.85, seed=5)
    kw = dict(iterations=20, shortlist=64, cavity_radius=0.03, z=1.96, accept_threshold=0.02,
              outer_clearance=0.02, pair_gap=0.01)
    out = {"workload": "design loop as a CUDA graph: 20 iterations on the unit icosphere L4, 100k candidates", "candidates": len(cand), **kw,
           "scout_walks": 2048, "validate_walks": 4096, "data": "synthetic"}
    hist = {}
    with tb.Mesh(V, F) as mesh:
        for prec in ("mixed", "fp64"):
            scout = tb.Config(walks=2048, precision=prec, seed=SEED, stream=0, epsilon=EPSILON, max_steps=MAX_STEPS,
                              source=sources.constant(1.0))
            val = tb.Config(walks=4096, precision=prec, seed=SEED, stream=1, epsilon=EPSILON, max_steps=MAX_STEPS,
                            source=sources.constant(1.0))
            mesh.design_loop(cand, scout, val, **dict(kw, iterations=1))  # warm-up and graph capture path
            t0 = time.perf_counter()
            h, cav, summ = mesh.design_loop(cand, scout, val, **kw)
            dt = time.perf_counter() - t0
            hist[prec] = h
            if prec == "mixed":
                cav_mixed = cav
            out[prec] = {"seconds": dt, "iterations_per_s": kw["iterations"] / dt, "accepted": int(h["accepted"].sum()),
                         "launches": summ["launches"]}
        # Replay each mixed-form validation in FP64 with the loop's keys:
        # stream 1, repeat = iteration, site index = the choice's shortlist
        # slot, the cavities present then.
        h, cav = hist["mixed"], cav_mixed
        same = []
        for it in range(kw["iterations"]):
            if h["chosen"][it] == 0xFFFFFFFF:
                continue
            val = tb.Config(walks=4096, precision="fp64", seed=SEED, stream=1, epsilon=EPSILON, max_steps=MAX_STEPS,
                            source=sources.constant(1.0), repeat=it, site_offset=int(h["slot"][it]),
                            cavity_radius=kw["cavity_radius"])
            c = cav[: int(h["n_cavities"][it])]
            r, _ = mesh.estimate(cand[int(h["chosen"][it])][None, :], val, cavities=c if len(c) else None)
            lower64 = float(r["score"][0] - kw["z"] * r["score_se"][0])
            same.append({"iteration": it, "lower_mixed": float(h["lower"][it]), "lower_fp64": lower64,
                         "accept_mixed": bool(h["accepted"][it]), "accept_fp64": bool(lower64 > kw["accept_threshold"])})
        out["accept_identical_given_chosen"] = all(s["accept_mixed"] == s["accept_fp64"] for s in same)
        out["accept_replay"] = same
    out["decisions_identical"] = bool(np.array_equal(hist["mixed"]["chosen"], hist["fp64"]["chosen"]) and
                                      np.array_equal(hist["mixed"]["accepted"], hist["fp64"]["accepted"]))
    for prec in ("mixed", "fp64"):
        out[f"chosen_{prec}"] = hist[prec]["chosen"].tolist()
        out[f"accepted_{prec}"] = hist[prec]["accepted"].tolist()
        out[f"lower_{prec}"] = hist[prec]["lower"].tolist()
    return out


def run_unit_sphere(args):
    """Plain-method workload (not the headline line): the unit sphere as an
    icosphere L4 (5,120 triangles), Dirichlet data g = x0^2 - x1^2 + 0.5 x2,
    adjoint source the mean over r < 0.5, 64 sites uniform in r < 0.9 (seed
    0), 1,024 paired walks per site with a Green point, eps = 1e-4, FP64 (the
    mixed form beside it).  The gradient form's cross-index product and the
    Neumann-cavity TD D_T = 3/2 grad u . grad p - q u against the analytic
    fields, GPU site-estimates/s through twos_estimate_gradient (host
    buffers), and the oracle's restatement of the same form on the host
    cores (counter stream, OpenMP) on the same 64 sites."""
    import twos_b200 as tb
    V, F = tb.geometry.icosphere(4)
    rng = np.random.default_rng(0)
    d = rng.normal(size=(64, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    sites = d * (0.9 * rng.random(64) ** (1 / 3))[:, None]
    boundary = tb.sources.quadratic((1.0, -1.0, 0.0)) + tb.sources.linear(0.5, 2)
    q = tb.sources.ball_mean_density((0.0, 0.0, 0.0), 0.5)
    x0, x1, x2 = sites.T
    g = x0 ** 2 - x1 ** 2 + 0.5 * x2
    grad_g = np.c_[2 * x0, -2 * x1, 0.5 * np.ones(len(sites))]
    r = np.linalg.norm(sites, axis=1)
    c = 1.0 / (4.0 / 3.0 * np.pi * 0.5 ** 3)
    grad_p = np.where(r[:, None] < 0.5, -c * sites / 3.0, -sites / (4.0 * np.pi * r[:, None] ** 3))
    qx = np.where(r < 0.5, c, 0.0)
    cross_exact = np.sum(grad_g * grad_p, axis=1)
    td_exact = 1.5 * cross_exact - qx * g
    base = dict(walks=1024, mode="paired", seed=SEED, epsilon=1e-4, max_steps=4096, green=True, source=[],
                adjoint=q, boundary=boundary)
    out = {"workload": "unit sphere (icosphere L4, 5,120 triangles), Neumann-cavity TD, 64 sites x 1,024 walks",
           "data": "synthetic", "steps": args.steps, "warmup": args.warmup}
    with tb.Mesh(V, F) as mesh:
        for prec in ("fp64", "mixed"):
            cfg = tb.Config(precision=prec, **base)
            for w in range(args.warmup):
                cfg.repeat = 1000 + w
                mesh.estimate_gradient(sites, cfg)
            times, ktimes = [], []
            for k in range(args.steps):
                cfg.repeat = k
                t0 = time.perf_counter()
                rows, summ = mesh.estimate_gradient(sites, cfg)
                times.append(time.perf_counter() - t0)
                ktimes.append(summ["kernel_seconds"])
            z = (rows["cross"] - cross_exact) / rows["cross_se"]
            td = 1.5 * rows["cross"] - qx * rows["u"]
            # The TD's standard error bounded by the parts' (|cov| <= sd sd).
            zt = (td - td_exact) / (1.5 * rows["cross_se"] + np.abs(qx) * rows["u_se"])
            out[prec] = {"site_estimates_per_s": len(sites) / float(np.median(times)),
                         "seconds": float(np.median(times)), "kernel_seconds": float(np.median(ktimes)),
                         "steps_per_walk": summ["steps"] / summ["paths"], "grid_steps": summ["grid_steps"],
                         "cross_max_abs_z": float(np.max(np.abs(z))), "cross_share_abs_z_below_3":
                         float(np.mean(np.abs(z) < 3)), "cross_mean_z": float(np.mean(z)),
                         "u_mean_abs_error": float(np.mean(np.abs(rows["u"] - g))),
                         "td_rms_error": float(np.sqrt(np.mean((td - td_exact) ** 2))),
                         "td_rms": float(np.sqrt(np.mean(td_exact ** 2))),
                         "td_max_abs_z": float(np.max(np.abs(zt))), "td_share_abs_z_below_3":
                         float(np.mean(np.abs(zt) < 3)), "td_rms_z": float(np.sqrt(np.mean(zt ** 2)))}
    if not args.no_cpu:
        sys.path.insert(0, str(REPO / "oracle"))
        import oracle
        oracle.build()
        threads = oracle.default_threads()
        om = oracle.OracleMesh(V, F)

        def terms(ts):
            return [oracle.term(t.kind, t.amp, t.axis, t.offset, t.div, tuple(t.c), tuple(t.w)) for t in ts]

        sub = sites
        t0 = time.perf_counter()
        om.estimate_gradient(sub, rng=oracle.RNG_COUNTER, mode=1, walks=1024, seed=SEED, epsilon=1e-4,
                             max_steps=4096, green=True, source=[], adjoint=terms(q), boundary=terms(boundary),
                             threads=threads)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": len(sub) / dt, "unit": UNIT, "cores": threads, "kind": "port",
                               "sample": f"{len(sub)} sites x 1024 walks, oracle restatement of the gradient "
                                         f"form (counter stream), OpenMP {threads} threads, {dt:.1f} s"}
        out["fp64_over_cpu"] = out["fp64"]["site_estimates_per_s"] / out["cpu_baseline"]["value"]
    out["mixed_over_fp64"] = out["mixed"]["site_estimates_per_s"] / out["fp64"]["site_estimates_per_s"]
    out["td_error_ratio_mixed_over_fp64"] = out["mixed"]["td_rms_error"] / out["fp64"]["td_rms_error"]
    out["td_formula_check"] = ("D_T = 3/2 grad u . grad p - q u - f p, exact on a finite Neumann hole "
                               "(tests/test_neumann_hole_cpu.py)")
    return out


def main(argv=None):
    args = parse_args(argv)
    if args.workload == "design":
        print(json.dumps(run_design(args)), flush=True)
        return
    if args.workload == "housing":
        print(json.dumps(run_housing_box(args)), flush=True)
        return
    if args.workload == "batch":
        print(json.dumps(run_batch(args)), flush=True)
        return
    if args.workload == "unit-sphere":
        print(json.dumps(run_unit_sphere(args)), flush=True)
        return
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
