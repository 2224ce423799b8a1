"""Python face of libtwos.so: a mesh session and its estimator calls.

``Mesh`` owns a twos_mesh session (BVH resident on one GPU).  Its methods are
thin wrappers over the C ABI with numpy buffers:

* ``estimate``      per-site (u, p, score, score_se, same_index, steps, caps)
                    -- evaluate_site / paired_site of the reference
                    (benchmarks/compiled_bunny/src/wih_twos.cpp:674-717,
                    benchmarks/distinct_adjoint/adjoint.cpp:18-42);
* ``estimate_device`` the same with device-resident sites and results (torch
                    tensors or raw pointers);
* ``walk_samples``  per-walk u, p and steps;
* ``diffwos``       derivatives of u with respect to cavity centres and radii
                    (evaluate_differential_site, wih_twos.cpp:839-928);
* ``closest_point`` batched distance/closest point (wih_twos.cpp:339-359);
* ``inside``        ray-parity membership (wih_twos.cpp:361-394);
* ``topk_device``   top-k site indices.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _abi, sources
from ._abi import (DIFF_DTYPE, DIFF_STATS_DTYPE, MODE_COMPLIANCE, MODE_HOT, MODE_PAIRED, OK, PREC_FP64, PREC_MIXED,
                   Request, SITE_DTYPE, Summary, TwosError, check)

PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED}
MODES = {"compliance": MODE_COMPLIANCE, "paired": MODE_PAIRED, "hot": MODE_HOT}
SOURCE_MODES = {"center": _abi.SOURCE_CENTER, "green": _abi.SOURCE_GREEN, "exact": _abi.SOURCE_EXACT}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Config:
    """One estimation request (the reference's Options, wih_twos.cpp:73-101)."""
    walks: int = 16
    mode: str = "compliance"
    precision: str = "mixed"
    max_steps: int = 512
    seed: int = 20260912
    repeat: int = 0
    stream: int = 0
    epsilon: float = 5e-4
    cavity_radius: float = 0.0
    query_radius: float = 4.0
    green: bool | int | str = False  # False/"center", True/"green", or "exact" (TWOS_SOURCE_*)
    source: list = field(default_factory=lambda: sources.affine())
    adjoint: list = field(default_factory=list)
    skip_cavity_sites: bool | None = None
    site_offset: int = 0
    boundary: list = field(default_factory=list)  # Dirichlet data of u (gradient form)

    def to_request(self) -> Request:
        r = Request()
        r.mode = MODES[self.mode] if isinstance(self.mode, str) else int(self.mode)
        r.precision = PRECISIONS[self.precision] if isinstance(self.precision, str) else int(self.precision)
        r.walks = int(self.walks)
        r.max_steps = int(self.max_steps)
        r.seed = int(self.seed)
        r.repeat = int(self.repeat)
        r.stream = int(self.stream)
        r.epsilon = float(self.epsilon)
        r.cavity_radius = float(self.cavity_radius)
        r.query_radius = float(self.query_radius) if self.query_radius is not None else 0.0
        r.green = SOURCE_MODES[self.green] if isinstance(self.green, str) else int(self.green)
        if len(self.source) > _abi.MAX_TERMS or len(self.adjoint) > _abi.MAX_TERMS:
            raise ValueError("too many source terms")
        r.n_source, r.n_adjoint = len(self.source), len(self.adjoint)
        for i, t in enumerate(self.source):
            r.source[i] = t
        for i, t in enumerate(self.adjoint):
            r.adjoint[i] = t
        skip = self.skip_cavity_sites
        if skip is None:
            skip = r.mode != MODE_COMPLIANCE
        r.skip_cavity_sites = int(bool(skip))
        r.site_offset = int(self.site_offset)
        if len(self.boundary) > _abi.MAX_TERMS:
            raise ValueError("too many boundary terms")
        r.n_boundary = len(self.boundary)
        for i, t in enumerate(self.boundary):
            r.boundary[i] = t
        return r


def _summary_dict(s: Summary) -> dict:
    return {k: getattr(s, k) for k, _ in Summary._fields_}


class Mesh:
    """A triangle mesh resident on one GPU, with its BVH (FP32 and FP64)."""

    def __init__(self, vertices=None, faces=None, *, ply: str | None = None, device: int = 0):
        L = _abi.load()
        h = ctypes.c_void_p()
        if ply is not None:
            check(L.twos_mesh_open_ply(str(ply).encode(), device, ctypes.byref(h)))
        else:
            v = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
            f = np.ascontiguousarray(faces, dtype=np.uint32).reshape(-1, 3)
            check(L.twos_mesh_open(_ptr(v), len(v), _ptr(f), len(f), device, ctypes.byref(h)))
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            _abi.load().twos_mesh_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream=None):
        """Run the session's work on `stream` (torch.cuda.Stream, a raw handle, or None for its own)."""
        handle = getattr(stream, "cuda_stream", stream)
        check(_abi.load().twos_mesh_set_stream(self._h, ctypes.c_void_p(handle or 0)))

    def set_tuning(self, block=128, refill=1, step_threshold=1, blocks_per_sm=0, grid_threshold=0.1, units=8,
                   entry=1, grid_fp64=0, bvh_width=2, lane_walks=1, wavefront=0):
        """Walk-kernel launch tuning; grid_threshold is the mixed form's
        distance-grid bound (in grid spacings) above which a step skips its
        closest-point query, 0 to query every step; units is the number of
        traversal units a lane runs per warp-loop iteration; entry 1 starts
        qualifying mixed-form queries at the entry-node table's node;
        grid_fp64 1 gives the FP64 compliance form the grid and entry nodes
        too (a like-for-like comparison of precision); bvh_width 2 or 4 picks
        the mixed form's binary or four-wide BVH traversal; lane_walks is the
        number of walks a lane claims from the work queue at once; wavefront
        > 0 runs the mixed centre-source modes in the wavefront form with that
        many walks in flight (a multiple of 256)."""
        t = _abi.Tuning(int(block), int(refill), int(step_threshold), int(blocks_per_sm), float(grid_threshold),
                        int(units), int(entry), int(grid_fp64), int(bvh_width), int(lane_walks), int(wavefront))
        check(_abi.load().twos_mesh_set_tuning(self._h, ctypes.byref(t)))

    def get_tuning(self) -> dict:
        t = _abi.Tuning()
        check(_abi.load().twos_mesh_get_tuning(self._h, ctypes.byref(t)))
        return {"block": t.block, "refill": t.refill, "step_threshold": t.step_threshold,
                "blocks_per_sm": t.blocks_per_sm,
                # The ABI keeps a float; report the shortest decimal that rounds to it (0.1, not 0.10000000149).
                "grid_threshold": float(str(np.float32(t.grid_threshold))), "units": t.units,
                "entry": t.entry, "grid_fp64": t.grid_fp64, "bvh_width": t.bvh_width,
                "lane_walks": t.lane_walks, "wavefront": t.wavefront}

    def info(self) -> dict:
        i = _abi.MeshInfo()
        check(_abi.load().twos_mesh_get_info(self._h, ctypes.byref(i)))
        return {"vertices": i.vertices, "faces": i.faces, "bvh_nodes": i.bvh_nodes, "bvh_depth": i.bvh_depth,
                "device": i.device, "bounds_min": list(i.bounds_min), "bounds_max": list(i.bounds_max),
                "center": list(i.center), "mixed_delta": i.mixed_delta, "build_seconds": i.build_seconds,
                "device_bytes": i.device_bytes, "grid_dims": list(i.grid_dims), "grid_spacing": i.grid_spacing}

    # ------------------------------------------------------------------ queries
    def closest_point(self, points, precision="fp64", query_radius=0.0, with_points=True):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        n = len(pts)
        dist = np.empty(n)
        closest = np.empty((n, 3)) if with_points else None
        check(_abi.load().twos_closest_point(self._h, PRECISIONS[precision], _ptr(pts), n, float(query_radius),
                                             _ptr(dist), _ptr(closest)))
        return (dist, closest) if with_points else dist

    def distance_bound(self, points):
        """The mixed form's distance-grid lower bound at each point
        (twos_mesh_distance_bound); NaN outside the grid."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.empty(len(pts))
        check(_abi.load().twos_mesh_distance_bound(self._h, _ptr(pts), len(pts), _ptr(out)))
        return out

    def inside(self, points):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(len(pts), dtype=np.uint8)
        check(_abi.load().twos_inside(self._h, _ptr(pts), len(pts), _ptr(out)))
        return out.astype(bool)

    # ------------------------------------------------------------------ estimator
    def estimate(self, sites, config: Config, cavities=None, raise_on_caps=True, out=None):
        """Per-site estimates (structured array with SITE_DTYPE fields) and the call summary.

        `out` may be a preallocated SITE_DTYPE array (e.g. a view of pinned memory)."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        if out is None:
            out = np.zeros(len(s), dtype=SITE_DTYPE)
        elif out.dtype != np.dtype(SITE_DTYPE) or len(out) != len(s) or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous SITE_DTYPE array with one row per site")
        req = config.to_request()
        summ = Summary()
        rc = _abi.load().twos_estimate(self._h, ctypes.byref(req), _ptr(s), len(s), _ptr(cav), len(cav), _ptr(out),
                                       ctypes.byref(summ))
        if rc != _abi.OK and not (not raise_on_caps and summ.error_flags == 0 and summ.caps > 0):
            check(rc)
        return out, _summary_dict(summ)

    def estimate_device(self, d_sites, n_sites, d_out, config: Config, cavities=None):
        """Device-resident sites (n x 3 float64) and rows (n x 56 bytes); pointers or torch tensors."""
        def addr(x):
            return x.data_ptr() if hasattr(x, "data_ptr") else int(x)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        req = config.to_request()
        summ = Summary()
        check(_abi.load().twos_estimate_device(self._h, ctypes.byref(req), ctypes.c_void_p(addr(d_sites)),
                                               int(n_sites), _ptr(cav), len(cav), ctypes.c_void_p(addr(d_out)),
                                               ctypes.byref(summ)))
        return _summary_dict(summ)

    def design_loop(self, candidates, scout: Config, validate: Config, iterations=20, shortlist=64,
                    cavity_radius=0.03, z=1.96, accept_threshold=0.0, outer_clearance=0.0, pair_gap=0.0,
                    cavities=None, use_graph=True):
        """Scout -> top-k -> fresh validation -> lower-bound argmax -> accept/insert, on the
        device (twos_design_loop).  Returns (history, cavities, summary)."""
        cand = np.ascontiguousarray(candidates, dtype=np.float64).reshape(-1, 3)
        cav0 = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        P = _abi.DesignParams()
        P.iterations, P.shortlist = int(iterations), int(shortlist)
        P.cavity_radius, P.z, P.accept_threshold = float(cavity_radius), float(z), float(accept_threshold)
        P.outer_clearance, P.pair_gap, P.use_graph = float(outer_clearance), float(pair_gap), int(bool(use_graph))
        hist = np.zeros(int(iterations), dtype=_abi.DESIGN_DTYPE)
        cav_out = np.zeros((len(cav0) + int(iterations), 3))
        n_out = ctypes.c_uint32()
        rs, rv = scout.to_request(), validate.to_request()
        summ = Summary()
        check(_abi.load().twos_design_loop(self._h, ctypes.byref(rs), ctypes.byref(rv), _ptr(cand), len(cand),
                                           _ptr(cav0) if len(cav0) else None, len(cav0), ctypes.byref(P),
                                           _ptr(hist), _ptr(cav_out), ctypes.byref(n_out), ctypes.byref(summ)))
        return hist, cav_out[: n_out.value].copy(), _summary_dict(summ)

    def walk_samples(self, sites, config: Config, cavities=None):
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        n, w = len(s), int(config.walks)
        u = np.empty((n, w))
        p = np.empty((n, w))
        st = np.empty((n, w), dtype=np.uint32)
        req = config.to_request()
        check(_abi.load().twos_walk_samples(self._h, ctypes.byref(req), _ptr(s), n, _ptr(cav), len(cav), _ptr(u),
                                            _ptr(p), _ptr(st)))
        return {"u": u, "p": p, "steps": st & 0x7FFFFFFF, "caps": (st >> 31).astype(bool)}

    def trace_grid_steps(self, sites, config: Config, capacity: int = 1 << 22):
        """Every grid step of a mixed compliance estimate (twos_trace_grid_steps):
        (points [k][3] in original coordinates, bounds [k], total grid steps)."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        pts = np.zeros((capacity, 3))
        bnd = np.zeros(capacity)
        cnt = ctypes.c_uint64()
        req = config.to_request()
        check(_abi.load().twos_trace_grid_steps(self._h, ctypes.byref(req), _ptr(s), len(s), int(capacity), _ptr(pts),
                                                _ptr(bnd), ctypes.byref(cnt)))
        k = min(int(cnt.value), capacity)
        return pts[:k], bnd[:k], int(cnt.value)

    def finalize_samples(self, u, p=None, steps=None, mode: str = "compliance", precision: str = "fp64"):
        """The device's per-site reduction (twos_finalize_samples) of given
        per-walk samples u, p [n_sites, walks]: rows of SITE_DTYPE, as
        twos_estimate writes them for walks with these payoffs."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.ndim != 2:
            raise ValueError("u must be [n_sites, walks]")
        n, w = u.shape
        pp = None if p is None else np.ascontiguousarray(p, dtype=np.float64).reshape(n, w)
        st = None if steps is None else np.ascontiguousarray(steps, dtype=np.uint32).reshape(n, w)
        out = np.zeros(n, dtype=SITE_DTYPE)
        check(_abi.load().twos_finalize_samples(self._h, PRECISIONS[precision], MODES[mode], _ptr(u), _ptr(pp),
                                                _ptr(st), n, w, _ptr(out)))
        return out

    def diffwos(self, sites, config: Config, cavities, diff_offset: float = 0.02,
                enclosure_fallback: bool = False, strict: bool = True):
        """Differential WoS (twos_diffwos): returns (rows [n_sites, n_cav] of
        DIFF_DTYPE, stats [n_sites] of DIFF_STATS_DTYPE, summary).  With
        strict=False a capped walk or an unsafe offset is reported in
        summary["error"] instead of raised, as the study backend's error
        return carries the rows along (study.cpp:309-310)."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        rows = np.zeros((len(s), len(cav)), dtype=DIFF_DTYPE)
        stats = np.zeros(len(s), dtype=DIFF_STATS_DTYPE)
        req = config.to_request()
        summ = Summary()
        L = _abi.load()
        rc = L.twos_diffwos(self._h, ctypes.byref(req), float(diff_offset), int(bool(enclosure_fallback)), _ptr(s),
                            len(s), _ptr(cav), len(cav), _ptr(rows), _ptr(stats), ctypes.byref(summ))
        out = _summary_dict(summ)
        out["parity_rays"] = out.pop("node_tests")
        out["enclosure_fallbacks"] = out.pop("plane_tests")
        out["unsafe_offsets"] = out.pop("triangle_tests")
        out["error"] = None
        if rc != OK:
            msg = L.twos_last_error().decode(errors="replace")
            if strict or not msg.startswith("unsafe differential path"):
                raise TwosError(rc, msg)
            out["error"] = msg
        return rows, stats, out

    def rqmc(self, sites, config: Config, u_boundary, p_boundary, method: str = "array", batches: int = 4,
             record: bool = False):
        """Array-RQMC, matched MC, neighbour reuse or Sobol-over-steps RQMC
        (twos_rqmc; the methods 'array', 'mc', 'neighbors' and 'rqmc' (here
        also 'sobol') of sampling.py:118-132): returns
        (batch_u, batch_p [batches, n_sites], td [n_sites], summary), td the
        batch cross-fit -(sum a sum b - sum ab)/(R(R-1)) of sampling.py:90-92.
        With record=True the summary also holds the per-walk record:
        walk_first [batches, n_sites, walks, 3], walk_u / walk_p
        [batches, n_sites, walks] and site_radius [n_sites]."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        p = _abi.RqmcParams()
        p.method = {"mc": _abi.RQMC_MC, "array": _abi.RQMC_ARRAY, "neighbors": _abi.RQMC_NEIGHBOUR,
                    "neighbours": _abi.RQMC_NEIGHBOUR, "rqmc": _abi.RQMC_SOBOL, "sobol": _abi.RQMC_SOBOL}[method]
        p.batches = int(batches)
        p.n_u_boundary, p.n_p_boundary = len(u_boundary), len(p_boundary)
        for i, t in enumerate(u_boundary):
            p.u_boundary[i] = t
        for i, t in enumerate(p_boundary):
            p.p_boundary[i] = t
        bu = np.zeros((batches, len(s)))
        bp = np.zeros((batches, len(s)))
        td = np.zeros(len(s))
        rec = None
        if record:
            w = int(config.walks)
            rec = {"walk_first": np.zeros((batches, len(s), w, 3)), "walk_u": np.zeros((batches, len(s), w)),
                   "walk_p": np.zeros((batches, len(s), w)), "site_radius": np.zeros(len(s))}
            for k, v in rec.items():
                setattr(p, k, v.ctypes.data)
        req = config.to_request()
        summ = Summary()
        check(_abi.load().twos_rqmc(self._h, ctypes.byref(req), ctypes.byref(p), _ptr(s), len(s), _ptr(bu), _ptr(bp),
                                    _ptr(td), ctypes.byref(summ)))
        out = _summary_dict(summ)
        if rec is not None:
            out.update(rec)
        return bu, bp, td, out

    def estimate_gradient(self, sites, config: Config, cavities=None):
        """Gradient samples and the cross-index gradient product
        (twos_estimate_gradient): rows of GRADIENT_DTYPE and the summary.
        config must be paired; config.boundary holds the primal's Dirichlet
        data on the mesh."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        rows = np.zeros(len(s), dtype=_abi.GRADIENT_DTYPE)
        req = config.to_request()
        summ = Summary()
        check(_abi.load().twos_estimate_gradient(self._h, ctypes.byref(req), _ptr(s), len(s),
                                                 _ptr(cav) if len(cav) else None, len(cav), _ptr(rows),
                                                 ctypes.byref(summ)))
        return rows, _summary_dict(summ)

    def validate(self, sites, config: Config, cavities=None, radius_cap: float = 0.1, value_cap: float = 0.1,
                 strict: bool = True):
        """Certified fresh-sample validation (twos_validate; run_minimum_benefit,
        minimum_benefit.hpp:145-188).  Returns (samples [n_sites, walks] of
        CERT_SAMPLE_DTYPE, stages [n_sites, n_stages] of VALIDATE_STAGE_DTYPE,
        summary).  With strict=False a containment failure is reported in
        summary["error"] with the samples, instead of raised."""
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        n, w = len(s), int(config.walks)
        samples = np.zeros((n, w), dtype=_abi.CERT_SAMPLE_DTYPE)
        stages = np.zeros((n, _abi.VALIDATE_MAX_STAGES), dtype=_abi.VALIDATE_STAGE_DTYPE)
        n_stages = ctypes.c_uint32(0)
        req = config.to_request()
        params = _abi.ValidateParams(float(radius_cap), float(value_cap))
        summ = Summary()
        L = _abi.load()
        rc = L.twos_validate(self._h, ctypes.byref(req), ctypes.byref(params), _ptr(s), n,
                             _ptr(cav) if len(cav) else None, len(cav), _ptr(samples), _ptr(stages),
                             ctypes.byref(n_stages), ctypes.byref(summ))
        out = _summary_dict(summ)
        out["containment_failures"] = out.pop("node_tests")
        out["error"] = None
        if rc != OK:
            msg = L.twos_last_error().decode(errors="replace")
            if strict or "containment" not in msg:
                raise TwosError(rc, msg)
            out["error"] = msg
        return samples, stages[:, : n_stages.value].copy(), out

    def topk_device(self, d_keys, n, k, d_index):
        def addr(x):
            return x.data_ptr() if hasattr(x, "data_ptr") else int(x)
        check(_abi.load().twos_topk_device(self._h, ctypes.c_void_p(addr(d_keys)), int(n), int(k),
                                           ctypes.c_void_p(addr(d_index))))


def ball_green_integral(cases, device: int = 0):
    """The EXACT source's closed-form ball integral evaluated on the GPU
    (twos_ball_green_integral; exact_bump_green, study.cpp:64-77): cases is
    an [n, 4] array of (d, r, R, A); returns the n integrals."""
    c = np.ascontiguousarray(cases, dtype=np.float64).reshape(-1, 4)
    out = np.zeros(len(c))
    check(_abi.load().twos_ball_green_integral(_ptr(c), len(c), _ptr(out), int(device)))
    return out


def l2_read_gbs(device: int = 0, mib: int = 64, passes: int = 20) -> float:
    """Measured L2 read bandwidth of the device in GB/s (twos_l2_read_gbs):
    32-byte vector loads over an L2-resident buffer of `mib` MiB."""
    g = ctypes.c_double()
    check(_abi.load().twos_l2_read_gbs(int(device), int(mib) << 20, int(passes), ctypes.byref(g)))
    return float(g.value)


def sobol_directions(dims: int, bits: int = 10) -> np.ndarray:
    """The Sobol' direction numbers of the 'sobol' RQMC method
    (twos_sobol_directions, host only): [dims, bits] uint32, most significant
    digit first."""
    out = np.zeros((int(dims), int(bits)), dtype=np.uint32)
    check(_abi.load().twos_sobol_directions(int(dims), int(bits), out.ctypes.data))
    return out


def estimate_batch(meshes, sites_list, configs, cavities_list=None):
    """Several (mesh, sites, config) jobs in one persistent launch
    (twos_estimate_batch).  Returns one SITE_DTYPE array per job and the
    batch summary."""
    n = len(meshes)
    if not (len(sites_list) == len(configs) == n):
        raise ValueError("meshes, sites_list and configs must have the same length")
    cavities_list = cavities_list or [None] * n
    sites = [np.ascontiguousarray(s, dtype=np.float64).reshape(-1, 3) for s in sites_list]
    cavs = [np.zeros((0, 3)) if c is None else np.ascontiguousarray(c, dtype=np.float64).reshape(-1, 3)
            for c in cavities_list]
    outs = [np.zeros(len(s), dtype=SITE_DTYPE) for s in sites]
    reqs = (Request * n)(*[c.to_request() for c in configs])
    vp = ctypes.c_void_p
    mesh_arr = (vp * n)(*[m._h.value for m in meshes])
    site_arr = (vp * n)(*[s.ctypes.data for s in sites])
    nsite_arr = (ctypes.c_uint32 * n)(*[len(s) for s in sites])
    cav_arr = (vp * n)(*[c.ctypes.data if len(c) else None for c in cavs])
    ncav_arr = (ctypes.c_uint32 * n)(*[len(c) for c in cavs])
    out_arr = (vp * n)(*[o.ctypes.data for o in outs])
    summ = Summary()
    check(_abi.load().twos_estimate_batch(mesh_arr, reqs, n, site_arr, nsite_arr, cav_arr, ncav_arr, out_arr,
                                          ctypes.byref(summ)))
    return outs, _summary_dict(summ)

