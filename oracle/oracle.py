"""TEST INFRASTRUCTURE ONLY -- Python side of the CPU oracle.

The oracle restates the reference TWoS backend on the host so the CUDA product
can be checked against it.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this module; the product never does.

Contents
--------
* ctypes bindings to ``oracle/_build/libtwos_oracle.so`` (``twos_oracle.cpp``):
  FP64 closest point (BVH or brute force, with box/triangle test counts),
  per-walk samples and per-site estimates in the reference's own
  ``mt19937_64`` stream or in the GPU's counter stream.
* numpy restatements of the reference's readers and statistics:
  ``load_ascii_ply`` (benchmarks/compiled_bunny/src/wih_twos.cpp:437-493),
  ``read_points`` (wih_twos.cpp:508-522), ``crossfit_square``
  (benchmarks/stanford_bunny/run_bunny_benchmark.py:257-269),
  ``crossfit_product`` (experiments/run_controlled_experiments.py:79-87) and
  the shortlist/rescore selection rule (run_bunny_benchmark.py:302-337).
"""
from __future__ import annotations

import ctypes
import gzip
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libtwos_oracle.so"

MODE_COMPLIANCE, MODE_PAIRED, MODE_HOT = 0, 1, 2
RNG_REFERENCE, RNG_COUNTER = 0, 1
TERM_CONST, TERM_LINEAR, TERM_GAUSS, TERM_BUMP, TERM_BOX, TERM_BALL = range(6)


class Term(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("axis", ctypes.c_int32),
        ("amp", ctypes.c_double), ("offset", ctypes.c_double), ("div", ctypes.c_double),
        ("c", ctypes.c_double * 3), ("w", ctypes.c_double * 3),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("rng", ctypes.c_int32),
        ("walks", ctypes.c_int32), ("max_steps", ctypes.c_int32),
        ("seed", ctypes.c_uint64), ("repeat", ctypes.c_uint32), ("stream", ctypes.c_uint32),
        ("epsilon", ctypes.c_double), ("cavity_radius", ctypes.c_double),
        ("query_radius", ctypes.c_double),
        ("green", ctypes.c_int32), ("n_source", ctypes.c_int32), ("n_adjoint", ctypes.c_int32),
        ("skip_cavity_sites", ctypes.c_int32), ("weight_order", ctypes.c_int32),
        ("threads", ctypes.c_int32),
        ("source", Term * 8), ("adjoint", Term * 8),
        ("n_boundary", ctypes.c_int32), ("pad", ctypes.c_int32), ("boundary", Term * 8),
    ]


class Site(ctypes.Structure):
    _fields_ = [
        ("u", ctypes.c_double), ("p", ctypes.c_double), ("score", ctypes.c_double),
        ("score_se", ctypes.c_double), ("same_index", ctypes.c_double),
        ("steps", ctypes.c_uint64), ("caps", ctypes.c_uint64),
    ]


REFERENCE = Path("/root/reference")


def build() -> Path:
    """Compile the oracle with its Makefile (system g++, no FMA contraction),
    and, where the reference's source tree is present, the reference's own
    backend against the shim headers (oracle/_ref/wih_twos; elsewhere the
    prebuilt binary is used as it is)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    if (REFERENCE / "benchmarks/compiled_bunny/src/wih_twos.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REFERENCE={REFERENCE}"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_mesh_new.restype = ctypes.c_void_p
        L.oracle_mesh_new.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32]
        L.oracle_mesh_free.argtypes = [ctypes.c_void_p]
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_bvh_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                                      ctypes.POINTER(ctypes.c_int)]
        L.oracle_closest_point.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_double,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.oracle_walk_samples.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
            ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p]
        L.oracle_estimate.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
            ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_diffwos.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p]
        L.oracle_exact_bump_green.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_hilbert_key.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_hilbert_key.restype = ctypes.c_uint32
        L.oracle_rqmc.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_sobol_directions.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p]
        L.oracle_sobol_directions.restype = None
        L.oracle_neighbour_means.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32] + \
            [ctypes.c_void_p] * 6
        L.oracle_neighbour_means.restype = None
        L.oracle_estimate_gradient.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
            ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_validate.argtypes = [
            ctypes.c_void_p, ctypes.POINTER(Params), ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p]
        assert L.oracle_sizeof_params() == ctypes.sizeof(Params)
        assert L.oracle_sizeof_site() == ctypes.sizeof(Site)
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def exact_bump_green(cases):
    """exact_bump_green (study.cpp:64-77, long double as the reference) for an
    [n, 4] array of (d, r, R, A) cases; raises on a negative integral."""
    c = np.ascontiguousarray(cases, dtype=np.float64).reshape(-1, 4)
    out = np.zeros(len(c))
    if lib().oracle_exact_bump_green(_ptr(c), len(c), _ptr(out)):
        raise RuntimeError(lib().oracle_last_error().decode())
    return out


def green_ball_quadrature(d, r, R, A):
    """Independent check of the closed form: the Green-volume integral of the
    bump over the ball, int_0^r (t - t^2/r) <f>_t dt with <f>_t the bump's
    mean over the sphere of radius t about the ball centre (a restatement of
    the reference's quadrature check, matched_accuracy/check_integral.py:11-20,
    written from the same integral), by scipy adaptive quadrature split at
    the support's kinks."""
    from scipy.integrate import quad

    def angular(t):
        # Mean of f over the sphere of radius t: half the integral over the
        # cosine c in [-1, 1] of A (a - b c)_+^2 (c flipped), with
        # a = 1 - (d^2 + t^2)/R^2 and b = 2 d t / R^2.
        if d * t == 0:
            return A * max(0.0, 1 - (d * d + t * t) / (R * R)) ** 2
        a = 1 - (d * d + t * t) / (R * R)
        b = 2 * d * t / (R * R)
        if a + b <= 0:
            return 0.0
        hi = min(1.0, a / b)

        def P(c):
            return a * a * c - a * b * c * c + b * b * c ** 3 / 3

        return A * (P(hi) - P(-1)) / 2

    cuts = sorted(set([0.0, r] + [t for t in (abs(d - R), d + R) if 0 < t < r]))
    return sum(quad(lambda t: (t - t * t / r) * angular(t), lo, hi, epsabs=1e-13 * A * R * R, epsrel=1e-10)[0]
               for lo, hi in zip(cuts[:-1], cuts[1:]))


# --------------------------------------------------------------------------- sources
def term(kind, amp=1.0, axis=0, offset=0.0, div=1.0, c=(0.0, 0.0, 0.0), w=(1.0, 1.0, 1.0)) -> Term:
    t = Term()
    t.kind, t.axis, t.amp, t.offset, t.div = kind, axis, amp, offset, div
    t.c[:] = list(c)
    t.w[:] = list(w)
    return t


def affine_source(slope=0.65):
    """wih_twos.cpp:550-552: f = 1 + slope*(y + 0.5)."""
    return [term(TERM_CONST, 1.0), term(TERM_LINEAR, slope, axis=1, offset=0.5)]


def housing_source():
    """wih_twos.cpp:553-565: 0.08 + 5.2 chip_a + 4.6 chip_b + 2.0 regulator."""
    return [
        term(TERM_CONST, 0.08),
        term(TERM_GAUSS, 5.2, c=(-0.48, -0.18, -0.08), w=(0.24, 0.22, 0.16)),
        term(TERM_GAUSS, 4.6, c=(0.43, 0.19, -0.07), w=(0.21, 0.20, 0.15)),
        term(TERM_GAUSS, 2.0, c=(0.02, -0.31, -0.02), w=(0.30, 0.16, 0.19)),
    ]


def sensor_source(side=1):
    """adjoint.cpp:11-15 with the --sensor-side flip of adjoint.cpp:98-102."""
    return [term(TERM_BUMP, 1.0, c=(0.55 * side, 0.18 * side, -0.03), w=(0.13, 0.0, 0.0))]


def load_study_config(path):
    """benchmarks/submission_study/study.cpp:37-42: a sensor line (x y z r)
    then heat lines (x y z r A).  Returns (sensor (x, y, z, r), heat source
    terms: sum of A * (1 - |x-c|^2/r^2)_+^2 in file order, study.cpp:27-35)."""
    rows = [list(map(float, line.split())) for line in open(path) if line.strip()]
    sensor = tuple(rows[0][:4])
    heat = [term(TERM_BUMP, r[4], c=tuple(r[:3]), w=(r[3], 0.0, 0.0)) for r in rows[1:]]
    if not heat:
        raise RuntimeError("missing compact heat sources")
    return sensor, heat


# --------------------------------------------------------------------------- mesh
class OracleMesh:
    def __init__(self, vertices: np.ndarray, faces: np.ndarray):
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.uint32)
        h = lib().oracle_mesh_new(_ptr(self.vertices), len(self.vertices), _ptr(self.faces), len(self.faces))
        if not h:
            raise RuntimeError(lib().oracle_last_error().decode())
        self.handle = h

    def __del__(self):
        if getattr(self, "handle", None):
            lib().oracle_mesh_free(self.handle)
            self.handle = None

    def bvh_info(self):
        n = ctypes.c_uint64()
        d = ctypes.c_int()
        lib().oracle_bvh_info(self.handle, ctypes.byref(n), ctypes.byref(d))
        return int(n.value), int(d.value)

    def closest_point(self, points, brute=False, radius=np.inf, threads=0):
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        n = len(pts)
        dist = np.empty(n)
        closest = np.empty((n, 3))
        tri = np.empty(n, dtype=np.uint32)
        counts = np.zeros((n, 2), dtype=np.uint64)
        lib().oracle_closest_point(self.handle, _ptr(pts), n, int(brute), float(radius),
                                   _ptr(dist), _ptr(closest), _ptr(tri), _ptr(counts), threads)
        return dist, closest, tri, counts

    def _params(self, **kw) -> Params:
        p = Params()
        p.mode = kw.get("mode", MODE_COMPLIANCE)
        p.rng = kw.get("rng", RNG_REFERENCE)
        p.walks = kw["walks"]
        p.max_steps = kw.get("max_steps", 512)
        p.seed = kw.get("seed", 20260912)
        p.repeat = kw.get("repeat", 0)
        p.stream = kw.get("stream", 0)
        p.epsilon = kw.get("epsilon", 5e-4)
        p.cavity_radius = kw.get("cavity_radius", 0.0)
        p.query_radius = kw.get("query_radius", 4.0)
        p.green = int(kw.get("green", False))
        src = kw.get("source", affine_source())
        adj = kw.get("adjoint", [])
        p.n_source, p.n_adjoint = len(src), len(adj)
        for i, t in enumerate(src):
            p.source[i] = t
        for i, t in enumerate(adj):
            p.adjoint[i] = t
        p.skip_cavity_sites = int(kw.get("skip_cavity_sites", p.mode != MODE_COMPLIANCE))
        p.weight_order = kw.get("weight_order", 0 if p.mode == MODE_COMPLIANCE else 1)
        p.threads = kw.get("threads", 0)
        bnd = kw.get("boundary", [])
        p.n_boundary = len(bnd)
        for i, t in enumerate(bnd):
            p.boundary[i] = t
        return p

    def walk_samples(self, sites, site_ids=None, cavities=None, count_tests=False, **kw):
        p = self._params(**kw)
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        ids = None if site_ids is None else np.ascontiguousarray(site_ids, dtype=np.uint64)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64)
        n = len(s)
        u = np.empty((n, p.walks))
        pp = np.empty((n, p.walks))
        st = np.empty((n, p.walks), dtype=np.uint32)
        tests = np.zeros((n, p.walks, 2), dtype=np.uint64) if count_tests else None
        rc = lib().oracle_walk_samples(self.handle, ctypes.byref(p), _ptr(s), _ptr(ids), n, _ptr(cav),
                                       len(cav), _ptr(u), _ptr(pp), _ptr(st), _ptr(tests))
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        out = {"u": u, "p": pp, "steps": st & 0x7FFFFFFF, "caps": (st >> 31).astype(bool)}
        if count_tests:
            out["aabb_tests"] = tests[..., 0]
            out["tri_tests"] = tests[..., 1]
        return out

    def diffwos(self, sites, cavities, diff_offset, site_ids=None, enclosure_fallback=True, **kw):
        """evaluate_differential_site over sites (wih_twos.cpp:839-928) in the
        reference stream.  Returns (derivs [n, ncav, 8] = dc(3), dc_se(3), dR,
        dR_se; stats [n, 7]; totals (distance queries, parity rays, fallbacks))."""
        p = self._params(**kw)
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        ids = None if site_ids is None else np.ascontiguousarray(site_ids, dtype=np.uint64)
        out = np.zeros((len(s), len(cav), 8))
        stats = np.zeros((len(s), 7), dtype=np.uint64)
        totals = np.zeros(3, dtype=np.uint64)
        rc = lib().oracle_diffwos(self.handle, ctypes.byref(p), float(diff_offset), int(bool(enclosure_fallback)),
                                  _ptr(s), _ptr(ids), len(s), _ptr(cav), len(cav), _ptr(out), _ptr(stats),
                                  _ptr(totals))
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        return out, stats, totals

    def rqmc(self, sites, method, batches, generator, u_boundary, p_boundary, record=False, **kw):
        """The GPU's lockstep Array-RQMC (method 1) / MC (method 0) / MC with
        neighbour reuse (method 2) / Sobol-over-steps RQMC (method 3) in the
        counter stream: (batch_u, batch_p
        [batches, n_sites], steps, caps), plus the per-walk record dict
        (walk_first, walk_u, walk_p, site_radius) when record is true."""
        p = self._params(**kw)
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        lo = np.ascontiguousarray(self.vertices.min(0))
        hi = np.ascontiguousarray(self.vertices.max(0))
        ub = (Term * max(1, len(u_boundary)))(*u_boundary)
        pb = (Term * max(1, len(p_boundary)))(*p_boundary)
        n, w = len(s), p.walks
        bu = np.zeros((batches, n))
        bp = np.zeros((batches, n))
        tot = np.zeros(2, dtype=np.uint64)
        rec = {"walk_first": np.zeros((batches, n, w, 3)), "walk_u": np.zeros((batches, n, w)),
               "walk_p": np.zeros((batches, n, w)), "site_radius": np.zeros(n)}
        keep = record or method == 2
        rc = lib().oracle_rqmc(self.handle, ctypes.byref(p), method if method in (1, 3) else 0, int(batches),
                               int(generator),
                               _ptr(lo), _ptr(hi), ctypes.cast(ub, ctypes.c_void_p), len(u_boundary),
                               ctypes.cast(pb, ctypes.c_void_p), len(p_boundary), _ptr(s), n, _ptr(bu), _ptr(bp),
                               _ptr(tot), *[_ptr(rec[k]) if keep else None for k in
                                            ("walk_first", "walk_u", "walk_p", "site_radius")])
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        if method == 2:
            lib().oracle_neighbour_means(_ptr(s), n, int(batches), w, _ptr(rec["walk_first"]), _ptr(rec["walk_u"]),
                                         _ptr(rec["walk_p"]), _ptr(rec["site_radius"]), _ptr(bu), _ptr(bp))
        out = (bu, bp, int(tot[0]), int(tot[1]))
        return out + (rec,) if record else out

    def estimate_gradient(self, sites, cavities=None, samples=False, **kw):
        """The GPU gradient form in the counter stream (rng must be the counter
        stream): rows (u, p, grad_u, grad_p, cross, cross_se, u_se, p_se), steps/caps, and
        optionally the per-walk samples [n, walks, 8]."""
        p = self._params(**kw)
        if p.rng != RNG_COUNTER:
            raise ValueError("the gradient form is defined in the counter stream")
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        rows = np.zeros((len(s), 12))
        counts = np.zeros((len(s), 2), dtype=np.uint64)
        walks = np.zeros((len(s), p.walks, 8)) if samples else None
        rc = lib().oracle_estimate_gradient(self.handle, ctypes.byref(p), _ptr(s), len(s), _ptr(cav), len(cav),
                                            _ptr(rows), _ptr(counts), _ptr(walks))
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        out = {"u": rows[:, 0], "p": rows[:, 1], "grad_u": rows[:, 2:5], "grad_p": rows[:, 5:8], "cross": rows[:, 8],
               "cross_se": rows[:, 9], "u_se": rows[:, 10], "p_se": rows[:, 11], "steps": counts[:, 0],
               "caps": counts[:, 1]}
        if samples:
            out["samples"] = walks
        return out

    def validate(self, sites, radius_cap, value_cap, site_ids=None, cavities=None, **kw):
        """Certified fresh samples (minimum_benefit.hpp cert_walk) at each site:
        dict of value, steps, capped, clipped, contained ([n_sites, walks]) and
        clearance (the certified domain distance at each site)."""
        p = self._params(**kw)
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        ids = None if site_ids is None else np.ascontiguousarray(site_ids, dtype=np.uint64)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64).reshape(-1, 3)
        n, w = len(s), p.walks
        value = np.zeros((n, w))
        steps = np.zeros((n, w), dtype=np.uint32)
        flags = np.zeros((n, w), dtype=np.uint8)
        clearance = np.zeros(n)
        rc = lib().oracle_validate(self.handle, ctypes.byref(p), float(radius_cap), float(value_cap), _ptr(s),
                                   _ptr(ids), n, _ptr(cav), len(cav), _ptr(value), _ptr(steps), _ptr(flags),
                                   _ptr(clearance))
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        return {"value": value, "steps": steps, "capped": (flags & 1) != 0, "clipped": (flags & 2) != 0,
                "contained": (flags & 4) == 0, "clearance": clearance}

    def estimate(self, sites, site_ids=None, cavities=None, **kw):
        p = self._params(**kw)
        s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        ids = None if site_ids is None else np.ascontiguousarray(site_ids, dtype=np.uint64)
        cav = np.zeros((0, 3)) if cavities is None else np.ascontiguousarray(cavities, dtype=np.float64)
        n = len(s)
        out = (Site * n)()
        rc = lib().oracle_estimate(self.handle, ctypes.byref(p), _ptr(s), _ptr(ids), n, _ptr(cav), len(cav),
                                   ctypes.cast(out, ctypes.c_void_p))
        if rc:
            raise RuntimeError(lib().oracle_last_error().decode())
        arr = np.frombuffer(out, dtype=np.dtype([
            ("u", "f8"), ("p", "f8"), ("score", "f8"), ("score_se", "f8"), ("same_index", "f8"),
            ("steps", "u8"), ("caps", "u8")]), count=n)
        return arr.copy()


# --------------------------------------------------------------------------- readers
def _open_text(path):
    path = str(path)
    if path.endswith(".gz"):
        return gzip.open(path, "rt")
    return open(path, "r")


def load_ascii_ply(path):
    """Restates wih_twos.cpp:437-493: ASCII triangle PLY, FP64 vertices.

    The header must declare ``format ascii``, a vertex and a face count and
    end with ``end_header``; every face must be a triangle with indices in
    range.  Errors carry the reference's messages.
    """
    with _open_text(path) as fh:
        vertex_count = face_count = 0
        ascii = header_done = False
        for line in fh:
            words = line.split()
            if not words:
                continue
            if words[0] == "format":
                ascii = len(words) > 1 and words[1] == "ascii"
            elif words[0] == "element":
                kind = words[1] if len(words) > 1 else ""
                count = int(words[2]) if len(words) > 2 else 0
                if kind == "vertex":
                    vertex_count = count
                if kind == "face":
                    face_count = count
            elif words[0] == "end_header":
                header_done = True
                break
        if not ascii or not header_done or vertex_count == 0 or face_count == 0:
            raise RuntimeError("expected a nonempty ASCII triangle PLY mesh")
        vertices = np.empty((vertex_count, 3))
        for i in range(vertex_count):
            parts = fh.readline().split()
            if len(parts) < 3:
                raise RuntimeError("truncated PLY vertex section")
            vertices[i] = [float(parts[0]), float(parts[1]), float(parts[2])]
        faces = np.empty((face_count, 3), dtype=np.uint32)
        for i in range(face_count):
            parts = fh.readline().split()
            if len(parts) < 4 or int(parts[0]) != 3:
                raise RuntimeError("expected valid triangular PLY faces")
            idx = [int(parts[1]), int(parts[2]), int(parts[3])]
            if min(idx) < 0 or max(idx) >= vertex_count:
                raise RuntimeError("expected valid triangular PLY faces")
            faces[i] = idx
    return vertices, faces


def read_points(path):
    """Restates wih_twos.cpp:508-522: comma or whitespace x,y,z rows; '#' comments."""
    pts = []
    with _open_text(path) as fh:
        for line in fh:
            line = line.rstrip("\n")
            if not line or line[0] == "#":
                continue
            parts = line.replace(",", " ").split()
            if len(parts) >= 3:
                try:
                    pts.append([float(parts[0]), float(parts[1]), float(parts[2])])
                except ValueError:
                    continue
    if not pts:
        raise RuntimeError("points file contains no points")
    return np.array(pts)


# --------------------------------------------------------------------------- statistics
def crossfit_square(samples):
    """run_bunny_benchmark.py:257-269: U-statistic of u^2 and jackknife SE."""
    samples = np.asarray(samples, dtype=float)
    n = samples.shape[1]
    sums = samples.sum(axis=1)
    sums2 = np.sum(samples ** 2, axis=1)
    estimate = (sums ** 2 - sums2) / (n * (n - 1))
    leave_sums = sums[:, None] - samples
    leave_sums2 = sums2[:, None] - samples ** 2
    leave = (leave_sums ** 2 - leave_sums2) / ((n - 1) * (n - 2))
    leave_mean = leave.mean(axis=1, keepdims=True)
    se = np.sqrt((n - 1) / n * np.sum((leave - leave_mean) ** 2, axis=1))
    return estimate, se


def sobol_directions(dims, bits=10):
    """The Sobol' direction numbers of twos_rqmc's SOBOL method, [dims, bits]
    uint32 (most significant digit first): oracle_sobol_directions."""
    out = np.zeros((int(dims), int(bits)), dtype=np.uint32)
    lib().oracle_sobol_directions(int(dims), int(bits), out.ctypes.data)
    return out


def crossfit_product(a, b):
    """experiments/run_controlled_experiments.py:79-87: minus the off-diagonal
    mean of a_i b_j along the last axis (the reference's sign: an estimate of
    -E[A]E[B], the TD of a compliance-type objective)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    n = a.shape[-1]
    if n < 2:
        raise ValueError("cross-fitting requires at least two pairs")
    return -(np.sum(a, axis=-1) * np.sum(b, axis=-1) - np.sum(a * b, axis=-1)) / (n * (n - 1))


CROSSFIT_SEED = 20260912  # run_controlled_experiments.py:34 (SEED); the experiment takes spawn index 2 (:800-801)


def crossfit_experiment_draws(correlation, rng, n=32, replicates=30000, mu=(0.8, 0.65), sigma=(0.5, 0.6)):
    """One correlation of run_crossfit_experiment (run_controlled_experiments.py:250-271):
    the paired samples a, b and the independent b' [replicates, n], drawn in the
    reference's order (z1, z2, z3 standard normals)."""
    z1 = rng.standard_normal(size=(replicates, n))
    z2 = rng.standard_normal(size=(replicates, n))
    z3 = rng.standard_normal(size=(replicates, n))
    a = mu[0] + sigma[0] * z1
    b = mu[1] + sigma[1] * (correlation * z1 + np.sqrt(1.0 - correlation * correlation) * z2)
    b_independent = mu[1] + sigma[1] * z3
    return a, b, b_independent


def crossfit_experiment(estimator=None, n=32, replicates=30000):
    """run_crossfit_experiment (run_controlled_experiments.py:250-321): for each
    correlation in linspace(-0.9, 0.9, 10), the four estimators' mean and bias
    against true_td = -mu_a mu_b.  `estimator(a, b)` replaces the cross-fit
    estimator (crossfit_product by default), so a device reduction can be
    dropped into the same seeded experiment.  Rows as dicts keyed like the
    reference's crossfit_bias.csv."""
    estimator = estimator or crossfit_product
    rng = np.random.default_rng(np.random.SeedSequence(CROSSFIT_SEED).spawn(5)[2])
    mu_a, mu_b = 0.8, 0.65
    true_td = -mu_a * mu_b
    rows = []
    for correlation in np.linspace(-0.9, 0.9, 10):
        a, b, bi = crossfit_experiment_draws(correlation, rng, n, replicates)
        estimates = {
            "Same-seed product": -np.mean(a * b, axis=1),
            "Product of means": -np.mean(a, axis=1) * np.mean(b, axis=1),
            "Cross-fit TWoS": estimator(a, b),
            "Independent batches": -np.mean(a, axis=1) * np.mean(bi, axis=1),
        }
        for method, values in estimates.items():
            err = values - true_td
            rows.append({"method": method, "correlation": float(correlation), "true_td": true_td,
                         "mean_estimate": float(np.mean(values)), "bias": float(np.mean(err)),
                         "bias_se": float(np.std(err, ddof=1) / np.sqrt(replicates)),
                         "rmse": float(np.sqrt(np.mean(err * err)))})
    return rows


def cross_jackknife_se(a, b):
    """Leave-one-out jackknife SE of the cross statistic (the compliance
    formula of wih_twos.cpp:698-712 applied to the product a_i b_j, i != j)."""
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    n = a.shape[-1]
    sa = a.sum(axis=-1, keepdims=True)
    sb = b.sum(axis=-1, keepdims=True)
    sab = np.sum(a * b, axis=-1, keepdims=True)
    leave = ((sa - a) * (sb - b) - (sab - a * b)) / ((n - 1) * (n - 2))
    lm = leave.mean(axis=-1, keepdims=True)
    return np.sqrt((n - 1) / n * np.sum((leave - lm) ** 2, axis=-1))


def select_shortlist_rescore(scout, shortlist, validation, validation_se, z=1.96):
    """run_bunny_benchmark.py:323-331: top-`shortlist` by scout score, then
    argmax of validation - z*se.  Returns (chosen candidate index, lower)."""
    scout = np.asarray(scout, dtype=float)
    k = min(shortlist, len(scout))
    # Deterministic top-k: highest score first, lowest index on ties.
    order = np.lexsort((np.arange(len(scout)), -scout))[:k]
    lower = np.asarray(validation, dtype=float) - z * np.asarray(validation_se, dtype=float)
    local = int(np.argmax(lower))
    return int(order[local]), float(lower[local]), order


def design_loop(mesh: "OracleMesh", candidates, scout_kw, validate_kw, iterations, shortlist, cavity_radius,
                z=1.96, accept_threshold=0.0, outer_clearance=0.0, pair_gap=0.0, cavities=None):
    """FP64 restatement of the design loop on the GPU's counter stream:
    select_twos (run_bunny_benchmark.py:302-337) -- feasible scout, top-k by
    score, fresh rescore, argmax of score - z*se (run_bunny_benchmark.py:330-331)
    -- with insertion when the bound clears accept_threshold and the feasibility
    mask of run_bunny_benchmark.py:290-299.  Iteration i uses repeat = i;
    scout walks are keyed by candidate index, validation walks by shortlist
    slot.  Returns (history list of dicts, cavities array)."""
    cand = np.asarray(candidates, dtype=np.float64).reshape(-1, 3)
    cav = np.zeros((0, 3)) if cavities is None else np.asarray(cavities, dtype=np.float64).reshape(-1, 3)
    dist, _, _, _ = mesh.closest_point(cand)
    pair = 2.0 * cavity_radius + pair_gap
    feasible = dist >= cavity_radius + outer_clearance
    for c in cav:
        feasible &= np.sum((cand - c) ** 2, axis=1) >= pair * pair
    history = []
    ids = np.arange(len(cand), dtype=np.uint64)
    for it in range(iterations):
        scout = mesh.estimate(cand, site_ids=ids, cavities=cav, cavity_radius=cavity_radius, repeat=it,
                              rng=RNG_COUNTER, weight_order=1, **scout_kw)
        keys = np.where(feasible & ~np.isnan(scout["score"]), scout["score"], -np.inf)
        short = topk_indices(keys, shortlist)
        val = mesh.estimate(cand[short], site_ids=np.arange(len(short), dtype=np.uint64), cavities=cav,
                            cavity_radius=cavity_radius, repeat=it, rng=RNG_COUNTER, weight_order=1, **validate_kw)
        lower = val["score"] - z * val["score_se"]
        lower = np.where(np.isnan(lower), -np.inf, lower)
        slot = int(np.argmax(lower))
        c = int(short[slot])
        accepted = bool(lower[slot] > accept_threshold)
        history.append({"chosen": c, "accepted": accepted, "scout_score": float(scout["score"][c]),
                        "score": float(val["score"][slot]), "score_se": float(val["score_se"][slot]),
                        "lower": float(lower[slot])})
        if accepted:
            cav = np.vstack([cav, cand[c][None, :]])
            feasible &= np.sum((cand - cand[c]) ** 2, axis=1) >= pair * pair
    return history, cav


def topk_indices(score, k):
    """Top-k indices by score descending, ties broken by the lower index."""
    score = np.asarray(score, dtype=float)
    return np.lexsort((np.arange(len(score)), -score))[:k]


def default_threads():
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
