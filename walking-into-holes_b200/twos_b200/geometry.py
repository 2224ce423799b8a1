"""Synthetic geometry for the benchmark workloads, and PLY/CSV writers.

* ``icosphere(level)``: unit icosphere by midpoint subdivision of the
  icosahedron (20 * 4**level triangles; level 4 -> 5,120, level 7 -> 327,680).
* ``sh_displace``: radial displacement r = 1 + amplitude * S(theta, phi), S a
  sum of ``count`` real spherical harmonics of degree 1..max_degree.
  Coefficient law (fixed here, seed-driven): for k = 1..count, degree
  l ~ U{1..max_degree}, order m ~ U{-l..l}, coefficient a_k ~ N(0, 1/count);
  harmonics are orthonormal on the sphere times sqrt(4 pi) (unit RMS), so S
  has unit RMS in expectation.  numpy.random.default_rng(seed) draws l, m, a
  in that order per k.
* ``grid_sites``: n^3 cell centres of the bounding box, kept when inside
  the mesh by ray parity.
"""
from __future__ import annotations

import math

import numpy as np

_PHI = (1.0 + math.sqrt(5.0)) / 2.0


def icosahedron():
    v = np.array([
        [-1, _PHI, 0], [1, _PHI, 0], [-1, -_PHI, 0], [1, -_PHI, 0],
        [0, -1, _PHI], [0, 1, _PHI], [0, -1, -_PHI], [0, 1, -_PHI],
        [_PHI, 0, -1], [_PHI, 0, 1], [-_PHI, 0, -1], [-_PHI, 0, 1],
    ], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([
        [0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
        [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
        [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
        [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1],
    ], dtype=np.int64)
    return v, f


def icosphere(level: int):
    """Unit-radius icosphere with outward-oriented faces (vertices on the sphere)."""
    v, f = icosahedron()
    for _ in range(level):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, axis=1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        nf = len(f)
        a = inv[:nf] + base
        b = inv[nf:2 * nf] + base
        c = inv[2 * nf:] + base
        f = np.concatenate([
            np.stack([f[:, 0], a, c], axis=1),
            np.stack([f[:, 1], b, a], axis=1),
            np.stack([f[:, 2], c, b], axis=1),
            np.stack([a, b, c], axis=1),
        ])
    return v, f.astype(np.uint32)


def _real_sh(l, m, theta, phi):
    """Real spherical harmonic of unit RMS over the sphere (orthonormal * sqrt(4 pi))."""
    from scipy.special import sph_harm_y
    y = sph_harm_y(l, abs(m), theta, phi)
    if m > 0:
        val = math.sqrt(2.0) * (-1) ** m * y.real
    elif m < 0:
        val = math.sqrt(2.0) * (-1) ** m * y.imag
    else:
        val = y.real
    return val * math.sqrt(4.0 * math.pi)


def sh_field(points, seed: int, count: int = 8, max_degree: int = 6):
    rng = np.random.default_rng(seed)
    p = np.asarray(points, dtype=np.float64)
    r = np.linalg.norm(p, axis=1)
    theta = np.arccos(np.clip(p[:, 2] / r, -1.0, 1.0))
    phi = np.arctan2(p[:, 1], p[:, 0])
    s = np.zeros(len(p))
    for _ in range(count):
        l = int(rng.integers(1, max_degree + 1))
        m = int(rng.integers(-l, l + 1))
        a = float(rng.normal(0.0, 1.0 / math.sqrt(count)))
        s += a * _real_sh(l, m, theta, phi)
    return s


def sh_displace(vertices, seed: int, amplitude: float = 0.15, count: int = 8, max_degree: int = 6):
    s = sh_field(vertices, seed, count, max_degree)
    scale = 1.0 + amplitude * s
    if np.min(scale) <= 0.05:
        raise ValueError("displacement folds the sphere; choose another seed")
    return vertices * scale[:, None]


def noise_sphere(level: int, seed: int, amplitude: float = 0.15):
    """The noise-displaced icosphere workload (subdivision `level`, harmonic seed)."""
    v, f = icosphere(level)
    return sh_displace(v, seed, amplitude), f


def grid_points(lo, hi, n: int):
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    t = (np.arange(n) + 0.5) / n
    gx, gy, gz = np.meshgrid(lo[0] + t * (hi[0] - lo[0]), lo[1] + t * (hi[1] - lo[1]),
                             lo[2] + t * (hi[2] - lo[2]), indexing="ij")
    return np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)


def uniform_ball(n: int, radius: float, seed: int):
    """n points uniform in the ball |x| < radius (numpy default_rng(seed):
    directions from normals, radii by the cube-root transform)."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.random(n) ** (1.0 / 3.0)
    return d * r[:, None]


def write_ply(path, vertices, faces):
    v = np.asarray(vertices, dtype=np.float64)
    f = np.asarray(faces, dtype=np.int64)
    with open(path, "w") as fh:
        fh.write("ply\nformat ascii 1.0\n")
        fh.write(f"element vertex {len(v)}\nproperty double x\nproperty double y\nproperty double z\n")
        fh.write(f"element face {len(f)}\nproperty list uchar int vertex_indices\nend_header\n")
        np.savetxt(fh, v, fmt="%.17g")
        np.savetxt(fh, np.concatenate([np.full((len(f), 1), 3), f], axis=1), fmt="%d")


def write_points(path, points):
    np.savetxt(path, np.asarray(points, dtype=np.float64).reshape(-1, 3), delimiter=",", fmt="%.17g")
