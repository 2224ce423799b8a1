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


# --------------------------------------------------------------------- housing-like box
def cylinder_centres(seed: int = 34, count: int = 6, radius: float = 0.15, size=(4.0, 2.0), gap: float = 0.1):
    """Axis-z through-cylinder centres for the box [0, 4] x [0, 2] x [0, 1]:
    drawn uniformly from numpy.random.default_rng(seed), each kept when its
    disc stays `gap` from the box sides and from every kept disc, until
    `count` are kept (the builder's rule; the workload fixes seed 34)."""
    rng = np.random.default_rng(seed)
    keep = []
    lo = radius + gap
    while len(keep) < count:
        c = np.array([rng.uniform(lo, size[0] - lo), rng.uniform(lo, size[1] - lo)])
        if all(np.linalg.norm(c - k) >= 2 * radius + gap for k in keep):
            keep.append(c)
    return np.array(keep)


def box_minus_cylinders(h: float = 0.0115, seed: int = 34, radius: float = 0.15, size=(4.0, 2.0, 1.0)):
    """Closed, outward-oriented triangle surface of the box [0, sx] x [0, sy] x
    [0, sz] minus `count` = 6 through-cylinders of `radius` along z (centres
    from ``cylinder_centres(seed)``), with edge length about h (h = 0.0115
    gives 529,608 triangles).

    Construction: the rectangle's edges and the circles are sampled at
    spacing ~h; interior points of a hexagonal lattice of spacing h are kept
    at least 0.75 h away from every boundary; their Delaunay triangulation
    (scipy), minus the triangles whose centroid lies in a disc, is the top
    and the bottom face.  The box sides and the cylinder walls are strips of
    quadrilaterals between the same boundary points at nz + 1 heights, each
    split in two triangles; all pieces share their boundary vertices, so the
    surface is watertight.  Returns (vertices [n, 3], faces [m, 3] uint32,
    centres [6, 2])."""
    from scipy.spatial import Delaunay
    sx, sy, sz = size
    centres = cylinder_centres(seed, radius=radius, size=(sx, sy))
    # Boundary loops: the rectangle (counter-clockwise) and each circle.
    nxs, nys = max(2, int(round(sx / h))), max(2, int(round(sy / h)))
    rect = np.concatenate([
        np.c_[np.linspace(0, sx, nxs, endpoint=False), np.zeros(nxs)],
        np.c_[np.full(nys, sx), np.linspace(0, sy, nys, endpoint=False)],
        np.c_[np.linspace(sx, 0, nxs, endpoint=False), np.full(nxs, sy)],
        np.c_[np.zeros(nys), np.linspace(sy, 0, nys, endpoint=False)]])
    nc = max(12, int(round(2 * math.pi * radius / h)))
    ang = 2 * math.pi * np.arange(nc) / nc
    circles = [c + radius * np.c_[np.cos(ang), np.sin(ang)] for c in centres]
    # Interior: hexagonal lattice points away from every boundary.
    rows = np.arange(0.0, sy, h * math.sqrt(3) / 2)
    pts = [np.c_[np.arange((i % 2) * h / 2, sx, h), np.full(len(np.arange((i % 2) * h / 2, sx, h)), y)]
           for i, y in enumerate(rows)]
    interior = np.concatenate(pts)
    m = 0.75 * h
    keep = (interior[:, 0] > m) & (interior[:, 0] < sx - m) & (interior[:, 1] > m) & (interior[:, 1] < sy - m)
    for c in centres:
        keep &= np.linalg.norm(interior - c, axis=1) > radius + m
    interior = interior[keep]
    loops = [rect] + circles
    boundary = np.concatenate(loops)
    pts2 = np.concatenate([boundary, interior])
    tri = Delaunay(pts2).simplices
    cen = pts2[tri].mean(axis=1)
    inside_hole = np.zeros(len(tri), bool)
    for c in centres:
        inside_hole |= np.linalg.norm(cen - c, axis=1) < radius
    tri = tri[~inside_hole]
    # Orient 2D triangles counter-clockwise.
    a, b, c3 = pts2[tri[:, 0]], pts2[tri[:, 1]], pts2[tri[:, 2]]
    cross = (b[:, 0] - a[:, 0]) * (c3[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c3[:, 0] - a[:, 0])
    tri = np.where((cross > 0)[:, None], tri, tri[:, [0, 2, 1]])
    tri = tri[np.abs(cross) > 0]
    # Heights of the wall strips; the faces use the first and last level.
    nz = max(1, int(round(sz / h)))
    zs = np.linspace(0.0, sz, nz + 1)
    nb = len(boundary)
    npts = len(pts2)
    # Vertex blocks: bottom face (all 2D points at z=0), top face (z=sz),
    # then the boundary points at the inner heights.
    verts = [np.c_[pts2, np.zeros(npts)], np.c_[pts2, np.full(npts, sz)]]
    for z in zs[1:-1]:
        verts.append(np.c_[boundary, np.full(nb, z)])
    V = np.concatenate(verts)

    def ring_index(level, k):
        # Index of boundary point k at height level (0 .. nz).
        if level == 0:
            return k
        if level == nz:
            return npts + k
        return 2 * npts + (level - 1) * nb + k

    faces = [tri[:, [0, 2, 1]], tri + npts]  # bottom faces down (-z), top faces up (+z)
    start = 0
    for li, loop in enumerate(loops):
        n = len(loop)
        k = np.arange(n)
        k1 = (k + 1) % n
        for lv in range(nz):
            a0, b0 = ring_index(lv, start + k), ring_index(lv, start + k1)
            a1, b1 = ring_index(lv + 1, start + k), ring_index(lv + 1, start + k1)
            if li == 0:
                # Box sides: the loop runs counter-clockwise seen from +z, so
                # (a0, b0, b1) faces outward.
                faces.append(np.c_[a0, b0, b1])
                faces.append(np.c_[a0, b1, a1])
            else:
                # Cylinder walls face the cylinder axis (out of the solid).
                faces.append(np.c_[a0, b1, b0])
                faces.append(np.c_[a0, a1, b1])
        start += n
    F = np.concatenate(faces).astype(np.uint32)
    return V, F, centres


def disc_area_beyond(centre, radius: float, x0: float, right: bool = True) -> float:
    """Area of the disc |p - centre| <= radius with p.x >= x0 (right) or
    p.x <= x0 (left): a circular segment."""
    d = (x0 - centre[0]) if right else (centre[0] - x0)  # signed distance from the centre to the cut
    if d >= radius:
        return 0.0
    if d <= -radius:
        return math.pi * radius ** 2
    return radius ** 2 * math.acos(d / radius) - d * math.sqrt(radius ** 2 - d ** 2)


def box_region_volume(centres, radius: float, x0: float, right: bool, size=(4.0, 2.0, 1.0)) -> float:
    """Volume of {x >= x0} (right) or {x <= x0} of the box minus cylinders."""
    sx, sy, sz = size
    slab = (sx - x0 if right else x0) * sy * sz
    return slab - sz * sum(disc_area_beyond(c, radius, x0, right) for c in centres)


def box_interior_points(n: int, centres, radius: float, seed: int, size=(4.0, 2.0, 1.0)):
    """n points uniform in the box minus the cylinders (rejection sampling,
    numpy.random.default_rng(seed))."""
    rng = np.random.default_rng(seed)
    out = []
    need = n
    while need > 0:
        p = rng.random((2 * need + 16, 3)) * np.asarray(size)
        ok = np.ones(len(p), bool)
        for c in centres:
            ok &= np.hypot(p[:, 0] - c[0], p[:, 1] - c[1]) > radius
        p = p[ok][:need]
        out.append(p)
        need -= len(p)
    return np.concatenate(out)
