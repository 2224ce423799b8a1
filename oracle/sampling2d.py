"""TEST INFRASTRUCTURE: a restatement of the reference's 2D sampling study
(benchmarks/critical_baselines/sampling.py), the source of the Array-RQMC,
Sobol-over-steps RQMC and neighbour-reuse estimators that twos_rqmc runs in
3D on a mesh.  Pinned to the study's tracked per-site estimates
(critical_baselines/output/sampling_fields.csv) by tests/test_sampling2d_cpu.py,
so the algorithms the 3D kernel extends are checked against the reference's
own numbers:

* harmonic Dirichlet fields u, p on the unit disk or square (:16-19) and the
  distance / exit projection of each domain (:21-31);
* the 2D Hilbert index on a 2^13 grid (:33-46);
* walks (:48-71): MC draws, Sobol-over-steps RQMC (one scrambled Sobol point
  of dimension `cap` per walk, coordinate `step` at step `step`; scipy's
  generator, the reference's own dependency), and Array-RQMC (walks sorted by
  Hilbert key with converged paths last, the shifted Korobov lattice
  (a i / n + U) mod 1 assigned by rank);
* the neighbour-reuse means with geometry weights (1 - a)^4 / (1 - a^2)^2 and
  the Poisson-kernel ratio (:73-86);
* the cross-fit over batches (:88-90).
"""
from __future__ import annotations

import numpy as np

KOROBOV = {16: 7, 32: 7, 64: 19, 128: 49, 256: 75, 512: 189, 1024: 283, 2048: 857}  # sampling.py:14
STUDY_SEED = 20260914  # sampling.py:123


def harmonic_fields(z):
    """u = 0.28 + 0.58 x - 0.30 y + 0.22 (x^2 - y^2), p = 0.46 - 0.38 x + 0.34 y + 0.40 x y."""
    x, y = z.real, z.imag
    u = 0.28 + 0.58 * x - 0.30 * y + 0.22 * (x * x - y * y)
    p = 0.46 - 0.38 * x + 0.34 * y + 0.40 * x * y
    return u, p


def boundary_distance(z, domain):
    if domain == "disk":
        return 1 - np.abs(z)
    return 1 - np.maximum(np.abs(z.real), np.abs(z.imag))


def exit_point(z, domain):
    if domain == "disk":
        return z / np.abs(z)
    x, y = z.real.copy(), z.imag.copy()
    on_x = np.abs(x) >= np.abs(y)
    x[on_x] = np.sign(x[on_x])
    y[~on_x] = np.sign(y[~on_x])
    return x + 1j * y


def hilbert2(z, bits=13):
    """Hilbert distance of z's cell on the 2^bits grid over [-1, 1]^2, the
    rotate-and-flip form of the curve (quadrant digit (3 rx) ^ ry)."""
    side = 1 << bits
    x = np.clip(np.floor((z.real + 1) * side / 2), 0, side - 1).astype(np.int64)
    y = np.clip(np.floor((z.imag + 1) * side / 2), 0, side - 1).astype(np.int64)
    h = np.zeros(z.shape, dtype=np.int64)
    s = side // 2
    while s:
        rx = (x & s) > 0
        ry = (y & s) > 0
        h += s * s * ((3 * rx.astype(np.int64)) ^ ry.astype(np.int64))
        rotate = ~ry
        flip = rotate & rx
        x = np.where(flip, s - 1 - x, x)
        y = np.where(flip, s - 1 - y, y)
        x, y = np.where(rotate, y, x), np.where(rotate, x, y)
        s //= 2
    return h


def own_sobol_points(n, dims, rng):
    """n points of the Sobol' sequence of twos_rqmc's SOBOL method (the
    oracle's direction numbers: primitive polynomials in order, seeded odd
    initial values), scrambled as that method scrambles -- a random
    lower-triangular digit matrix with unit diagonal and a digital shift per
    coordinate -- with draws from `rng`: [n, dims] in (0, 1)."""
    import oracle
    bits = int(np.log2(n))
    v = oracle.sobol_directions(dims, bits).astype(np.uint64)
    r = np.arange(32, dtype=np.uint64)
    rows = rng.integers(0, 2 ** 32, size=(dims, 32), dtype=np.uint64)
    rows = (rows & ((np.uint64(0xffffffff) << (np.uint64(31) - r)) & np.uint64(0xffffffff))) | \
        (np.uint64(1) << (np.uint64(31) - r))
    parity = np.bitwise_count(rows[:, None, :] & v[:, :, None]) & 1
    dirs = np.bitwise_or.reduce(parity.astype(np.uint64) << (np.uint64(31) - r), axis=-1)
    x = np.broadcast_to(rng.integers(0, 2 ** 32, size=dims, dtype=np.uint64), (n, dims)).copy()
    idx = np.arange(n)
    for b in range(bits):
        x[(idx >> b) & 1 == 1] ^= dirs[:, b]
    return (x.astype(np.float64) + 0.5) / 2.0 ** 32


def walk_batch(starts, n, seed, domain, method, eps=1e-7, cap=256):
    """n walks from each start; returns (first step points, exit points).
    The random draws follow the study's order exactly: one generator per
    batch; RQMC draws one Sobol seed per start up front; Array-RQMC draws
    one lattice shift per start per step."""
    from scipy.stats import qmc
    rng = np.random.default_rng(seed)
    z = np.repeat(starts[:, None], n, axis=1).astype(complex)
    first = None
    if method == "rqmc":
        m = int(np.log2(n))
        points = np.stack([qmc.Sobol(cap, scramble=True, seed=int(s)).random_base2(m)
                           for s in rng.integers(0, 2 ** 31 - 1, len(starts))])
    elif method == "sobol_own":  # not in the study: the 3D method's sequence, one coordinate per step
        points = np.stack([own_sobol_points(n, cap, rng) for _ in starts])
    lattice = (KOROBOV.get(n, 1) * np.arange(n)) % n / n if method == "array" else None
    for step in range(cap):
        r = boundary_distance(z, domain)
        live = r > eps
        if not live.any():
            break
        if method == "array":
            keys = np.where(live, hilbert2(z), np.iinfo(np.int64).max)
            rank_order = np.argsort(keys, axis=1, kind="stable")
            shifted = (lattice[None, :] + rng.random((len(starts), 1))) % 1
            u = np.empty_like(shifted)
            np.put_along_axis(u, rank_order, shifted, axis=1)
        elif method in ("rqmc", "sobol_own"):
            u = points[:, :, step]
        else:
            u = rng.random(z.shape)
        z[live] += r[live] * np.exp(2j * np.pi * u[live])
        if first is None:
            first = z.copy()
    if np.any(boundary_distance(z, domain) > eps):
        raise RuntimeError("unconverged walks")
    return first, exit_point(z, domain)


def reuse_means(starts, first, exits, domain):
    """Each site's means pooled from every site y whose first ball B(y, r_y)
    contains it: site weight (1 - a)^4 / (1 - a^2)^2 with a = |x - y| / r_y,
    walk weight the Poisson-kernel ratio (r_y^2 - |x - y|^2) / |x - z1|^2."""
    u, p = harmonic_fields(exits)
    r = boundary_distance(starts, domain)
    out = np.zeros((len(starts), 2))
    for k, x in enumerate(starts):
        a = np.abs(x - starts) / r
        use = a < 1 - 1e-12
        w = (1 - a[use]) ** 4 / (1 - a[use] ** 2) ** 2
        ratio = (r[use][:, None] ** 2 - np.abs(x - starts[use, None]) ** 2) / np.abs(x - first[use]) ** 2
        out[k, 0] = np.sum(w * np.mean(ratio * u[use], axis=1)) / w.sum()
        out[k, 1] = np.sum(w * np.mean(ratio * p[use], axis=1)) / w.sum()
    return out[:, 0], out[:, 1]


def crossfit_batches(a, b):
    """-(sum a sum b - sum a b) / (R (R - 1)) over the R batches."""
    r = a.shape[0]
    return -(a.sum(axis=0) * b.sum(axis=0) - (a * b).sum(axis=0)) / (r * (r - 1))


def study_sites():
    g = np.linspace(-0.55, 0.55, 5)
    return (g[:, None] + 1j * g[None, :]).ravel()


def td_estimate(domain_id, domain, n, rep, method, batches=4):
    """One (domain, n, repetition, method) cell of the study: the cross-fit TD
    at the 25 sites over `batches` independent batches (sampling.py:126-139)."""
    starts = study_sites()
    a, b = [], []
    for batch in range(batches):
        seed = int(np.random.SeedSequence([STUDY_SEED, domain_id, n, rep, batch]).generate_state(1)[0])
        first, exits = walk_batch(starts, n, seed, domain, "mc" if method == "neighbors" else method)
        if method == "neighbors":
            u, p = reuse_means(starts, first, exits, domain)
        else:
            u, p = harmonic_fields(exits)
            u, p = u.mean(axis=1), p.mean(axis=1)
        a.append(u)
        b.append(p)
    return crossfit_batches(np.array(a), np.array(b))
