"""Site sharding over ranks (one process per GPU, torch.distributed).

The reference parallelises the site loop (benchmarks/compiled_bunny/src/
wih_twos.cpp:1825-1841: `omp parallel for schedule(dynamic, 4)` over sites);
sites are independent given the random stream's key, so the multi-GPU form
splits the sites into contiguous blocks, one per rank, runs each block with
its global site index as the stream's site offset, and gathers the result
rows once at the end.  The gathered rows are therefore identical, bit for
bit, to a one-rank run over all sites.

* `partition(cost, world)` -- contiguous blocks of nearly equal predicted
  cost (walks x predicted steps per site);
* `site_cost(distance, walks, epsilon)` -- the predicted cost of a site
  from its distance to the boundary;
* `gather_rows(local, counts, dist)` -- all ranks' rows in site order (one
  all_gather of fixed-size padded blocks);
* `maxloc(value, index, dist)` -- the (value, index) pair with the largest
  value over all ranks, ties to the smallest index (the design loop's choice);
* `merge_topk(keys, index, k, dist)` -- the global top-k of per-rank top-k
  lists (one all_gather of k pairs per rank), in the order the single-device
  top-k returns them: descending key, ties by ascending index.

Without a process group (`dist is None`) every function is the one-rank
identity, so the same code runs on one GPU.
"""
from __future__ import annotations

import numpy as np


def site_cost(distance, walks, epsilon: float):
    """Predicted cost of each site: walks x expected steps, with the steps of
    a walk-on-spheres path from distance d growing like log(d / epsilon)
    near the boundary plus a constant for the interior."""
    d = np.maximum(np.asarray(distance, dtype=np.float64), epsilon)
    return np.asarray(walks, dtype=np.float64) * (4.0 + np.log(d / epsilon))


def partition(cost, world: int) -> np.ndarray:
    """Boundaries b[0] = 0 <= b[1] <= ... <= b[world] = n of contiguous site
    blocks whose summed costs are as equal as the cut points allow: block r
    is sites [b[r], b[r+1]).  Deterministic, so every rank computes the same
    split from the same inputs."""
    cost = np.asarray(cost, dtype=np.float64)
    n = len(cost)
    if world < 1:
        raise ValueError("world must be >= 1")
    if np.any(cost < 0) or not np.all(np.isfinite(cost)):
        raise ValueError("costs must be finite and non-negative")
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    total = cum[-1]
    bounds = np.zeros(world + 1, dtype=np.int64)
    bounds[-1] = n
    for r in range(1, world):
        # First index whose prefix cost reaches r/world of the total.
        bounds[r] = int(np.searchsorted(cum, total * r / world, side="left"))
    bounds = np.maximum.accumulate(np.clip(bounds, 0, n))
    return bounds


def gather_rows(local: np.ndarray, counts, dist=None, device: str = "cpu") -> np.ndarray:
    """Concatenation, in rank order, of every rank's `local` rows (a numpy
    structured or plain array; counts[r] rows on rank r)."""
    if dist is None:
        return local
    import torch
    counts = [int(c) for c in counts]
    width = local.dtype.itemsize
    cap = max(counts) if counts else 0
    buf = np.zeros(cap * width, dtype=np.uint8)
    raw = np.ascontiguousarray(local).view(np.uint8).reshape(-1)
    buf[:raw.size] = raw
    t = torch.from_numpy(buf).to(device)
    parts = [torch.empty_like(t) for _ in counts]
    dist.all_gather(parts, t)
    out = [p.cpu().numpy()[:c * width] for p, c in zip(parts, counts)]
    return np.concatenate(out).view(local.dtype).reshape((-1,) + local.shape[1:])


def maxloc(value: float, index: int, dist=None, device: str = "cpu"):
    """The (value, index) pair with the largest value over all ranks; equal
    values go to the smallest index.  NaN never wins."""
    if dist is None:
        return float(value), int(index)
    import torch
    v = float(value) if np.isfinite(value) else -np.inf
    t = torch.tensor([v, float(index)], dtype=torch.float64, device=device)
    world = dist.get_world_size()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    pairs = [(float(p[0]), int(p[1])) for p in parts]
    return min(pairs, key=lambda vi: (-vi[0], vi[1]))


def merge_topk(keys, index, k: int, dist=None, device: str = "cpu"):
    """Global top-k (descending key, ties by ascending index) from each
    rank's local top-k (keys, global indices; at most k each, fewer when a
    rank has fewer sites).  Returns (keys, index) of length min(k, total)."""
    keys = np.asarray(keys, dtype=np.float64)
    index = np.asarray(index, dtype=np.int64)
    if dist is not None:
        import torch
        pad = np.full(k, -np.inf)
        pad[:len(keys)] = keys
        ipad = np.full(k, -1, dtype=np.float64)
        ipad[:len(index)] = index
        t = torch.tensor(np.concatenate([pad, ipad]), dtype=torch.float64, device=device)
        parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
        dist.all_gather(parts, t)
        allk, alli = [], []
        for p in parts:
            a = p.cpu().numpy()
            ok = a[k:] >= 0
            allk.append(a[:k][ok])
            alli.append(a[k:][ok].astype(np.int64))
        keys = np.concatenate(allk)
        index = np.concatenate(alli)
    keys = np.where(np.isfinite(keys), keys, -np.inf)
    order = np.lexsort((index, -keys))[:k]
    return keys[order], index[order]
