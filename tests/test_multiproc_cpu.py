"""Multi-rank host logic on CPU (gloo, world size 2).

* The bench's max-over-ranks device-time reduction and per-rank replica
  seeds (the replica mode).
* Site sharding (twos_b200.shard): the contiguous cost-weighted partition is
  disjoint and complete; each rank estimates its block with its global site
  indices as the stream's site offset (here the oracle in the GPU's counter
  stream stands in for the device, where each rank would call its own GPU),
  the rows are gathered once, and the gathered rows equal the
  one-rank rows bit for bit; the design loop's maxloc and the top-k merge of
  per-rank shortlists equal the single-array answers.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    return dist


def _run(fn, world=2):
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(fn, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        return dict(out)


def _replica_worker(rank, world, port, out):
    dist = _init(rank, world, port)
    import bench
    out[rank] = (bench.max_over_ranks(10.0 * (rank + 1), dist, "cpu"), bench.replica_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_seeds():
    res = _run(_replica_worker)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] != res[1][1]


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5


def _problem():
    import sys
    from conftest import PKG
    sys.path.insert(0, str(PKG))
    from twos_b200 import geometry
    V, F = geometry.icosphere(2)
    sites = geometry.uniform_ball(37, 0.8, seed=3)
    return V, F, sites


def _estimate(oracle, V, F, sites, ids):
    # The GPU's counter stream keyed by the global site index.
    return oracle.OracleMesh(V, F).estimate(sites, site_ids=ids, rng=oracle.RNG_COUNTER, walks=24, seed=9,
                                            epsilon=1e-3, max_steps=512,
                                            source=[oracle.term(oracle.TERM_CONST, 1.0)], threads=1)


def _rows(est):
    dt = np.dtype([("u", "f8"), ("score", "f8"), ("score_se", "f8"), ("steps", "u8")])
    r = np.zeros(len(est["u"]), dtype=dt)
    for k in dt.names:
        r[k] = est[k]
    return r


def _shard_worker(rank, world, port, out):
    dist = _init(rank, world, port)
    import oracle
    from twos_b200 import shard
    V, F, sites = _problem()
    d = np.linalg.norm(sites, axis=1)  # any per-site distance proxy: both ranks compute the same split
    b = shard.partition(shard.site_cost(1.0 - d, 24, 1e-3), world)
    lo, hi = int(b[rank]), int(b[rank + 1])
    ids = np.arange(lo, hi)
    rows = _rows(_estimate(oracle, V, F, sites[lo:hi], ids))
    gathered = shard.gather_rows(rows, np.diff(b), dist)
    # Design-loop reductions over the shard: best lower bound and a top-5 shortlist.
    lower = rows["score"] - 1.96 * rows["score_se"]
    j = int(np.argmax(lower)) if len(lower) else 0
    best = shard.maxloc(lower[j] if len(lower) else -np.inf, lo + j, dist)
    order = np.lexsort((ids, -rows["score"]))[:5]
    topk = shard.merge_topk(rows["score"][order], ids[order], 5, dist)
    out[rank] = (b.tolist(), gathered.tobytes(), best, topk[0].tolist(), topk[1].tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_site_sharding_equals_one_rank_bit_for_bit(oracle_mod):
    res = _run(_shard_worker)
    V, F, sites = _problem()
    full = _rows(_estimate(oracle_mod, V, F, sites, np.arange(len(sites))))
    b = res[0][0]
    assert b == res[1][0] and b[0] == 0 and b[-1] == len(sites) and b[0] < b[1] < b[2]
    for r in (0, 1):
        assert res[r][1] == full.tobytes()
    lower = full["score"] - 1.96 * full["score_se"]
    assert res[0][2] == res[1][2] == (float(np.max(lower)), int(np.argmax(lower)))
    order = np.lexsort((np.arange(len(full)), -full["score"]))[:5]
    for r in (0, 1):
        assert res[r][4] == order.tolist()
        assert res[r][3] == full["score"][order].tolist()


def test_partition_is_contiguous_balanced_and_complete():
    from twos_b200 import shard
    rng = np.random.default_rng(0)
    cost = rng.lognormal(size=1000)
    for world in (1, 2, 3, 8):
        b = shard.partition(cost, world)
        assert b[0] == 0 and b[-1] == 1000 and np.all(np.diff(b) >= 0) and len(b) == world + 1
        per = [cost[b[r]:b[r + 1]].sum() for r in range(world)]
        assert max(per) <= cost.sum() / world + cost.max()
    assert shard.partition(np.ones(3), 8).tolist()[-1] == 3
    with pytest.raises(ValueError):
        shard.partition([1.0, -1.0], 2)


def test_one_rank_identities():
    from twos_b200 import shard
    assert shard.maxloc(2.5, 7) == (2.5, 7)
    k, i = shard.merge_topk([3.0, 5.0, 5.0, np.nan], [4, 9, 2, 1], 3)
    assert k.tolist() == [5.0, 5.0, 3.0] and i.tolist() == [2, 9, 4]
