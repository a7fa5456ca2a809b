"""Sharding of a batch across ranks (CPU, gloo, world size 2).

The GPU walk is replaced here by the CPU oracle -- this test covers the
host-side partition and the end-of-run gather, which are the only multi-GPU
parts of the path (trajectories are independent; no data-path collective).
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from cmfw import shard

RES_DTYPE = oracle.OUT_F64_DTYPE


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        recs = oracle.make_inputs(3, 2, 900, 0, False)[:300]
        lo, hi = shard.shard_bounds(len(recs), rank, world)
        out = oracle.walk("f64", 3, 2, 0.5, 300, 30, recs[lo:hi], threads=1)
        full = np.zeros(hi - lo, dtype=RES_DTYPE.descr + [("index", "<i8")])
        for k in RES_DTYPE.names:
            full[k] = out[k]
        full["index"] = np.arange(lo, hi)
        s = shard.summarize(full, verified=out["valid"] == 1, top_k=5)
        merged = shard.gather_merge(s, top_k=5)
        q.put((rank, merged))
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_exactly():
    for n in (0, 1, 7, 10000):
        for world in (1, 2, 3, 8):
            parts = [shard.shard_bounds(n, r, world) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(parts, parts[1:]))
            sizes = [h - l for l, h in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard.shard_bounds(10, 2, 2)


def test_two_rank_gather_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    recs = oracle.make_inputs(3, 2, 900, 0, False)[:300]
    out = oracle.walk("f64", 3, 2, 0.5, 300, 30, recs, threads=1)
    full = np.zeros(len(out), dtype=RES_DTYPE.descr + [("index", "<i8")])
    for k in RES_DTYPE.names:
        full[k] = out[k]
    full["index"] = np.arange(len(out))
    want = shard.merge([shard.summarize(full, verified=out["valid"] == 1, top_k=5)], top_k=5)
    assert got[0] == got[1] == want
