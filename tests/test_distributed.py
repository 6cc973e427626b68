"""Multi-rank plumbing on CPU (gloo, world size 2): disjoint sample ranges,
accumulator merge, max-over-ranks timing."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bluetruthengine_b200 import distributed as D
        base = D.sample_base(rank, frames=5, samples_per_frame=4)
        rng = np.random.default_rng(rank)
        sums = rng.uniform(0, 10, size=(16, 3))
        mean = D.merge_accumulators(sums, samples_this_rank=20).numpy()
        slow = D.max_over_ranks(1.5 + rank)
        q.put((rank, base, mean, slow))
    finally:
        dist.destroy_process_group()


def test_two_rank_merge_and_ranges():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    bases = [o[1] for o in out]
    assert bases == [0, 20]                                  # disjoint sample ranges [0,20), [20,40)
    expect = (np.random.default_rng(0).uniform(0, 10, size=(16, 3)) +
              np.random.default_rng(1).uniform(0, 10, size=(16, 3))) / 40.0
    for o in out:
        assert np.allclose(o[2], expect, rtol=0, atol=1e-12)
        assert o[3] == 2.5
