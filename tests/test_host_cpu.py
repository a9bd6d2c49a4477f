"""Host-side logic without a GPU: phantoms, the algorithmic operation counts used by the roofline,
and the multi-process (replica) timing reduction of bench.py under a 2-rank gloo group."""
import os
import socket

import numpy as np
import pytest


def test_sphere_phantom_seeded():
    from doi_b200.phantoms import sphere_phantom
    a1, s1, sp1 = sphere_phantom(17, seed=3)
    a2, s2, sp2 = sphere_phantom(17, seed=3)
    a3, _, _ = sphere_phantom(17, seed=4)
    assert np.array_equal(a1, a2) and np.array_equal(s1, s2) and sp1 == sp2
    assert not np.array_equal(a1, a3)
    assert a1.size == 17 ** 3
    # at most background + 3 inclusion values
    assert len(np.unique(a1)) <= 4 and np.isclose(a1.min(), 0.01)
    for sph in sp1:
        assert 0.2 <= sph["r"] <= 0.6 and 2 * 0.01 <= sph["mua"] <= 10 * 0.01 and 0.5 <= sph["mus"] <= 2.0


def test_algorithmic_counts_brute_force():
    import bench
    for n in (3, 4, 5):
        c = bench.algorithmic_counts(n, 2)
        idx = np.array([(i, j, k) for i in range(n) for j in range(n) for k in range(n)])
        d = np.abs(idx[:, None, :] - idx[None, :, :]).sum(-1)
        assert c["pairs"] == n ** 3 * (n ** 3 - 1)
        assert c["steps"] == d.sum()


def _worker(rank, world, port, vals, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    m = bench.max_over_ranks(vals[rank])
    q.put((rank, m, bench.throughput(world, 5, m)))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_reduction_gloo():
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    vals = [120.0, 135.5]
    ps = [ctx.Process(target=_worker, args=(r, 2, port, vals, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, m, thr in res:
        assert m == 135.5
        assert abs(thr - 2 * 5 / 0.1355) < 1e-9
