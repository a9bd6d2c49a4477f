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


class _LinearFluxContext:
    """Stand-in for Context with a linear detector model flux = M [mu_a; mu_s] (host only), enough to
    drive the optimiser loop of doi_b200.inverse.reconstruct without a GPU."""

    def __init__(self, M):
        self.M = M
        self.n = M.shape[1] // 2
        self.mua = self.mus = None
        self.gradient_calls = 0

    def set_medium_voxel(self, mua, mus):
        self.mua, self.mus = np.array(mua), np.array(mus)

    def detector_flux(self, srcs, stop, det):
        return self.M @ np.concatenate([self.mua, self.mus])

    def gradient(self, srcs, stop, det, target):
        self.gradient_calls += 1
        r = self.detector_flux(srcs, stop, det) - target
        g = 2.0 * self.M.T @ r
        return float(r @ r), g[:self.n], g[self.n:]


@pytest.mark.parametrize("fit_mus", [True, False])
def test_reconstruct_host_loop(fit_mus):
    """Log-space steps keep the coefficients positive, every accepted step lowers the misfit (Armijo),
    fit_mus=False leaves mu_s untouched, and the context ends on the returned medium."""
    from doi_b200.inverse import reconstruct
    rng = np.random.default_rng(11)
    n = 12
    M = rng.uniform(0.0, 1.0, (30, 2 * n))
    mua_t, mus_t = rng.uniform(0.01, 0.05, n), rng.uniform(0.8, 1.2, n)
    ctx = _LinearFluxContext(M)
    target = M @ np.concatenate([mua_t, mus_t])
    mua0, mus0 = mua_t * 1.5, mus_t * (0.9 if fit_mus else 1.0)
    mua, mus, hist = reconstruct(ctx, None, None, None, target, mua0, mus0, iters=15, fit_mus=fit_mus)
    assert len(hist) >= 2 and hist[-1] < 0.5 * hist[0]
    assert all(b <= a for a, b in zip(hist, hist[1:]))
    assert (mua > 0).all() and (mus > 0).all()
    if not fit_mus:
        assert np.array_equal(mus, mus0)
    assert np.array_equal(ctx.mua, mua) and np.array_equal(ctx.mus, mus)


def test_reconstruct_reverts_when_no_step_is_accepted():
    """A fixed step far too large for every backtrack: the loop stops and the context is left on the
    last accepted medium (the start)."""
    from doi_b200.inverse import reconstruct
    rng = np.random.default_rng(5)
    n = 6
    M = rng.uniform(0.0, 1.0, (10, 2 * n))
    ctx = _LinearFluxContext(M)
    mua0, mus0 = np.full(n, 0.02), np.full(n, 1.0)
    target = M @ np.concatenate([mua0 * 0.5, mus0])
    mua, mus, hist = reconstruct(ctx, None, None, None, target, mua0, mus0, iters=3, step=1e6, max_backtrack=2)
    assert hist == hist[:1]
    assert np.array_equal(mua, mua0) and np.array_equal(ctx.mua, mua0) and np.array_equal(ctx.mus, mus0)
