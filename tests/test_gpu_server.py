"""The continuous-batching server (rte_server_*) on the GPU: every result is the same alone and in
a mix of grids, orders, media and source counts running concurrently; cancellation, admission
failure for a request larger than the HBM budget, and the latency statistics."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

DX = 0.1


def _request(rte, rng, n, L, nsrc):
    mua, mus, _ = rte.sphere_phantom(n, nspheres=int(rng.integers(0, 4)), seed=int(rng.integers(1 << 30)),
                                     rmin=0.1, rmax=0.25)
    srcs = []
    for _ in range(nsrc):
        f = int(rng.integers(0, 6))
        kind = rte.SRC_POINT if rng.random() < 0.5 else rte.SRC_BEAM
        a, b = (float(v) for v in rng.uniform(-0.3, 0.3, 2) * n * DX)
        srcs.append(rte.Source(pos_x=a, pos_y=b, pos_z=n * DX / 2 + a / 2, kind=kind, face=f))
    return mua, mus, srcs


def _alone(rte, n, L, prec, mua, mus, srcs, terms):
    ctx = rte.Context(n, n, n, dx=DX, nL=L, g=0.8, precision=prec, prop_thresh=4.0 * n * DX,
                      kernel_mode=rte.KERNEL_AUTO)
    ctx.set_medium_voxel(mua, mus)
    tr, rf, _ = ctx.forward_graph(srcs, terms)
    ctx.close()
    return tr, rf


def test_mix_equals_alone(rte):
    rng = np.random.default_rng(7)
    shapes = [(9, 3, 1, 1), (11, 2, 2, 1), (9, 3, 4, 1), (13, 3, 3, 1), (9, 3, 2, 0), (11, 2, 1, 1),
              (9, 3, 1, 1), (13, 3, 2, 1)]
    terms = 8
    reqs = [(n, L, prec) + _request(rte, rng, n, L, nsrc) for n, L, nsrc, prec in shapes]
    with rte.Server(workers=3) as srv:
        tickets = [srv.submit(mua, mus, srcs, n, dx=DX, nL=L, precision=prec, terms=terms)
                   for n, L, prec, mua, mus, srcs in reqs]
        results = [srv.wait(t, timeout=300) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    for (n, L, prec, mua, mus, srcs), (tr, rf, info) in zip(reqs, results):
        assert info["status"] == 0 and info["latency_ms"] >= info["service_ms"] > 0
        atr, arf = _alone(rte, n, L, prec, mua, mus, srcs, terms)
        assert rel(tr, atr) < 1e-12 and rel(rf, arf) < 1e-12, (n, L, len(srcs))


def test_context_reuse_with_new_medium(rte):
    """One worker: the second request of a shape reuses the first one's context and graph."""
    rng = np.random.default_rng(8)
    reqs = [_request(rte, rng, 9, 3, 2) for _ in range(3)]
    with rte.Server(workers=1) as srv:
        tickets = [srv.submit(mua, mus, srcs, 9, dx=DX, nL=3, terms=6) for mua, mus, srcs in reqs]
        results = [srv.wait(t) for t in tickets]
        assert srv.stats()["contexts"] == 1
    for (mua, mus, srcs), (tr, rf, _) in zip(reqs, results):
        atr, arf = _alone(rte, 9, 3, 1, mua, mus, srcs, 6)
        assert rel(tr, atr) < 1e-12 and rel(rf, arf) < 1e-12


def test_budget_and_cancel(rte):
    rng = np.random.default_rng(9)
    with rte.Server(workers=1, hbm_budget_gb=0.2) as srv:
        mua, mus, srcs = _request(rte, rng, 41, 5, 1)  # the stored 41^3 x 41^3 kernel alone is 19 GB
        big = srv.submit(mua, mus, srcs, 41, dx=DX, nL=5, terms=4)
        with pytest.raises(rte.RteError):
            srv.wait(big, timeout=60)
        small = [srv.submit(*_request(rte, rng, 9, 2, 1)[:3], 9, dx=DX, nL=2, terms=4) for _ in range(4)]
        cancelled = [srv.cancel(t) for t in small[1:]]
        for t, c in zip(small[1:], cancelled):
            if c:
                with pytest.raises(rte.RteError):
                    srv.wait(t)
            else:
                srv.wait(t)
        srv.wait(small[0])
        st = srv.stats()
    assert st["failed"] == 1 and st["cancelled"] == sum(cancelled)
    assert st["completed"] == 4 - sum(cancelled)


def test_orders_run_concurrently(rte):
    """Requests of orders 3, 5 and 7 on 17^3 grids (large enough for the launch autotuner) from four
    workers at once: the lower-order passes of a pair kernel size their shared memory by the context's
    order, so contexts of different orders configure the same kernels concurrently.  Every request
    completes and equals the same request alone (1e-6, mixed precision)."""
    rng = np.random.default_rng(11)
    n, terms = 17, 4
    reqs = [(Lq,) + _request(rte, rng, n, Lq, 1) for Lq in (3, 5, 7, 3, 5, 7, 5, 3)]
    with rte.Server(workers=4) as srv:
        tickets = [srv.submit(mua, mus, srcs, n, dx=DX, nL=Lq, terms=terms) for Lq, mua, mus, srcs in reqs]
        outs = [srv.wait(t, timeout=600) for t in tickets]
    for (Lq, mua, mus, srcs), (tr, rf, info) in zip(reqs, outs):
        tr0, rf0 = _alone(rte, n, Lq, rte.PREC_MIXED, mua, mus, srcs, terms)
        assert rel(tr, tr0) < 1e-6 and rel(rf, rf0) < 1e-6, (Lq, rel(tr, tr0), rel(rf, rf0))
