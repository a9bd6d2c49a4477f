"""GPU parity: the CUDA library (through its C ABI) against the FP64 oracle on the same inputs.

Tolerances: FP64 method 1e-11 relative L2 (rounding only); mixed precision 1e-5 relative L2 (the
north-star bound); FIM compat model 1e-6: the oracle's FIM mode walks paths with the reference's float
alpha (kernels.cu:56-60), the library with exact integer crossings, so tau differs by ~1e-7 relative.
"""
import numpy as np
import pytest

from conftest import real_to_complex, rel

pytestmark = pytest.mark.gpu


def _medium(rng, N, hetero=True):
    if not hetero:
        return np.full(N, 0.01), np.full(N, 1.0)
    mua = rng.uniform(0.005, 0.1, N)
    mus = rng.uniform(0.5, 2.0, N)
    return mua, mus


def _ctx(rte, O, nx, ny, nz, L, model, prec, g=0.8, kernel_mode=0, n=1.0, prop=None):
    dx = 0.1
    ctx = rte.Context(nx, ny, nz, dx=dx, nL=L, g=g, n=n, model=model, precision=prec, kernel_mode=kernel_mode,
                      prop_thresh=prop)
    cm = 1.0 / n if model != rte.MODEL_FIM else float(np.float32(1.0 / n))
    p = O.params(nx, ny, nz, dx, dx, dx, L, g, cm, ctx.cfg.prop_thresh, mode=model, ssv=1,
                 x_min=ctx.cfg.x_min, y_min=ctx.cfg.y_min, z_min=ctx.cfg.z_min)
    return ctx, p


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-5)])
@pytest.mark.parametrize("kernel_mode", [1, 2])
def test_prop_abs_exact_hetero(rte, oracle, prec, tol, kernel_mode):
    """kernel_mode 1 stores the pair kernel (FP32 for mixed precision, FP64 for the FP64 method), 2
    recomputes every path integral."""
    rng = np.random.default_rng(1)
    nx, ny, nz, L = 7, 6, 5, 3
    N, C = nx * ny * nz, (L + 1) ** 2
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_EXACT, prec, kernel_mode=kernel_mode)
    mua, mus = _medium(rng, N)
    ctx.set_medium_voxel(mua, mus)
    W = real_to_complex(rng.standard_normal((N, C)), L)
    for flag_scat in (1, 0):
        got = ctx.prop_abs(W, 1, flag_scat)
        ref = oracle.apply(p, mua, mus, W, 1, flag_scat)
        assert rel(got, ref) < tol, (flag_scat, rel(got, ref))
    ctx.close()


def test_prop_abs_general_complex_input(rte, oracle):
    """Input that is not the coefficient set of a real function takes two real solves."""
    rng = np.random.default_rng(2)
    nx, ny, nz, L = 5, 5, 4, 2
    N, C = nx * ny * nz, (L + 1) ** 2
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_EXACT, 0)
    mua, mus = _medium(rng, N)
    ctx.set_medium_voxel(mua, mus)
    W = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
    got = ctx.prop_abs(W, 1, 1)
    ref = oracle.apply(p, mua, mus, W, 1, 1)
    assert rel(got, ref) < 1e-11
    ctx.close()


@pytest.mark.parametrize("kernel_mode", [0, 1])
def test_prop_abs_fim_model(rte, oracle, kernel_mode):
    """FisherInfo_IO discretisation: SH table with the un-wrapped phi index, tissue-0 self term 0,
    g truncated to int in the scatter; FP64 method with the path integrals recomputed (0) or the FP64
    pair kernel stored (1)."""
    rng = np.random.default_rng(3)
    nx, ny, nz, L = 10, 10, 10, 2
    N, C = nx * ny * nz, (L + 1) ** 2
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_FIM, 0, g=0.8, kernel_mode=kernel_mode)
    tiss = rng.integers(0, 3, N).astype(np.uint8)
    mua_t = np.array([0.0, 0.01, 0.05])
    mus_t = np.array([0.0, 1.0, 1.5])
    ctx.set_medium_tissue(tiss, mua_t, mus_t)
    W = real_to_complex(rng.standard_normal((N, C)), L)
    for flag, fs in ((1, 1), (1, 0), (0, 1)):
        got = ctx.prop_abs(W, flag, fs)
        ref = oracle.apply(p, mua_t[tiss], mus_t[tiss], W, flag, fs)
        assert rel(got, ref) < 1e-6, (flag, fs, rel(got, ref))
    ctx.close()


def test_prop_abs_cpu_model(rte, oracle):
    rng = np.random.default_rng(4)
    nx, ny, nz, L = 6, 7, 8, 3
    N, C = nx * ny * nz, (L + 1) ** 2
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_CPU, 0, g=0.8)
    mua, mus = _medium(rng, N, hetero=False)
    ctx.set_medium_voxel(mua, mus)
    W = real_to_complex(rng.standard_normal((N, C)), L)
    got = ctx.prop_abs(W, 1, 1)
    ref = oracle.apply(p, mua, mus, W, 1, 1)
    assert rel(got, ref) < 1e-11
    ctx.close()


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-5)])
def test_forward_exact_spheres(rte, oracle, prec, tol):
    """Whole forward solve (source, 20 terms, final A, images) on a sphere phantom."""
    n, L = 11, 3
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=5, rmin=0.15, rmax=0.3)
    ctx, p = _ctx(rte, oracle, n, n, n, L, rte.MODEL_EXACT, prec)
    ctx.set_medium_voxel(mua, mus)
    src = rte.Source(pos_x=0.0, pos_y=0.0, mag=1.0, kind=rte.SRC_COLUMN)
    res = ctx.forward(src, rte.Stop(rte.STOP_FIXED, 20))
    ref = oracle.forward(p, mua, mus, src_kind=oracle.SRC_COLUMN, img_mode=0, stop_rule=oracle.STOP_FIXED,
                         max_terms=20)
    assert res["terms"] == 20
    assert rel(res["W"], ref["out"]) < tol
    assert rel(res["trans"], ref["trans"]) < tol
    assert rel(res["ref"], ref["ref"]) < tol
    ctx.close()


def test_neumann_reference_stop_rule_fim(rte, oracle):
    """Neumann(W, out, 1) with the reference's lambda rule: same term count, same distribution."""
    nx, ny, nz, L = 10, 10, 20, 2
    N = nx * ny * nz
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_FIM, 0, g=0.8, prop=10.0)
    tiss = np.ones(N, np.uint8)
    ctx.set_medium_tissue(tiss, [0.0, 0.01], [0.0, 1.0])
    src = ctx.source_beam(rte.Source(kind=rte.SRC_FIM))
    mua, mus = np.full(N, 0.01), np.full(N, 1.0)
    ref_src = oracle.source(p, mua, mus, kind=oracle.SRC_FIM)
    assert rel(src, ref_src) < 1e-14
    out, nt = ctx.neumann(src, src, 1, rte.Stop(rte.STOP_REFERENCE))
    ref_out, _, ref_nt = oracle.neumann(p, mua, mus, ref_src, ref_src, 1, oracle.STOP_REFERENCE, n0=2)
    assert nt == ref_nt
    assert rel(out, ref_out) < 1e-6
    tr, rf = ctx.images(out, rte.Source(kind=rte.SRC_FIM))
    otr, orf = oracle.images(p, mua, mus, ref_out, 1)
    assert rel(tr, otr) < 1e-6 and rel(rf, orf) < 1e-6
    ctx.close()


@pytest.mark.parametrize("n,L", [(9, 3), (7, 5), (7, 7)])
def test_forward_batch_matches_single(rte, oracle, n, L):
    """Four sources on one medium in one batched solve == four single solves (mixed precision), and
    each within 1e-5 of the FP64 oracle; L = 5 and 7 take the 32-source-tile kernels of wide rows
    (4 right-hand sides at L = 5, 2 and 4 at L = 7) and, at L = 7, the FP64 SH recurrence."""
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=8, rmin=0.15, rmax=0.25)
    srcs = [rte.Source(pos_x=x, pos_y=y) for x, y in ((-0.2, -0.2), (0.2, -0.2), (-0.2, 0.2), (0.0, 0.0))]
    stop = rte.Stop(rte.STOP_FIXED, 12)
    ctx, p = _ctx(rte, oracle, n, n, n, L, rte.MODEL_EXACT, rte.PREC_MIXED, kernel_mode=rte.KERNEL_STORE)
    ctx.set_medium_voxel(mua, mus)
    single = [ctx.forward(s, stop) for s in srcs]
    rb4 = None
    for nsrc in (4, 3, 2):
        rb = ctx.forward_batch(srcs[:nsrc], stop)
        rb4 = rb if nsrc == 4 else rb4
        for b in range(nsrc):
            assert rel(rb["W"][b], single[b]["W"]) < 1e-6
            assert rel(rb["trans"][b], single[b]["trans"]) < 1e-6 and rel(rb["ref"][b], single[b]["ref"]) < 1e-6
    for b, s in enumerate(srcs):
        ref = oracle.forward(p, mua, mus, src_kind=oracle.SRC_COLUMN, img_mode=0, stop_rule=oracle.STOP_FIXED,
                             max_terms=12, pos_x=s.pos_x, pos_y=s.pos_y)
        assert rel(rb4["W"][b], ref["out"]) < 1e-5
        assert rel(rb4["trans"][b], ref["trans"]) < 1e-5
    # preallocated result arrays (as pinned host buffers are passed) are written in place
    out = {"W": np.full_like(rb4["W"], np.nan), "trans": np.full_like(rb4["trans"], np.nan),
           "ref": np.full_like(rb4["ref"], np.nan)}
    rb = ctx.forward_batch(srcs, stop, out=out)
    assert rb["W"] is out["W"] and rb["trans"] is out["trans"]
    assert rel(out["W"], rb4["W"]) < 1e-12 and rel(out["ref"], rb4["ref"]) < 1e-12
    ctx.close()


@pytest.mark.parametrize("n,L", [(7, 6), (7, 7), (11, 6)])
def test_forward_batch_recomputed_high_order(rte, oracle, n, L):
    """Four sources, path integrals recomputed, L >= 6: the kernel whose two thread groups share each
    pair's walk (k_pair_mixed_grp) against four single solves (1e-6) and the FP64 oracle (1e-5); 11^3
    has 1331 voxels, more than one 1024-source chunk, so the FP32 chunk sums meet in the epilogue."""
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=5, rmin=0.15, rmax=0.25)
    srcs = [rte.Source(pos_x=x, pos_y=y) for x, y in ((-0.2, -0.2), (0.2, -0.2), (-0.2, 0.2), (0.0, 0.0))]
    stop = rte.Stop(rte.STOP_FIXED, 8)
    ctx, p = _ctx(rte, oracle, n, n, n, L, rte.MODEL_EXACT, rte.PREC_MIXED, kernel_mode=rte.KERNEL_RECOMPUTE)
    ctx.set_medium_voxel(mua, mus)
    rb = ctx.forward_batch(srcs, stop)
    for b, s in enumerate(srcs):
        single = ctx.forward(s, stop)
        assert rel(rb["W"][b], single["W"]) < 1e-6, (b, rel(rb["W"][b], single["W"]))
        ref = oracle.forward(p, mua, mus, src_kind=oracle.SRC_COLUMN, img_mode=0, stop_rule=oracle.STOP_FIXED,
                             max_terms=8, pos_x=s.pos_x, pos_y=s.pos_y)
        assert rel(rb["W"][b], ref["out"]) < 1e-5, (b, rel(rb["W"][b], ref["out"]))
        assert rel(rb["trans"][b], ref["trans"]) < 1e-5
    ctx.close()


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-9)])
def test_uniform_medium_convolution_path(rte, oracle, prec, tol):
    """A uniform medium in automatic kernel mode runs the operator as an FFT convolution: the same
    forward solve as the oracle and as the pair kernels (RTE_KERNEL_RECOMPUTE), single and batched."""
    nx, ny, nz, L = 9, 8, 7, 3
    N = nx * ny * nz
    mua, mus = np.full(N, 0.02), np.full(N, 1.3)
    stop = rte.Stop(rte.STOP_FIXED, 12)
    ctx, p = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_EXACT, prec, kernel_mode=rte.KERNEL_AUTO)
    ctx.set_medium_voxel(mua, mus)
    srcs = [rte.Source(pos_x=0.05, pos_y=-0.1), rte.Source(pos_x=-0.2, pos_y=0.1)]
    res = ctx.forward(srcs[0], stop)
    ref = oracle.forward(p, mua, mus, src_kind=oracle.SRC_COLUMN, img_mode=0, stop_rule=oracle.STOP_FIXED, max_terms=12,
                         pos_x=0.05, pos_y=-0.1)
    assert rel(res["W"], ref["out"]) < tol and rel(res["trans"], ref["trans"]) < tol
    W = real_to_complex(np.random.default_rng(4).standard_normal((N, (L + 1) ** 2)), L)
    assert rel(ctx.prop_abs(W, 1, 1), oracle.apply(p, mua, mus, W, 1, 1)) < tol
    assert rel(ctx.prop_abs(W, 0, 1), oracle.apply(p, mua, mus, W, 0, 1)) < tol
    if prec == 1:
        rb = ctx.forward_batch(srcs, stop)
        assert rel(rb["W"][0], res["W"]) < 1e-9
    ctx.close()
    pair, _ = _ctx(rte, oracle, nx, ny, nz, L, rte.MODEL_EXACT, 0, kernel_mode=rte.KERNEL_RECOMPUTE)
    pair.set_medium_voxel(mua, mus)
    assert rel(pair.forward(srcs[0], stop)["W"], res["W"]) < max(tol, 1e-12)
    pair.close()


@pytest.mark.parametrize("model", [0, 1, 2])
@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-6)])
def test_prop_abs_adjoint_is_the_transpose(rte, model, prec, tol):
    """rte_prop_abs_adjoint against the inner-product identity <y, A x> = <A^H y, x> on random complex
    inputs, for the exact, table (FisherInfo_IO: transposed pair kernels, since snapping directions to its
    table does not commute with negation) and CPU-package models.  The grid is even, so displacements with
    zero components (where the table's unwrapped phi depends on the sign of zero) are present."""
    rng = np.random.default_rng(12)
    n, L = 6, 2
    N, C = n ** 3, (L + 1) ** 2
    ctx = rte.Context(n, n, n, dx=0.1, nL=L, g=0.8, model=model, precision=prec,
                      kernel_mode=rte.KERNEL_STORE if prec else rte.KERNEL_RECOMPUTE)
    mua, mus = _medium(rng, N)
    ctx.set_medium_voxel(mua, mus)
    for _ in range(3):
        x = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
        y = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
        lhs = np.vdot(y, ctx.prop_abs(x, 1, 0))
        rhs = np.vdot(ctx.prop_abs_adjoint(y, 1), x)
        assert abs(lhs - rhs) <= tol * abs(lhs), (model, prec, lhs, rhs)
    ctx.close()
