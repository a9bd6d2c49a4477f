"""Parity at the benchmark's full size (33^3 voxels, L=5, 20 terms).  One operator application is checked
against the FP64 oracle on sampled destination voxels (a whole 20-term solve would take the oracle about an
hour); the mixed-precision batched solve against the plain FP64 GPU method (itself pinned to the oracle at
small sizes in test_gpu_parity.py) within the north-star bound 1e-5; and size-independent properties --
linearity in the source, a mirror symmetry, the uniform-medium convolution path, the modulated solve."""
import dataclasses

import numpy as np
import pytest

from conftest import real_to_complex, rel

pytestmark = pytest.mark.gpu

N1, L, T = 33, 5, 20


def _phantom(rte):
    return rte.sphere_phantom(N1, nspheres=3, seed=7)[:2]


def _ctx(rte, prec, **kw):
    km = rte.KERNEL_STORE if prec else rte.KERNEL_RECOMPUTE
    return rte.Context(N1, N1, N1, dx=0.1, nL=L, g=0.8, precision=prec, kernel_mode=kw.pop("km", km), **kw)


SRCS = [(0.825, 0.825), (-0.825, 0.825)]


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-5)])
def test_operator_matches_oracle_at_benchmark_size(rte, oracle, prec, tol):
    """One application D A W at the benchmark's size (33^3, L=5, the 3-sphere phantom of bench.py's
    first timed step) against the FP64 oracle on 512 seeded destination voxels x all 35,937 sources.
    The input is the collimated source plus a dense random real function, so every pair and every
    coefficient carries work.  FP64 method <= 1e-11, mixed precision <= 1e-5 (relative L2 over the
    sampled rows)."""
    mua, mus, _ = rte.sphere_phantom(N1, dx=0.1, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=3)
    N, C = N1 ** 3, (L + 1) ** 2
    rng = np.random.default_rng(11)
    with _ctx(rte, prec) as ctx:
        ctx.set_medium_voxel(mua, mus)
        W = ctx.source_beam(rte.Source(kind=rte.SRC_COLUMN))
        W = W + 1e-3 * real_to_complex(rng.standard_normal((N, C)), L)
        got = ctx.prop_abs(W, 1, 1)
        p = oracle.params(N1, N1, N1, 0.1, 0.1, 0.1, L, 0.8, 1.0, ctx.cfg.prop_thresh, mode=oracle.MODE_EXACT)
    dests = np.sort(rng.choice(N, 512, replace=False))
    ref = oracle.apply_subset(p, mua, mus, W, dests, 1, 1)
    err = rel(got[dests], ref[dests])
    assert err < tol, err


def test_mixed_batched_matches_fp64_method(rte):
    mua, mus = _phantom(rte)
    stop = rte.Stop(rte.STOP_FIXED, T)
    srcs = [rte.Source(pos_x=x, pos_y=y, kind=rte.SRC_COLUMN) for x, y in SRCS]
    with _ctx(rte, 1) as mx:
        mx.set_medium_voxel(mua, mus)
        rb = mx.forward_batch(srcs, stop)
    with _ctx(rte, 0) as fp:
        fp.set_medium_voxel(mua, mus)
        for b, s in enumerate(srcs):
            ref = fp.forward(s, stop)
            assert rel(rb["W"][b], ref["W"]) < 1e-5
            assert rel(rb["trans"][b], ref["trans"]) < 1e-5 and rel(rb["ref"][b], ref["ref"]) < 1e-5


def test_linearity_in_the_source(rte):
    """Doubling the beam magnitude doubles every output (a power of two: exact in both precisions)."""
    mua, mus = _phantom(rte)
    stop = rte.Stop(rte.STOP_FIXED, T)
    s1 = rte.Source(kind=rte.SRC_COLUMN, mag=1.0)
    with _ctx(rte, 1) as ctx:
        ctx.set_medium_voxel(mua, mus)
        a = ctx.forward(s1, stop)
        b = ctx.forward(dataclasses.replace(s1, mag=2.0), stop)
    for k in ("W", "trans", "ref"):
        assert rel(b[k], 2.0 * a[k]) < 1e-14, k


def test_mirror_symmetry(rte):
    """A beam entering the z = nZ-1 face of a medium equals the z = 0 beam in the z-mirrored medium,
    with transmission and reflection exchanged."""
    mua, mus = _phantom(rte)
    A = lambda v: v.reshape(N1, N1, N1)
    stop = rte.Stop(rte.STOP_FIXED, T)
    with _ctx(rte, 1) as ctx:
        ctx.set_medium_voxel(mua, mus)
        top = ctx.forward(rte.Source(kind=rte.SRC_BEAM, face=1), stop)
        ctx.set_medium_voxel(np.ascontiguousarray(A(mua)[::-1]).ravel(), np.ascontiguousarray(A(mus)[::-1]).ravel())
        bot = ctx.forward(rte.Source(kind=rte.SRC_BEAM, face=0), stop)
    flux = lambda W: W[:, 0].real.reshape(N1, N1, N1)
    assert rel(flux(top["W"])[::-1], flux(bot["W"])) < 2e-5
    assert rel(top["trans"], bot["ref"]) < 2e-5 and rel(top["ref"], bot["trans"]) < 2e-5


def test_uniform_medium_convolution_at_full_size(rte):
    N = N1 ** 3
    stop = rte.Stop(rte.STOP_FIXED, T)
    src = rte.Source(kind=rte.SRC_COLUMN)
    with _ctx(rte, 1, km=rte.KERNEL_AUTO) as ctx:
        ctx.set_medium_voxel(np.full(N, 0.01), np.full(N, 1.0))
        fft = ctx.forward(src, stop)
    with _ctx(rte, 0) as fp:
        fp.set_medium_voxel(np.full(N, 0.01), np.full(N, 1.0))
        ref = fp.forward(src, stop)
    for k in ("W", "trans", "ref"):
        assert rel(fft[k], ref[k]) < 1e-11, k


def test_modulated_mixed_matches_fp64_method(rte):
    mua, mus = _phantom(rte)
    stop = rte.Stop(rte.STOP_FIXED, T)
    src = rte.Source(kind=rte.SRC_COLUMN, modulation=0.7)
    with _ctx(rte, 1) as mx:
        mx.set_medium_voxel(mua, mus)
        a = mx.forward(src, stop)
    with _ctx(rte, 0) as fp:
        fp.set_medium_voxel(mua, mus)
        b = fp.forward(src, stop)
    for k in ("W", "trans", "ref"):
        assert rel(a[k], b[k]) < 1e-5, k
    assert np.abs(np.angle(a["trans"])).max() > 1e-3


def _config4(rte, prec, terms):
    """the 33^3 L=5 phantom of bench.py's gradient measurement (3 spheres, seed 4), 4
    collimated z=0 sources at (+-0.825, +-0.825) cm, 8x8 bins on each of the 6 faces, target flux from the
    phantom with every inclusion's coefficients scaled by (1 + 0.05 N(0,1))."""
    mua, mus, sph = rte.sphere_phantom(N1, dx=0.1, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=4)
    rng = np.random.default_rng(44)
    pa, ps = mua.copy(), mus.copy()
    for sp in sph:
        ka, ks = 1 + 0.05 * rng.standard_normal(2)
        pa[mua == sp["mua"]] *= ka
        ps[mus == sp["mus"]] *= ks
    ctx = rte.Context(N1, N1, N1, dx=0.1, nL=L, g=0.8, precision=prec, kernel_mode=rte.KERNEL_STORE)
    srcs = [rte.Source(pos_x=x, pos_y=y, kind=rte.SRC_COLUMN) for x, y in
            ((-0.825, -0.825), (0.825, -0.825), (-0.825, 0.825), (0.825, 0.825))]
    stop = rte.Stop(rte.STOP_FIXED, terms)
    det = rte.Detector(nbins=8, faces=63)
    ctx.set_medium_voxel(pa, ps)
    target = ctx.detector_flux(srcs, stop, det)
    ctx.set_medium_voxel(mua, mus)
    return ctx, mua, mus, srcs, stop, det, target


def test_gradient_finite_differences_at_config4_size(rte):
    """The adjoint gradient at config 4's size in FP64 (stored FP64 pair kernel) against central finite
    differences on 10 seeded voxels for mu_a and 10 for mu_s, tolerance 1e-5.  Every evaluation takes 40
    terms (the series has converged to ~1e-12 there, so the factorised adjoint is the derivative of the
    40-term model to that level, and FD evaluations never differ in their term count).  Steps are 1e-4
    relative to the voxel's mu_t for both coefficients: a single voxel moves the loss by ~1e-7 relative per
    1e-4 of mu_t, and mu_a is 1% of mu_t, so a step relative to mu_a alone leaves a loss difference only
    ~1e4 times the FP64 rounding of the loss (measured: 1.03e-5 relative FD error for mu_a at that step,
    5.7e-9 for mu_s)."""
    ctx, mua, mus, srcs, stop, det, target = _config4(rte, rte.PREC_FP64, 40)
    loss, ga, gs = ctx.gradient(srcs, stop, det, target)

    def Lf(a, s):
        ctx.set_medium_voxel(a, s)
        return float(np.sum((ctx.detector_flux(srcs, stop, det) - target) ** 2))

    assert abs(Lf(mua, mus) - loss) < 1e-12 * loss
    rng = np.random.default_rng(10)
    va, vs = rng.choice(mua.size, 10, replace=False), rng.choice(mua.size, 10, replace=False)
    fd = {"a": [], "s": []}
    for key, arr, vox in (("a", mua, va), ("s", mus, vs)):
        for v in vox:
            h = 1e-4 * (mua[v] + mus[v])
            p = arr.copy()
            p[v] += h
            lp = Lf(p, mus) if key == "a" else Lf(mua, p)
            p[v] -= 2 * h
            lm = Lf(p, mus) if key == "a" else Lf(mua, p)
            fd[key].append((lp - lm) / (2 * h))
    ctx.close()
    ea, es = rel(ga[va], np.array(fd["a"])), rel(gs[vs], np.array(fd["s"]))
    assert ea < 1e-5 and es < 1e-5, (ea, es)


def test_gradient_mixed_vs_fp64_at_config4_size(rte):
    """The mixed-precision gradient of config 4 (20 terms, as bench.py times it) within 1e-5 of the FP64
    method's on the same 20-term model."""
    out = {}
    for prec in (rte.PREC_FP64, rte.PREC_MIXED):
        ctx, mua, mus, srcs, stop, det, target = _config4(rte, prec, T)
        out[prec] = ctx.gradient(srcs, stop, det, target)
        ctx.close()
    a, b = out[rte.PREC_MIXED], out[rte.PREC_FP64]
    assert abs(a[0] - b[0]) < 1e-5 * b[0]
    assert rel(a[1], b[1]) < 1e-5 and rel(a[2], b[2]) < 1e-5, (rel(a[1], b[1]), rel(a[2], b[2]))
