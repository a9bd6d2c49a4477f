"""Parity at the benchmark's full size (33^3 voxels, L=5, 20 terms), where the oracle would take hours:
the mixed-precision batched solve against the plain FP64 GPU method (itself pinned to the oracle at small
sizes in test_gpu_parity.py) within the north-star bound 1e-5, and size-independent properties --
linearity in the source, a mirror symmetry, the uniform-medium convolution path, the modulated solve."""
import dataclasses

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

N1, L, T = 33, 5, 20


def _phantom(rte):
    return rte.sphere_phantom(N1, nspheres=3, seed=7)[:2]


def _ctx(rte, prec, **kw):
    km = rte.KERNEL_STORE if prec else rte.KERNEL_RECOMPUTE
    return rte.Context(N1, N1, N1, dx=0.1, nL=L, g=0.8, precision=prec, kernel_mode=kw.pop("km", km), **kw)


SRCS = [(0.825, 0.825), (-0.825, 0.825)]


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
