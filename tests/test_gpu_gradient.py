"""Adjoint gradient of the binned-flux misfit (rte_gradient) against central finite differences of the
loss (step 1e-4 relative, 50 random voxels, for mu_a and mu_s) in FP64, and the mixed-precision gradient
against the FP64 one.  The series is run to convergence (relative L2 stop 1e-13) so the factorised
adjoint is the exact derivative of the discrete model."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _setup(rte, prec, n=7, L=2):
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=21, rmin=0.12, rmax=0.2)
    ctx = rte.Context(n, n, n, dx=0.1, nL=L, g=0.8, precision=prec,
                      kernel_mode=rte.KERNEL_STORE if prec == rte.PREC_MIXED else rte.KERNEL_RECOMPUTE)
    srcs = [rte.Source(pos_x=-0.15, pos_y=0.05), rte.Source(pos_x=0.12, pos_y=-0.1)]
    stop = rte.Stop(rte.STOP_REL_L2, 400, 1e-13)
    det = rte.Detector(nbins=4, faces=63)
    rng = np.random.default_rng(3)
    pa = mua * (1 + 0.05 * rng.standard_normal(mua.size))
    ps = mus * (1 + 0.05 * rng.standard_normal(mus.size))
    ctx.set_medium_voxel(pa, ps)
    target = ctx.detector_flux(srcs, stop, det)
    ctx.set_medium_voxel(mua, mus)
    return ctx, mua, mus, srcs, stop, det, target


def test_gradient_matches_finite_differences(rte):
    ctx, mua, mus, srcs, stop, det, target = _setup(rte, rte.PREC_FP64)
    loss, ga, gs = ctx.gradient(srcs, stop, det, target)

    def L(a, s):
        ctx.set_medium_voxel(a, s)
        return float(np.sum((ctx.detector_flux(srcs, stop, det) - target) ** 2))

    assert abs(L(mua, mus) - loss) < 1e-12 * max(loss, 1e-30)
    rng = np.random.default_rng(9)
    vox = rng.choice(mua.size, 50, replace=False)
    fd_a, fd_s = [], []
    for v in vox:
        for arr, out in ((mua, fd_a), (mus, fd_s)):
            h = 1e-4 * arr[v]
            p = arr.copy()
            p[v] += h
            lp = L(p, mus) if arr is mua else L(mua, p)
            p[v] -= 2 * h
            lm = L(p, mus) if arr is mua else L(mua, p)
            out.append((lp - lm) / (2 * h))
    ctx.set_medium_voxel(mua, mus)
    fd_a, fd_s = np.array(fd_a), np.array(fd_s)
    assert rel(ga[vox], fd_a) < 1e-5, rel(ga[vox], fd_a)
    assert rel(gs[vox], fd_s) < 1e-5, rel(gs[vox], fd_s)
    ctx.close()


def test_gradient_mixed_vs_fp64(rte):
    c64, mua, mus, srcs, stop, det, target = _setup(rte, rte.PREC_FP64)
    _, ga64, gs64 = c64.gradient(srcs, stop, det, target)
    c64.close()
    c32, *_ = _setup(rte, rte.PREC_MIXED)
    _, ga32, gs32 = c32.gradient(srcs, stop, det, target)
    c32.close()
    assert rel(ga32, ga64) < 1e-4 and rel(gs32, gs64) < 1e-4, (rel(ga32, ga64), rel(gs32, gs64))


def test_reconstruct_decreases_misfit(rte):
    """The log-space optimiser on top of the adjoint gradient lowers the flux misfit of a mis-scaled
    medium at every accepted step, several-fold in a few iterations."""
    ctx, mua, mus, srcs, stop, det, _ = _setup(rte, rte.PREC_FP64)
    stop = rte.Stop(rte.STOP_REL_L2, 400, 1e-10)
    target = ctx.detector_flux(srcs, stop, det)  # data of the true medium
    _, _, hist = rte.reconstruct(ctx, srcs, stop, det, target, mua * 1.3, mus * 0.85, iters=6)
    assert all(b <= a for a, b in zip(hist, hist[1:]))
    assert hist[-1] < 0.3 * hist[0], hist
    ctx.close()
