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


@pytest.mark.parametrize("L", [2, 7])
def test_gradient_mixed_vs_fp64(rte, L):
    """At L = 7 the back-projection keeps the destination rows in shared memory and runs the SH
    recurrence in FP64."""
    c64, mua, mus, srcs, stop, det, target = _setup(rte, rte.PREC_FP64, L=L)
    _, ga64, gs64 = c64.gradient(srcs, stop, det, target)
    c64.close()
    c32, *_ = _setup(rte, rte.PREC_MIXED, L=L)
    _, ga32, gs32 = c32.gradient(srcs, stop, det, target)
    c32.close()
    assert rel(ga32, ga64) < 1e-5 and rel(gs32, gs64) < 1e-5, (rel(ga32, ga64), rel(gs32, gs64))


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


def _image_problem(rte, prec, n=9, L=2, ntis=3, model=None, image=0):
    """A sphere phantom given as a tissue map (types 1..ntis-1 in the inclusions), a collimated z = 0 beam and
    the transmission (image 0) or reflection (1) image of a perturbed medium as the measured image g."""
    mua, mus, sph = rte.sphere_phantom(n, nspheres=ntis - 2, seed=31, rmin=0.15, rmax=0.25)
    tiss = np.ones(n ** 3, np.uint8)
    for t, sp in enumerate(sph, start=2):
        tiss[(mua == sp["mua"]) & (mus == sp["mus"])] = t
    assert all((tiss == t).any() for t in range(1, ntis))
    ctx = rte.Context(n, n, n, dx=0.1, nL=L, g=0.8, precision=prec, model=rte.MODEL_EXACT if model is None else model,
                      kernel_mode=rte.KERNEL_STORE if prec == rte.PREC_MIXED else rte.KERNEL_RECOMPUTE)
    src = rte.Source(pos_x=0.05, pos_y=-0.05, kind=rte.SRC_COLUMN)
    rng = np.random.default_rng(5)
    ctx.set_medium_voxel(mua * (1 + 0.1 * rng.standard_normal(mua.size)), mus * (1 + 0.1 * rng.standard_normal(mus.size)))
    r = ctx.forward(src, rte.Stop(rte.STOP_FIXED, 12))
    ctx.set_medium_voxel(mua, mus)
    if image == 1:
        return ctx, mua, mus, tiss, src, r["ref"].real.ravel()
    return ctx, mua, mus, tiss, src, r["trans"].real.ravel()


def test_image_gradient_reference_model_matches_region_tangents(rte):
    """The adjoint form of the reference's tangent gradient (compute_grad_rte.cu:273-385): av times the sum of
    the per-voxel gradient over each tissue mask equals rte_region_gradient's grad2 (one tangent solve per
    tissue, proper masks) to 1e-6 in FP64, and single-voxel regions reproduce the GPU package's per-voxel
    tangent gradient (inverse_rte.cu:293-433)."""
    ctx, mua, mus, tiss, src, g = _image_problem(rte, rte.PREC_FP64)
    stop = rte.Stop(rte.STOP_FIXED, 15)
    loss, ga, gs = ctx.image_gradient(src, stop, g, image=0, deriv=rte.DERIV_REFERENCE)
    grada, grada2, grads, grads2, _, res2 = ctx.region_gradient(src, stop, g, tiss, 3, compat=False)
    assert abs(loss - res2) <= 1e-12 * res2
    got_a = np.array([0.01 * ga[tiss == t].sum() for t in (1, 2)])
    got_s = np.array([1.0 * gs[tiss == t].sum() for t in (1, 2)])
    assert rel(got_a, grada2[1:]) < 1e-6, (got_a, grada2)
    assert rel(got_s, grads2[1:]) < 1e-6, (got_s, grads2)
    rng = np.random.default_rng(2)
    for v in rng.choice(mua.size, 3, replace=False):
        one = np.full(mua.size, 2, np.uint8)
        one[v] = 1
        _, a2, _, s2, _, _ = ctx.region_gradient(src, stop, g, one, 3, compat=False)
        assert abs(0.01 * ga[v] - a2[1]) <= 1e-6 * abs(a2[1]) + 1e-18, (v, ga[v], a2[1])
        assert abs(gs[v] - s2[1]) <= 1e-6 * abs(s2[1]) + 1e-18, (v, gs[v], s2[1])
    ctx.close()


def test_image_gradient_reference_model_fim_files(rte):
    """The same identity on the reference's own discretisation (FisherInfo_IO model: table SH, its scatter and
    image weights) and on the reflection image."""
    ctx, mua, mus, tiss, src, g = _image_problem(rte, rte.PREC_FP64, n=10, model=rte.MODEL_FIM)
    stop = rte.Stop(rte.STOP_FIXED, 10)
    _, ga, gs = ctx.image_gradient(src, stop, g, image=0, deriv=rte.DERIV_REFERENCE)
    _, grada2 = ctx.region_gradient(src, stop, g, tiss, 3, compat=False)[:2]
    got = np.array([0.01 * ga[tiss == t].sum() for t in (1, 2)])
    assert rel(got, grada2[1:]) < 1e-6, (got, grada2)
    ctx.close()


def test_image_gradient_exact_matches_finite_differences(rte):
    """The exact derivative of the image misfit (one forward + one adjoint series + back-projection) against
    central finite differences on 20 seeded voxels, FP64, 60 terms (converged to rounding; a fixed count so
    that the two FD evaluations never stop at different terms).  Steps are 1e-4 relative to the voxel's mu_t
    for both coefficients: mu_a is ~1% of mu_t here, and a step relative to mu_a alone would put the loss
    difference near its FP64 rounding."""
    for image in (0, 1):
        ctx, mua, mus, tiss, src, g = _image_problem(rte, rte.PREC_FP64, n=7, image=image)
        stop = rte.Stop(rte.STOP_FIXED, 60)
        loss, ga, gs = ctx.image_gradient(src, stop, g, image=image, deriv=rte.DERIV_EXACT)

        def Lf(a, s):
            ctx.set_medium_voxel(a, s)
            r = ctx.forward(src, stop, want_W=False)
            return float(np.sum((r["trans" if image == 0 else "ref"].real.ravel() - g) ** 2))

        assert abs(Lf(mua, mus) - loss) < 1e-12 * loss
        vox = np.random.default_rng(4 + image).choice(mua.size, 20, replace=False)
        fa, fs = [], []
        for v in vox:
            h = 1e-4 * (mua[v] + mus[v])
            for arr, out in ((mua, fa), (mus, fs)):
                p = arr.copy()
                p[v] += h
                lp = Lf(p, mus) if arr is mua else Lf(mua, p)
                p[v] -= 2 * h
                lm = Lf(p, mus) if arr is mua else Lf(mua, p)
                out.append((lp - lm) / (2 * h))
        ctx.set_medium_voxel(mua, mus)
        assert rel(ga[vox], np.array(fa)) < 1e-5, (image, rel(ga[vox], np.array(fa)))
        assert rel(gs[vox], np.array(fs)) < 1e-5, (image, rel(gs[vox], np.array(fs)))
        ctx.close()


def test_image_gradient_mixed_vs_fp64(rte):
    out = {}
    for prec in (rte.PREC_FP64, rte.PREC_MIXED):
        ctx, mua, mus, tiss, src, g = _image_problem(rte, prec, n=11, L=3)
        stop = rte.Stop(rte.STOP_FIXED, 20)
        out[prec] = [ctx.image_gradient(src, stop, g, image=0, deriv=d) for d in (rte.DERIV_EXACT, rte.DERIV_REFERENCE)]
        ctx.close()
    for d in range(2):
        a, b = out[rte.PREC_MIXED][d], out[rte.PREC_FP64][d]
        assert rel(a[1], b[1]) < 1e-5 and rel(a[2], b[2]) < 1e-5, (d, rel(a[1], b[1]), rel(a[2], b[2]))
