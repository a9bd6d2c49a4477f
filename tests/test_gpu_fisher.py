"""Fisher information from tangent solves (rte_fisher) on the GPU: the sensitivity J of the binned
exitant flux to the position and contrast of inclusions (smooth partial-volume rasterisation)
against central finite differences of rte_detector_flux, F against J^T diag(1/flux) J, and the
mixed-precision F against FP64.  Series run to convergence (relative L2 1e-13) so the tangent of the
converged model is the exact derivative."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

N_SIDE, L = 9, 2


def _problem(rte, prec, kernel_mode=None, Lq=L):
    sph = rte.random_spheres(N_SIDE, 2, seed=3, rmin=0.15, rmax=0.25)
    if kernel_mode is None:
        kernel_mode = rte.KERNEL_STORE if prec == rte.PREC_MIXED else rte.KERNEL_RECOMPUTE
    ctx = rte.Context(N_SIDE, N_SIDE, N_SIDE, dx=0.1, nL=Lq, g=0.9, precision=prec, kernel_mode=kernel_mode)
    mua, mus, dmua, dmus = rte.smooth_sphere_phantom(N_SIDE, sph, mua_bg=0.02, mus_bg=2.0)
    ctx.set_medium_voxel(mua, mus)
    c = 0.45 - 0.45  # face centres of the 0.9 cm box (x, y centred on 0, z from 0.05 to 0.85)
    srcs = [rte.Source(pos_x=c, pos_y=c, kind=rte.SRC_BEAM, face=0),
            rte.Source(pos_y=0.05, pos_z=0.45, kind=rte.SRC_BEAM, face=4)]
    return ctx, sph, srcs, mua, mus, dmua, dmus


def _flux(rte, ctx, sph, srcs, stop, det):
    mua, mus, _, _ = rte.smooth_sphere_phantom(N_SIDE, sph, mua_bg=0.02, mus_bg=2.0)
    ctx.set_medium_voxel(mua, mus)
    return ctx.detector_flux(srcs, stop, det)


def test_sensitivity_matches_finite_differences(rte):
    ctx, sph, srcs, mua, mus, dmua, dmus = _problem(rte, rte.PREC_FP64)
    stop = rte.Stop(rte.STOP_REL_L2, 600, 1e-13)
    det = rte.Detector(nbins=3, faces=63)
    F, J = ctx.fisher(srcs, stop, det, dmua, dmus, want_J=True)
    y = ctx.detector_flux(srcs, stop, det)
    P = dmua.shape[0]
    for p in range(P):
        i, k = divmod(p, 4)
        h = 1e-5 if k < 3 else 1e-5 * sph[i]["ka"]
        fd = []
        for sgn in (1, -1):
            sp = [dict(x) for x in sph]
            if k < 3:
                cc = list(sp[i]["c"])
                cc[k] += sgn * h
                sp[i]["c"] = cc
            else:
                sp[i]["ka"] += sgn * h
            fd.append(_flux(rte, ctx, sp, srcs, stop, det))
        fdj = (fd[0] - fd[1]) / (2 * h)
        assert rel(J[..., p], fdj) < 1e-5, (p, rel(J[..., p], fdj))
    Jm = J.reshape(-1, P)
    w = np.where(y.ravel() > 0, 1.0 / np.where(y.ravel() > 0, y.ravel(), 1.0), 0.0)
    assert rel(F, Jm.T @ (w[:, None] * Jm)) < 1e-12
    assert np.allclose(F, F.T) and np.linalg.eigvalsh(F).min() > -1e-12 * np.abs(F).max()
    ctx.close()


@pytest.mark.parametrize("Lq,stored", [(2, True), (2, False), (5, False), (7, False)])
def test_fisher_mixed_vs_fp64(rte, Lq, stored):
    """Mixed precision against the FP64 method, with the stored FP32 kernel or with the path integrals
    recomputed in every term (the Fisher benchmark's form): J and F within 1e-5 (measured 1.6e-7 and
    2.3e-7 at L = 2, stored).  The 8 parameters run as two groups of four tangent series (at L = 7 with
    the kernel whose two thread groups share each pair's walk).  F weights bins by 1/flux, so on detectors
    with near-zero-flux bins its relative error can exceed J's."""
    stop = rte.Stop(rte.STOP_REL_L2, 600, 1e-12)
    det = rte.Detector(nbins=3, faces=63)
    out = []
    for prec in (rte.PREC_FP64, rte.PREC_MIXED):
        mode = None if prec == rte.PREC_FP64 else (rte.KERNEL_STORE if stored else rte.KERNEL_RECOMPUTE)
        ctx, sph, srcs, mua, mus, dmua, dmus = _problem(rte, prec, mode, Lq)
        out.append(ctx.fisher(srcs, stop, det, dmua, dmus, want_J=True))
        ctx.close()
    (F64, J64), (F32, J32) = out
    assert rel(J32, J64) < 1e-5, rel(J32, J64)
    assert rel(F32, F64) < 1e-5, rel(F32, F64)


def test_fisher_adds_over_sources(rte):
    """F is a sum over sources: two sources in one call against the sum of two one-source calls, mixed
    precision, path integrals recomputed, L = 5 (four-parameter tangent groups)."""
    stop = rte.Stop(rte.STOP_REL_L2, 600, 1e-12)
    det = rte.Detector(nbins=3, faces=63)
    ctx, sph, srcs, mua, mus, dmua, dmus = _problem(rte, rte.PREC_MIXED, rte.KERNEL_RECOMPUTE, 5)
    F2, J2 = ctx.fisher(srcs, stop, det, dmua, dmus, want_J=True)
    F0, J0 = ctx.fisher(srcs[:1], stop, det, dmua, dmus, want_J=True)
    F1, J1 = ctx.fisher(srcs[1:], stop, det, dmua, dmus, want_J=True)
    ctx.close()
    assert rel(J2[0], J0[0]) < 1e-6 and rel(J2[1], J1[0]) < 1e-6, (rel(J2[0], J0[0]), rel(J2[1], J1[0]))
    assert rel(F2, F0 + F1) < 1e-6, rel(F2, F0 + F1)


def test_fisher_six_beams_mixed_vs_fp64(rte):
    """Six face-centre beams on a strongly scattering medium (mu_s 2, g 0.9), 16x16 bins on every face:
    the detector has dim bins, whose 1/flux weights amplify flux errors in F.  Mixed precision (FP64
    forward solves, mixed tangent series) against the FP64 method: F and J within 1e-5."""
    n, Lq = 17, 3
    stop = rte.Stop(rte.STOP_FIXED, 20)
    det = rte.Detector(nbins=16, faces=63)
    sph = rte.random_spheres(n, 2, seed=7, rmin=0.2, rmax=0.3)
    mua, mus, dmua, dmus = rte.smooth_sphere_phantom(n, sph, mua_bg=0.02, mus_bg=2.0)
    h = n * 0.1 / 2
    srcs = [rte.Source(kind=rte.SRC_BEAM, face=0), rte.Source(kind=rte.SRC_BEAM, face=1, pos_z=n * 0.1)] + \
           [rte.Source(kind=rte.SRC_BEAM, face=f, pos_z=h) for f in (2, 3, 4, 5)]
    out = {}
    for prec in (rte.PREC_FP64, rte.PREC_MIXED):
        ctx = rte.Context(n, n, n, dx=0.1, nL=Lq, g=0.9, precision=prec, kernel_mode=rte.KERNEL_RECOMPUTE)
        ctx.set_medium_voxel(mua, mus)
        out[prec] = ctx.fisher(srcs, stop, det, dmua, dmus, want_J=True)
        ctx.close()
    (F64, J64), (F32, J32) = out[rte.PREC_FP64], out[rte.PREC_MIXED]
    assert rel(J32, J64) < 1e-5, rel(J32, J64)
    assert rel(F32, F64) < 1e-5, rel(F32, F64)
