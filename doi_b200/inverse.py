"""Optimiser loop for the inverse problem on top of the adjoint gradient (rte_gradient).

The reference's inverse mains step tissue types or coefficients by the sign of region gradients with
fixed step sizes (GPU package/src/inverse_rte.cu:448-485, FisherInfo_IO/src/compute_grad_rte.cu:
396-420).  Here the per-voxel coefficients are updated in log space, mu <- mu exp(-step mu dL/dmu),
which keeps them positive, with a backtracking (Armijo) step so the misfit decreases at every
accepted iteration.
"""
import numpy as np


def reconstruct(ctx, srcs, stop, det, target, mua0, mus0, iters=10, step=None, fit_mus=True, shrink=0.5,
                armijo=1e-4, max_backtrack=8):
    """Fit per-voxel (mu_a, mu_s) to the binned flux `target` (shape of Context.detector_flux).

    Returns (mua, mus, history) where history lists the misfit after each accepted step (first entry:
    the starting misfit).  ctx keeps the last medium it was given."""
    mua = np.array(mua0, np.float64)
    mus = np.array(mus0, np.float64)
    ctx.set_medium_voxel(mua, mus)
    loss, ga, gs = ctx.gradient(srcs, stop, det, target)
    hist = [loss]
    if not fit_mus:
        gs = np.zeros_like(gs)
    for _ in range(iters):
        # directions in log space: d(log mu) = -mu * dL/dmu
        da, ds = -mua * ga, -mus * gs
        slope = -float(np.dot(da, da) + np.dot(ds, ds))
        if slope == 0.0:
            break
        t = step if step is not None else 0.1 / max(np.abs(da).max(), np.abs(ds).max())
        for _ in range(max_backtrack):
            na, ns = mua * np.exp(t * da), mus * np.exp(t * ds)
            ctx.set_medium_voxel(na, ns)
            trial = float(np.sum((ctx.detector_flux(srcs, stop, det) - target) ** 2))
            if trial <= loss + armijo * t * slope:
                break
            t *= shrink
        else:
            ctx.set_medium_voxel(mua, mus)
            break
        mua, mus = na, ns
        loss, ga, gs = ctx.gradient(srcs, stop, det, target)
        if not fit_mus:
            gs = np.zeros_like(gs)
        hist.append(loss)
    return mua, mus, hist
