"""Intensity modulation on the GPU (CPU package/src/RTE_uniform.c:120-176): mu_a -> mu_a + i*modulation/(c/n),
so mu_t has a uniform imaginary part kappa and the radiance is complex.  The pair kernels (FP64 and
mixed, stored and recomputed), the complex self-voxel term (table and power series), the sources, the
series with every stop rule and the images are checked against the oracle with the same kappa, which
test_oracle_golden.py pins to the CPU package's own modulated runs."""
import dataclasses

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

DX = 0.1
MOD = 0.7  # c = n = 1: kappa = 0.7 / cm


def _ctx(rte, n, L, prec, km=None, model=None):
    km = km if km is not None else (rte.KERNEL_STORE if prec else rte.KERNEL_RECOMPUTE)
    return rte.Context(n, n, n, dx=DX, nL=L, g=0.8, precision=prec, kernel_mode=km,
                       model=model if model is not None else rte.MODEL_EXACT)


def _params(oracle, ctx, n, L, kappa, mode=None):
    return oracle.params(n, n, n, DX, DX, DX, L, 0.8, 1.0, ctx.cfg.prop_thresh,
                         mode=oracle.MODE_EXACT if mode is None else mode, ssv=1, x_min=ctx.cfg.x_min,
                         y_min=ctx.cfg.y_min, z_min=ctx.cfg.z_min, kappa=kappa)


def _random_dist(rng, N, C):
    return rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))


@pytest.mark.parametrize("prec,km,tol", [(0, 2, 1e-11), (1, 1, 2e-6), (1, 2, 2e-6)])
@pytest.mark.parametrize("flag,flag_scat", [(1, 1), (1, 0), (0, 1)])
def test_prop_abs_modulated(rte, oracle, prec, km, tol, flag, flag_scat):
    """One application of [D] A with the complex mu_t on an arbitrary complex distribution."""
    n, L = 7, 3
    N, C = n ** 3, (L + 1) ** 2
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=5, rmin=0.15, rmax=0.3)
    ctx = _ctx(rte, n, L, prec, km)
    ctx.set_medium_voxel(mua, mus)
    ctx.set_modulation(MOD)
    W = _random_dist(np.random.default_rng(1), N, C)
    W = oracle.apply(_params(oracle, ctx, n, L, 0.0), mua, mus, W, 1, 0)  # a smooth complex field
    got = ctx.prop_abs(W, flag, flag_scat)
    p = _params(oracle, ctx, n, L, MOD)
    ctx.close()
    ref = oracle.apply(p, mua, mus, W, flag, flag_scat)
    assert rel(got, ref) < tol


def test_prop_abs_modulated_power_series(rte, oracle):
    """More than 4096 distinct mu_t: the self term takes the power series in the complex mu_t."""
    n, L = 17, 2
    N, C = n ** 3, (L + 1) ** 2
    rng = np.random.default_rng(3)
    mua, mus = rng.uniform(0.005, 0.05, N), rng.uniform(0.5, 2.0, N)
    ctx = _ctx(rte, n, L, 0)
    ctx.set_medium_voxel(mua, mus)
    ctx.set_modulation(MOD)
    W = np.zeros((N, C), np.complex128)
    W[:, 0] = rng.uniform(0, 1, N) + 0.3j * rng.uniform(0, 1, N)
    got = ctx.prop_abs(W, 1, 1)
    p = _params(oracle, ctx, n, L, MOD)
    ctx.close()
    dests = rng.choice(N, 24, replace=False).astype(np.int32)
    ref = oracle.apply_subset(p, mua, mus, W, dests, 1, 1)
    assert rel(got[dests], ref[dests]) < 1e-11


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-5)])
@pytest.mark.parametrize("rule", ["fixed", "reference"])
def test_neumann_modulated(rte, oracle, prec, tol, rule):
    n, L = 9, 3
    N, C = n ** 3, (L + 1) ** 2
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=8, rmin=0.15, rmax=0.3)
    ctx = _ctx(rte, n, L, prec)
    ctx.set_medium_voxel(mua, mus)
    ctx.set_modulation(MOD)
    p = _params(oracle, ctx, n, L, MOD)
    xi = oracle.source(p, mua, mus, pos_x=0.0, pos_y=0.0, kind=oracle.SRC_COLUMN)  # complex source
    if rule == "fixed":
        out, nt = ctx.neumann(xi, xi, 1, rte.Stop(rte.STOP_FIXED, 7))
        ref, _, nref = oracle.neumann(p, mua, mus, xi, xi, 1, oracle.STOP_FIXED, max_terms=7)
    else:
        out, nt = ctx.neumann(xi, xi, 1, rte.Stop(rte.STOP_REFERENCE))
        ref, _, nref = oracle.neumann(p, mua, mus, xi, xi, 1, oracle.STOP_REFERENCE, n0=2)
    ctx.close()
    assert nt == nref
    assert rel(out, ref) < tol


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 1e-5)])
@pytest.mark.parametrize("kind", ["column", "point"])
def test_forward_modulated(rte, oracle, prec, tol, kind):
    """rte_forward at the source's modulation: complex source (complex attenuation along the column),
    complex series, images with the complex ballistic term."""
    n, L, T = 9, 3, 8
    N, C = n ** 3, (L + 1) ** 2
    mua, mus, _ = rte.sphere_phantom(n, nspheres=2, seed=12, rmin=0.15, rmax=0.3)
    ctx = _ctx(rte, n, L, prec)
    ctx.set_medium_voxel(mua, mus)
    p = _params(oracle, ctx, n, L, MOD)
    if kind == "column":
        src = rte.Source(pos_x=0.1, pos_y=-0.2, kind=rte.SRC_COLUMN, mag=1.5, modulation=MOD)
        res = ctx.forward(src, rte.Stop(rte.STOP_FIXED, T))
        xi = oracle.source(p, mua, mus, pos_x=0.1, pos_y=-0.2, mag=1.5, kind=oracle.SRC_COLUMN)
        out, _, _ = oracle.neumann(p, mua, mus, xi, xi, 1, oracle.STOP_FIXED, max_terms=T)
        tr, rf = oracle.images(p, mua, mus, out, 0, pos_x=0.1, pos_y=-0.2, mag=1.5)
    else:
        src = rte.Source(pos_x=0.1, pos_y=-0.2, kind=rte.SRC_POINT, face=0, mag=2.0, modulation=MOD)
        res = ctx.forward(src, rte.Stop(rte.STOP_FIXED, T))
        cx, cy = int((0.1 - ctx.cfg.x_min) / DX), int((-0.2 - ctx.cfg.y_min) / DX)
        q = np.zeros((N, C), np.complex128)
        q[cy * n + cx, 0] = 2.0 / (np.sqrt(4 * np.pi) * DX ** 3)
        daq = oracle.apply(p, mua, mus, q, 1, 1)
        out, _, _ = oracle.neumann(p, mua, mus, daq, q + daq, 1, oracle.STOP_FIXED, max_terms=T)
        tr, rf = oracle.images(p, mua, mus, out, 0, with_ballistic=0)
    ctx.close()
    assert res["terms"] == T
    assert rel(res["W"], out) < tol
    assert rel(res["trans"], tr) < tol and rel(res["ref"], rf) < tol
    assert np.abs(np.angle(res["trans"])).max() > 1e-3  # a real phase delay


def test_cpu_model_modulated_series_matches_oracle(rte, oracle):
    """CPU-package model (uniform medium, its quadratures) under modulation: rte_neumann with the
    package's stop rule, against the oracle restatement that reproduces the package's own runs."""
    n, L = 9, 2
    N = n ** 3
    ctx = rte.Context(n, n, n, dx=DX, nL=L, g=0.8, model=rte.MODEL_CPU, precision=0, prop_thresh=10.0,
                      kernel_mode=rte.KERNEL_AUTO)
    mua, mus = np.full(N, 0.02), np.full(N, 1.5)
    ctx.set_medium_voxel(mua, mus)
    src = rte.Source(diam=0.1, kind=rte.SRC_CPU)
    xi = ctx.source_beam(src)  # built before the modulation, as the package does
    ctx.set_modulation(0.5)
    out, nt = ctx.neumann(xi, xi, 1, rte.Stop(rte.STOP_REFERENCE))
    p = _params(oracle, ctx, n, L, 0.5, mode=oracle.MODE_CPU)
    ref, _, nref = oracle.neumann(p, mua, mus, xi, xi, 1, oracle.STOP_REFERENCE, n0=1)
    ctx.close()
    assert nt == nref
    assert rel(out, ref) < 1e-11


def test_modulation_back_to_zero_and_limits(rte):
    """Setting the modulation back to 0 restores the steady-state operator exactly; a vanishing
    modulation is continuous; the entry points without a complex form refuse loudly."""
    n, L = 7, 2
    mua, mus, _ = rte.sphere_phantom(n, nspheres=1, seed=2, rmin=0.15, rmax=0.3)
    ctx = _ctx(rte, n, L, 1)
    ctx.set_medium_voxel(mua, mus)
    stop = rte.Stop(rte.STOP_FIXED, 6)
    src = rte.Source(kind=rte.SRC_COLUMN)
    a = ctx.forward(src, stop)
    b = ctx.forward(dataclasses.replace(src, modulation=1e-9), stop)
    c = ctx.forward(src, stop)  # the solve resets the context to the source's modulation (0)
    assert rel(b["W"], a["W"]) < 1e-6 and rel(c["W"], a["W"]) < 1e-14
    ctx.set_modulation(0.3)
    with pytest.raises(rte.RteError):
        ctx.gradient([src], stop, rte.Detector(4, 63), np.zeros((1, 6, 4, 4)))
    with pytest.raises(rte.RteError):
        ctx.forward_graph([src], 4)
    with pytest.raises(rte.RteError):  # |mu_t + i kappa| beyond the self-term series: refused, state kept
        ctx.set_modulation(1e5)
    assert rel(ctx.forward(src, stop)["W"], a["W"]) < 1e-14
    ctx.close()
    fim = rte.Context(8, 8, 8, dx=DX, nL=2, model=rte.MODEL_FIM, precision=0)
    with pytest.raises(rte.RteError):
        fim.set_modulation(0.3)
    fim.close()


@pytest.mark.parametrize("prec,tol", [(0, 1e-11), (1, 2e-6)])
@pytest.mark.parametrize("mod", [0.0, MOD])
def test_anisotropic_voxels_and_modulation(rte, oracle, prec, tol, mod):
    """Non-cubic grid with three different voxel edges (the reference's Delta = (max - min) / n per
    axis), with and without modulation, heterogeneous medium, every flag combination."""
    nx, ny, nz, L = 6, 7, 5, 3
    dx, dy, dz = 0.1, 0.12, 0.08
    N, C = nx * ny * nz, (L + 1) ** 2
    rng = np.random.default_rng(11)
    mua, mus = rng.uniform(0.005, 0.1, N), rng.uniform(0.5, 2.0, N)
    ctx = rte.Context(nx, ny, nz, dx=dx, dy=dy, dz=dz, nL=L, g=0.8, precision=prec, model=rte.MODEL_EXACT,
                      kernel_mode=rte.KERNEL_STORE if prec else rte.KERNEL_RECOMPUTE)
    ctx.set_medium_voxel(mua, mus)
    ctx.set_modulation(mod)
    p = oracle.params(nx, ny, nz, dx, dy, dz, L, 0.8, 1.0, ctx.cfg.prop_thresh, mode=oracle.MODE_EXACT, ssv=1,
                      x_min=ctx.cfg.x_min, y_min=ctx.cfg.y_min, z_min=ctx.cfg.z_min, kappa=mod)
    W = _random_dist(rng, N, C)
    W = oracle.apply(p, mua, mus, W, 1, 0)
    for flag, fs in ((1, 1), (1, 0), (0, 1)):
        got = ctx.prop_abs(W, flag, fs)
        ref = oracle.apply(p, mua, mus, W, flag, fs)
        assert rel(got, ref) < tol, (flag, fs, rel(got, ref))
    ctx.close()
