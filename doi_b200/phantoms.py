"""Seeded synthetic phantoms (the reference ships only two 20^3 tissue maps; the benchmark media are
synthetic: uniform background plus spherical inclusions, values sampled at voxel centres)."""
import numpy as np


def grid_centres(nx, ny, nz, dx, x_min=None, y_min=None, z_min=0.0):
    x_min = -nx * dx / 2 if x_min is None else x_min
    y_min = -ny * dx / 2 if y_min is None else y_min
    xs = x_min + (np.arange(nx) + 0.5) * dx
    ys = y_min + (np.arange(ny) + 0.5) * dx
    zs = z_min + (np.arange(nz) + 0.5) * dx
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")  # (nz, ny, nx): x fastest
    return X, Y, Z


def uniform_phantom(nx, ny, nz, mua=0.01, mus=1.0):
    n = nx * ny * nz
    return np.full(n, float(mua)), np.full(n, float(mus))


def sphere_phantom(n, dx=0.1, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=0, rmin=0.2, rmax=0.6,
                   mua_contrast=(2.0, 10.0), mus_contrast=(0.5, 2.0), ny=None, nz=None):
    """Background plus `nspheres` spheres (radius ~U[rmin,rmax] cm, centre uniform over the box shrunk
    by the radius, mu_a x U[mua_contrast], mu_s x U[mus_contrast]); later spheres overwrite earlier
    ones.  Box: x, y centred on 0, z from 0.  Returns (mua, mus, spheres) with per-voxel arrays."""
    nx = n
    ny = n if ny is None else ny
    nz = n if nz is None else nz
    rng = np.random.Generator(np.random.PCG64(seed))
    X, Y, Z = grid_centres(nx, ny, nz, dx)
    lo = np.array([-nx * dx / 2, -ny * dx / 2, 0.0])
    hi = np.array([nx * dx / 2, ny * dx / 2, nz * dx])
    mua = np.full(X.shape, float(mua_bg))
    mus = np.full(X.shape, float(mus_bg))
    spheres = []
    for _ in range(nspheres):
        r = rng.uniform(rmin, rmax)
        c = rng.uniform(lo + r, hi - r)
        ka = rng.uniform(*mua_contrast)
        ks = rng.uniform(*mus_contrast)
        inside = (X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2 <= r * r
        mua[inside] = mua_bg * ka
        mus[inside] = mus_bg * ks
        spheres.append(dict(r=r, centre=c.tolist(), mua=mua_bg * ka, mus=mus_bg * ks))
    return mua.ravel(), mus.ravel(), spheres


def smooth_sphere_phantom(n, spheres, dx=0.1, mua_bg=0.02, mus_bg=2.0, width=None):
    """Background plus spheres rasterised with a linear partial-volume ramp of `width` (default one
    voxel) across each surface, so the medium is differentiable in the sphere parameters:
        f_i(v) = clip(1/2 + (r_i - |x_v - c_i|) / width, 0, 1),
        mu_a = mu_a,bg (1 + sum_i (ka_i - 1) f_i),  mu_s = mu_s,bg (1 + sum_i (ks_i - 1) f_i).
    spheres: dicts with centre c (cm, box x,y centred on 0, z from 0), radius r, contrasts ka, ks.
    Returns (mua, mus, dmua, dmus) with the derivative fields for the parameters
    (cx, cy, cz, ka) of every sphere in order: arrays of shape (4 * len(spheres), n^3)."""
    w = dx if width is None else width
    X, Y, Z = grid_centres(n, n, n, dx)
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    N = n ** 3
    mua = np.full(N, float(mua_bg))
    mus = np.full(N, float(mus_bg))
    dmua = np.zeros((4 * len(spheres), N))
    dmus = np.zeros((4 * len(spheres), N))
    for i, sp in enumerate(spheres):
        c = np.asarray(sp["c"], float)
        rel = pos - c
        rho = np.linalg.norm(rel, axis=1)
        u = 0.5 + (sp["r"] - rho) / w
        f = np.clip(u, 0.0, 1.0)
        ramp = (u > 0.0) & (u < 1.0)
        # d f / d c = (x - c) / (w rho) inside the ramp
        dfdc = np.where(ramp[:, None], rel / (w * np.maximum(rho, 1e-300))[:, None], 0.0)
        mua += mua_bg * (sp["ka"] - 1.0) * f
        mus += mus_bg * (sp["ks"] - 1.0) * f
        for a in range(3):
            dmua[4 * i + a] = mua_bg * (sp["ka"] - 1.0) * dfdc[:, a]
            dmus[4 * i + a] = mus_bg * (sp["ks"] - 1.0) * dfdc[:, a]
        dmua[4 * i + 3] = mua_bg * f
    return mua, mus, dmua, dmus


def random_spheres(n, count, seed=0, dx=0.1, rmin=0.2, rmax=0.6, ka=(2.0, 10.0), ks=(0.5, 2.0)):
    """Seeded inclusions inside the box (centres at least one radius plus one voxel from the faces)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo = np.array([-n * dx / 2, -n * dx / 2, 0.0])
    hi = np.array([n * dx / 2, n * dx / 2, n * dx])
    out = []
    for _ in range(count):
        r = rng.uniform(rmin, rmax)
        out.append(dict(c=rng.uniform(lo + r + dx, hi - r - dx).tolist(), r=r, ka=rng.uniform(*ka),
                        ks=rng.uniform(*ks)))
    return out
