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
