"""ctypes binding of the FP64 oracle (liboracle.so built from rte_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm as the checker.  Distributions are complex128 arrays of shape
(N, C) in the reference's layout (voxel r = (z*nY + y)*nX + x, coefficient cnt = l*l+l+m).
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MODE_EXACT, MODE_FIM, MODE_CPU = 0, 1, 2
SRC_COLUMN, SRC_FIM, SRC_CPU = 0, 1, 2
STOP_REFERENCE, STOP_FIXED, STOP_REL_L2 = 0, 1, 2


class OrcParams(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("x_min", ctypes.c_double), ("y_min", ctypes.c_double), ("z_min", ctypes.c_double),
                ("L", ctypes.c_int), ("g", ctypes.c_double), ("cm", ctypes.c_double),
                ("prop_thresh", ctypes.c_double), ("mode", ctypes.c_int), ("ssv", ctypes.c_int),
                ("nthreads", ctypes.c_int), ("kappa", ctypes.c_double)]


class OrcSource(ctypes.Structure):
    _fields_ = [("pos_x", ctypes.c_double), ("pos_y", ctypes.c_double), ("pos_z", ctypes.c_double),
                ("diam", ctypes.c_double), ("mag", ctypes.c_double), ("kind", ctypes.c_int)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (run oracle/build.sh)")
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        P = ctypes.POINTER(OrcParams)
        S = ctypes.POINTER(OrcSource)
        L.orc_apply.argtypes = [P, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int]
        L.orc_apply_subset.argtypes = [P, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_int), ctypes.c_long]
        L.orc_source.argtypes = [P, dp, dp, S, dp]
        L.orc_neumann.argtypes = [P, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.orc_neumann_split.argtypes = [P, dp, dp, dp, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.orc_images.argtypes = [P, dp, dp, S, ctypes.c_int, ctypes.c_int, dp, dp, dp]
        L.orc_sh_complex.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, dp]
        L.orc_assoc_legendre.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.orc_assoc_legendre.restype = ctypes.c_double
        L.orc_path_integral.argtypes = [P, dp] + [ctypes.c_int] * 7
        L.orc_path_integral.restype = ctypes.c_double
        L.orc_self_matrix.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, dp]
        L.orc_table_clamps.restype = ctypes.c_long
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def params(nx, ny, nz, dx, dy, dz, L, g, cm, prop_thresh, mode=MODE_EXACT, ssv=1,
           x_min=None, y_min=None, z_min=0.0, nthreads=0, kappa=0.0):
    """kappa: imaginary part of mu_t under intensity modulation (modulation * n / c)."""
    if x_min is None:
        x_min = -nx * dx / 2.0
    if y_min is None:
        y_min = -ny * dy / 2.0
    return OrcParams(nx, ny, nz, dx, dy, dz, x_min, y_min, z_min, L, g, cm, prop_thresh, mode, ssv,
                     nthreads, kappa)


def ncoef(L):
    return (L + 1) * (L + 1)


def apply(p, mua, mus, W, flag=1, flag_scat=1):
    """One pass of the reference operator: out = D A W (flag_scat=1) or A W."""
    N = p.nx * p.ny * p.nz
    C = ncoef(p.L)
    mua = np.ascontiguousarray(mua, np.float64).ravel()
    mus = np.ascontiguousarray(mus, np.float64).ravel()
    W = np.ascontiguousarray(W, np.complex128).reshape(N, C)
    out = np.zeros((N, C), np.complex128)
    lib().orc_apply(ctypes.byref(p), _dp(mua), _dp(mus), _dp(W.view(np.float64)),
                    _dp(out.view(np.float64)), flag, flag_scat)
    return out


def apply_subset(p, mua, mus, W, dests, flag=1, flag_scat=1):
    """The operator for the listed destination voxels only (rows of the result outside the list are 0)."""
    N = p.nx * p.ny * p.nz
    C = ncoef(p.L)
    mua = np.ascontiguousarray(mua, np.float64).ravel()
    mus = np.ascontiguousarray(mus, np.float64).ravel()
    W = np.ascontiguousarray(W, np.complex128).reshape(N, C)
    d = np.ascontiguousarray(dests, np.int32)
    out = np.zeros((N, C), np.complex128)
    lib().orc_apply_subset(ctypes.byref(p), _dp(mua), _dp(mus), _dp(W.view(np.float64)), _dp(out.view(np.float64)),
                           flag, flag_scat, d.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(d))
    return out


def source(p, mua, mus, pos_x=0.0, pos_y=0.0, diam=0.1, mag=1.0, kind=SRC_COLUMN):
    N = p.nx * p.ny * p.nz
    C = ncoef(p.L)
    mua = np.ascontiguousarray(mua, np.float64).ravel()
    mus = np.ascontiguousarray(mus, np.float64).ravel()
    W = np.zeros((N, C), np.complex128)
    s = OrcSource(pos_x, pos_y, 0.0, diam, mag, kind)
    lib().orc_source(ctypes.byref(p), _dp(mua), _dp(mus), ctypes.byref(s), _dp(W.view(np.float64)))
    return W


def neumann(p, mua, mus, W, out, flag=1, stop_rule=STOP_FIXED, max_terms=20, tol=1e-7, n0=2, mut_self=None):
    """Neumann(W, out, flag) of the reference; returns (A*sum, last term, number of terms).
    mut_self: per-voxel mu_t of the self-voxel term when it differs from mua + mus (the path
    integrals and the scatter keep mua, mus), as in the FisherInfo_IO mains whose device tissue
    table goes stale (rte_snr.cu:239, rte_fim.cu:231, compute_grad_rte.cu:431)."""
    mua = np.ascontiguousarray(mua, np.float64).ravel()
    mus = np.ascontiguousarray(mus, np.float64).ravel()
    W = np.array(W, np.complex128, copy=True)
    out = np.array(out, np.complex128, copy=True)
    nt = ctypes.c_int(0)
    ms = None if mut_self is None else np.ascontiguousarray(mut_self, np.float64).ravel()
    lib().orc_neumann_split(ctypes.byref(p), _dp(mua), _dp(mus), None if ms is None else _dp(ms),
                            _dp(W.view(np.float64)), _dp(out.view(np.float64)), flag, stop_rule, max_terms, tol, n0,
                            ctypes.byref(nt))
    return out, W, nt.value


def images(p, mua, mus, out, img_mode, pos_x=0.0, pos_y=0.0, diam=0.1, mag=1.0, with_ballistic=1):
    mua = np.ascontiguousarray(mua, np.float64).ravel()
    mus = np.ascontiguousarray(mus, np.float64).ravel()
    out = np.ascontiguousarray(out, np.complex128)
    trans = np.zeros(p.nx * p.ny, np.complex128)
    ref = np.zeros(p.nx * p.ny, np.complex128)
    s = OrcSource(pos_x, pos_y, 0.0, diam, mag, 0)
    lib().orc_images(ctypes.byref(p), _dp(mua), _dp(mus), ctypes.byref(s), img_mode, with_ballistic,
                     _dp(out.view(np.float64)), _dp(trans.view(np.float64)), _dp(ref.view(np.float64)))
    return trans.reshape(p.ny, p.nx), ref.reshape(p.ny, p.nx)


def forward(p, mua, mus, src_kind=SRC_COLUMN, img_mode=0, stop_rule=STOP_FIXED, max_terms=20, tol=1e-7,
            n0=2, pos_x=0.0, pos_y=0.0, diam=0.1, mag=1.0):
    """Reference forward solve (rte.cu:139-210): source, Neumann, images."""
    src = source(p, mua, mus, pos_x, pos_y, diam, mag, src_kind)
    out, _, nt = neumann(p, mua, mus, src, src, 1, stop_rule, max_terms, tol, n0)
    tr, rf = images(p, mua, mus, out, img_mode, pos_x, pos_y, diam, mag)
    return dict(src=src, out=out, trans=tr, ref=rf, terms=nt)


def sh_complex(L, theta, phi):
    out = np.zeros(ncoef(L), np.complex128)
    lib().orc_sh_complex(L, theta, phi, _dp(out.view(np.float64)))
    return out


def path_integral(p, mut, src, dst, fp32ref=False):
    mut = np.ascontiguousarray(mut, np.float64).ravel()
    return lib().orc_path_integral(ctypes.byref(p), _dp(mut), src[0], src[1], src[2], dst[0], dst[1],
                                   dst[2], int(fp32ref))


def self_matrix(quad, L, ssv, mut, dx, dy, dz):
    C = ncoef(L)
    out = np.zeros((C, C), np.complex128)
    lib().orc_self_matrix(quad, L, ssv, mut, dx, dy, dz, _dp(out.view(np.float64)))
    return out


def downsample_image(img, nx, ny, ds):
    """Pure-Python restatement of downsample_image (FisherInfo_IO/src/dist.cu:271-289) on a flat
    nX*nY image: out[i*(nY//ds) + j] += img[(i*ds + a)*nY + j*ds + b], loops in the reference's
    order (i, j, a, b), sums from zero (the reference's malloc block is not cleared).  Returns the
    (nX//ds)*(nY//ds) values the reference's loops write."""
    img = np.asarray(img, np.complex128).ravel()
    mx, my = nx // ds, ny // ds
    out = [0j] * (nx * ny // (ds * ds))
    for i in range(mx):
        for j in range(my):
            for a in range(ds):
                for b in range(ds):
                    out[i * my + j] += img[(i * ds + a) * ny + j * ds + b]
    return np.array(out[:mx * my], np.complex128)
