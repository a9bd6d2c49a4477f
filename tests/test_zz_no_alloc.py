"""rte_attenuate_noalloc: the entry point for callers that may not allocate device memory.

It is checked against the context API (rte_prop_abs with flag = 1, flag_scat = 0), whose result
is the same pair sum plus the self-voxel term.  The self term only involves a voxel's own input,
so with input supported on one colour of a 3D checkerboard, the two results must agree on the
other colour.  Two calls in a row (each colour once, then a repeat) also check that the shared
scratch array carries nothing from one call into the next.  Tolerance: 1e-11 relative L2 (both
paths are FP64).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from conftest import real_to_complex, rel

pytestmark = pytest.mark.gpu


def _call(lib, nx, ny, nz, dx, L, prop, cm, d_mut, d_in, d_out, stream):
    f = lib.rte_attenuate_noalloc
    f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                                 ctypes.c_void_p]
    return f(nx, ny, nz, dx, dx, dx, L, prop, cm, d_mut, d_in, d_out, stream)


def test_attenuate_noalloc_matches_context_path(rte):
    import torch
    lib = rte.load_library()
    rng = np.random.default_rng(11)
    nx, ny, nz, L, dx = 7, 6, 5, 3, 0.1
    N, C = nx * ny * nz, (L + 1) ** 2
    mua = rng.uniform(0.005, 0.1, N)
    mus = rng.uniform(0.5, 2.0, N)
    ctx = rte.Context(nx, ny, nz, dx=dx, nL=L, g=0.8, precision=rte.PREC_FP64, model=rte.MODEL_EXACT)
    ctx.set_medium_voxel(mua, mus)
    prop = ctx.cfg.prop_thresh
    colour = ((np.arange(N) % nx) + (np.arange(N) // nx) % ny + np.arange(N) // (nx * ny)) % 2
    dev = torch.device("cuda:0")
    d_mut = torch.tensor(mua + mus, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def make(col):
        W = real_to_complex(rng.standard_normal((N, C)), L) + 0.25j * real_to_complex(rng.standard_normal((N, C)), L)
        W[colour != col] = 0.0
        return W

    W0, W1 = make(0), make(1)
    outs = []
    for col, W in ((0, W0), (1, W1), (0, W0)):
        d_in = torch.from_numpy(np.ascontiguousarray(W)).to(dev)
        d_out = torch.full((N, C), complex(np.nan, np.nan), dtype=torch.complex128, device=dev)
        rc = _call(lib, nx, ny, nz, dx, L, prop, 1.0, d_mut.data_ptr(), d_in.data_ptr(), d_out.data_ptr(),
                   stream.cuda_stream)
        assert rc == 0, lib.rte_last_error(None)
        torch.cuda.synchronize(dev)
        got = d_out.cpu().numpy()
        ref = ctx.prop_abs(W, 1, 0)
        other = colour != col
        assert np.all(np.isfinite(got))
        assert rel(got[other], ref[other]) < 1e-11, rel(got[other], ref[other])
        outs.append(got)
    # same input, same result: nothing of the previous call leaks through the shared scratch
    assert np.array_equal(outs[0], outs[2])
    ctx.close()


def test_attenuate_noalloc_rejects_oversize(rte):
    import torch
    lib = rte.load_library()
    dev = torch.device("cuda:0")
    d = torch.zeros(8, dtype=torch.float64, device=dev)
    # 64^3 voxels at nL = 7 need ~ 5 x 262144 x 64 doubles, far beyond the 64 MiB scratch
    rc = _call(lib, 64, 64, 64, 0.1, 7, 100.0, 1.0, d.data_ptr(), d.data_ptr(), d.data_ptr(), None)
    assert rc == 6  # RTE_ERR_UNSUPPORTED
    assert b"scratch" in lib.rte_last_error(None)
