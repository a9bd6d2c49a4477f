"""The FP64 oracle against golden outputs of the reference's own code (tests/golden/make_golden.py).

FIM fixtures: the FisherInfo_IO kernels and host code run on the CPU (oracle/_ref/fim_host); the
oracle's FIM mode must reproduce them to rounding (1e-12 relative L2), including the term count of
the reference stop rule, the source, the self-voxel table and both exitance images.
CPU fixtures: the CPU package (oracle/_ref/rte_cpu) images and term count; oracle CPU mode.
Modulated CPU fixtures pin the oracle's complex mu_t (kappa): the package's whole modulated main
(RTE_uniform.c:120-196) is restated on the oracle below and must reproduce every output file.
Downsample fixtures: the reference's downsample_image (dist.cu:271-289) on seeded images.
"""
import os

import numpy as np
import pytest

from conftest import rel

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIM_CASES = ["fim_uniform_10x10x20_L2", "fim_tissues_10x10x20_L2", "fim_shipped_nonuni_20_L1",
             "fim_tissues_10x10x20_L4"]
FIM_APPLY_CASES = [c for c in FIM_CASES if c != "fim_shipped_nonuni_20_L1"]
CPU_CASES = ["cpu_uniform_11_L3", "cpu_isotropic_9_L2", "cpu_uniform_9_L5"]
MOD_CASES = ["cpu_modulated_9_L2", "cpu_modulated_wide_9_L3"]


def _fim_params(O, g):
    nx, ny, nz, L = (int(g[k]) for k in ("nx", "ny", "nz", "nL"))
    dx = float(g["delX"])
    # Geometry extents are floats in the reference; delX (written by the run) already carries that
    return O.params(nx, ny, nz, dx, dx, dx, L, float(g["g"]), float(g["cm"]), float(np.float32(g["prop"])),
                    mode=O.MODE_FIM, ssv=1, x_min=-nx * 0.05, y_min=-ny * 0.05)


@pytest.mark.parametrize("case", FIM_CASES)
def test_fim_forward(oracle, case):
    g = np.load(os.path.join(GOLD, case + ".npz"))
    p = _fim_params(oracle, g)
    tiss = g["tiss"]
    mua, mus = g["mua_t"][tiss], g["mus_t"][tiss]
    src = oracle.source(p, mua, mus, kind=oracle.SRC_FIM)
    assert rel(src, g["src"]) < 1e-13
    out, _, nt = oracle.neumann(p, mua, mus, src, src, 1, oracle.STOP_REFERENCE, n0=2)
    assert nt == int(g["terms"])
    assert rel(out, g["out"]) < 1e-12
    tr, rf = oracle.images(p, mua, mus, out, 1, mag=float(g["mag"]))
    assert rel(tr, g["trans"]) < 1e-12
    assert rel(rf, g["ref"]) < 1e-12


@pytest.mark.parametrize("case", FIM_APPLY_CASES)
def test_fim_single_pass(oracle, case):
    """One prop_abs pass of the reference kernels on a random complex input."""
    g = np.load(os.path.join(GOLD, case + ".npz"))
    p = _fim_params(oracle, g)
    tiss = g["tiss"]
    mua, mus = g["mua_t"][tiss], g["mus_t"][tiss]
    N, C = tiss.size, (int(g["nL"]) + 1) ** 2
    rng = np.random.default_rng(int(g["apply_seed"]))
    W = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
    for flag, fs in ((1, 1), (1, 0), (0, 1)):
        got = oracle.apply(p, mua, mus, W, flag, fs)
        ref = g[f"apply_{flag}{fs}"]
        assert rel(got, ref) < 1e-12, (flag, fs)


@pytest.mark.parametrize("case", FIM_CASES)
def test_fim_self_voxel_table(oracle, case):
    g = np.load(os.path.join(GOLD, case + ".npz"))
    L = int(g["nL"])
    dx = float(g["delX"])
    for t in range(1, len(g["mua_t"])):
        mut = float(g["mua_t"][t] + g["mus_t"][t])
        D = oracle.self_matrix(0, L, 1, mut, dx, dx, dx)
        assert rel(D, g["diag"][:, :, t]) < 1e-13


@pytest.mark.parametrize("case", CPU_CASES)
def test_cpu_package_forward(oracle, case):
    g = np.load(os.path.join(GOLD, case + ".npz"))
    n, L = int(g["n"]), int(g["nL"])
    N = n ** 3
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, float(g["g"]), 1.0, 10.0, mode=oracle.MODE_CPU,
                      x_min=-n * 0.05, y_min=-n * 0.05)
    mua, mus = np.full(N, float(g["mua"])), np.full(N, float(g["mus"]))
    r = oracle.forward(p, mua, mus, src_kind=oracle.SRC_CPU, img_mode=2, stop_rule=oracle.STOP_REFERENCE, n0=1,
                       diam=float(g["diam"]))
    assert r["terms"] == int(g["terms"])
    assert rel(r["trans"], g["trans"]) < 1e-12
    assert rel(r["ref"], g["ref"]) < 1e-12


@pytest.mark.parametrize("case", CPU_CASES)
def test_cpu_package_side_faces_and_photons(rte, oracle, case):
    """rte_cpu_face_outputs on the oracle's final distribution reproduces the CPU package's side-face
    images (1e-12) and its printed photon number (6 decimals) for the same input."""
    g = np.load(os.path.join(GOLD, case + ".npz"))
    n, L = int(g["n"]), int(g["nL"])
    N = n ** 3
    lo, hi = -n * 0.05, n * 0.05
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, float(g["g"]), 1.0, 10.0, mode=oracle.MODE_CPU, x_min=lo, y_min=lo)
    mua, mus = np.full(N, float(g["mua"])), np.full(N, float(g["mus"]))
    r = oracle.forward(p, mua, mus, src_kind=oracle.SRC_CPU, img_mode=2, stop_rule=oracle.STOP_REFERENCE, n0=1,
                       diam=float(g["diam"]))
    src = rte.Source(diam=float(g["diam"]), kind=rte.SRC_CPU)
    sides, ph = rte.rte.cpu_face_outputs(r["out"], n, n, n, L, lo, hi, lo, hi, 0.0, n * 0.1, src,
                                         float(g["mua"]) + float(g["mus"]))
    for q in range(4):
        # the package writes each side image through its z-face writer: header (nX, nY), then the
        # buffer (index k + u*nZ) in order -- for these cubic grids the same array read as (nY, nX)
        assert rel(sides[q].ravel(), g[f"side{q + 1}"].ravel()) < 1e-12, q
    assert abs(ph.real - float(g["photons"])) < 5e-7


def _cpu_stop(p, fi, n, W, out):
    """StopIteration of the CPU package (Kernels_selfsub.c:1184-1220) on the layer z = nZ-1."""
    N2 = p.nx * p.ny
    sw = W.reshape(p.nz, N2, -1)[-1].real.sum()
    so = out.reshape(p.nz, N2, -1)[-1].real.sum()
    hi = 0.0
    if n > 1:
        if so == 0.0:
            return True, fi
        hi = 1.0 - (sw / so) * (1.0 / (1.0 - (sw / so) / fi))
        fi = sw / so
        if hi > 1.0 or hi < 0.0:
            hi = 0.0
    return hi > 0.9999, fi


def cpu_package_main(O, g):
    """The CPU package's main on the oracle, output for output (RTE_uniform.c:64-196): steady state,
    then with modulation != 0 the modulated continuation exactly as written (the second source built
    with the real mu_a and the magnitude divided by the column count again, Dist.c:1113-1114; the
    modulated terms added to the steady-state result; out2 = A src; CombineOuts)."""
    n, L = int(g["n"]), int(g["nL"])
    N, C = n ** 3, (L + 1) ** 2
    lo = -n * 0.05
    mod = float(g["modulation"]) if "modulation" in g else 0.0
    mag = float(g["mag"]) if "mag" in g else 1.0
    diam = float(g["diam"])
    p0 = O.params(n, n, n, 0.1, 0.1, 0.1, L, float(g["g"]), 1.0, 10.0, mode=O.MODE_CPU, x_min=lo, y_min=lo)
    pk = O.params(n, n, n, 0.1, 0.1, 0.1, L, float(g["g"]), 1.0, 10.0, mode=O.MODE_CPU, x_min=lo, y_min=lo,
                  kappa=mod)  # c = n = 1: kappa = modulation
    mua, mus = np.full(N, float(g["mua"])), np.full(N, float(g["mus"]))
    r = O.forward(p0, mua, mus, src_kind=O.SRC_CPU, img_mode=2, stop_rule=O.STOP_REFERENCE, n0=1, diam=diam, mag=mag)
    xs = (np.arange(n) + 0.5) * 0.1 + lo
    X, Y = np.meshgrid(xs, xs)
    cols = int((np.sqrt(X ** 2 + Y ** 2) <= (diam + 1e-16) / 2).sum())
    mag1 = mag / cols  # source->mag after GenerateSourceBeam
    out = r["out"].copy()
    out2 = out
    terms_mod = 0
    p_img, mag_img = p0, mag1
    if mod != 0.0:
        src = O.source(p0, mua, mus, diam=diam, mag=mag1, kind=O.SRC_CPU)  # real mu_a, mag1 / cols
        W, fi, k = src.copy(), 1.0, 1
        flag = 1 if float(g["g"]) != 0.0 else 0
        while True:
            stop, fi = _cpu_stop(p0, fi, k, W, out)
            if stop:
                break
            W = O.apply(pk, mua, mus, W, flag, 1)
            out = out + W
            k += 1
        terms_mod = k - 1
        out2 = O.apply(pk, mua, mus, src, 1, 0)
        p_img, mag_img = pk, mag1 / cols
    # phase image of out2 (Dist.c:71-131): diffuse transmission with weight 1/(100-1), ballistic, degrees
    tr_d, _ = O.images(p_img, mua, mus, out2, 2, diam=diam, mag=mag_img * cols, with_ballistic=0)
    zs = (n - 1) * 0.1 + 0.05
    ball = mag_img * np.exp(-complex(float(g["mua"]) + float(g["mus"]), mod) * (zs + 0.05))
    phase = np.angle(tr_d * 100.0 / 99.0 + np.where(np.sqrt(X ** 2 + Y ** 2) <= diam / 2, ball, 0.0)) * 180 / np.pi
    if mod != 0.0:
        out = 0.5 * out + 0.25 * out2 + 0.25 * np.conj(out2)
        tr, rf = O.images(p_img, mua, mus, out, 2, diam=diam, mag=mag_img * cols)
    else:
        tr, rf = r["trans"], r["ref"]
    return dict(out=out, trans=tr, ref=rf, phase=phase, terms=r["terms"], terms_mod=terms_mod, mag_img=mag_img,
                mut=complex(float(g["mua"]) + float(g["mus"]), mod))


@pytest.mark.parametrize("case", CPU_CASES + MOD_CASES)
def test_cpu_package_main_with_modulation(rte, oracle, case):
    """The oracle restatement of the CPU package's main reproduces every file the package writes:
    transmission / reflection (1e-12), phase image (1e-10 degrees), side faces (1e-12), photon
    number (printed to 6 decimals) and both term counts."""
    g = np.load(os.path.join(GOLD, case + ".npz"))
    n, L = int(g["n"]), int(g["nL"])
    r = cpu_package_main(oracle, g)
    assert r["terms"] == int(g["terms"])
    assert r["terms_mod"] == int(g["terms_mod"])
    assert rel(r["trans"], g["trans"]) < 1e-12
    assert rel(r["ref"], g["ref"]) < 1e-12
    assert np.abs(r["phase"] - g["phase"]).max() < 1e-10
    lo, hi = -n * 0.05, n * 0.05
    src = rte.Source(diam=float(g["diam"]), mag=r["mag_img"], kind=rte.SRC_CPU)
    sides, ph = rte.rte.cpu_face_outputs(r["out"], n, n, n, L, lo, hi, lo, hi, 0.0, n * 0.1, src, r["mut"])
    for q in range(4):
        assert rel(sides[q].ravel(), g[f"side{q + 1}"].ravel()) < 1e-12, q
    assert abs(ph.real - float(g["photons"])) < 5e-7


@pytest.mark.parametrize("case", ["fim_downsample_20x20", "fim_downsample_24x18"])
def test_fim_downsample_image(rte, oracle, case):
    """downsample_image as the reference's own function computed it (run inside fim_host with the
    allocator's zero fill), bit-exact: the oracle's loop restatement and the library's
    rte_downsample_image, on a square and a non-square image and factors that leave a ragged edge."""
    g = np.load(os.path.join(GOLD, case + ".npz"))
    nx, ny, img = int(g["nx"]), int(g["ny"]), g["img"]
    for ds in (int(v) for v in g["factors"]):
        ref = g[f"ds{ds}"]
        assert np.array_equal(oracle.downsample_image(img, nx, ny, ds), ref)
        # the library takes the image as the (nY, nX) array of the y*nX + x layout
        assert np.array_equal(rte.downsample_image(img.reshape(ny, nx), ds).ravel(), ref)
