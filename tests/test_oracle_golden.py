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
import re

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


def _fim_main_setup(oracle, g, mua_t, mus_t, tiss, stale=None):
    """Forward solve of a FisherInfo_IO main on the oracle (FIM model, reference stop rule).
    stale: the tissue tables (mua, mus) the device kernels still hold.  The SNR and gradient mains
    change tissue values on the host and call populate_info_dev() without keeping its result
    (rte_snr.cu:239, compute_grad_rte.cu:431), so the path integrals and the scatter read the .par
    values while the source, the self-voxel table and the images use the new ones."""
    p = _fim_params(oracle, g)
    mua, mus = np.asarray(mua_t)[tiss], np.asarray(mus_t)[tiss]
    src = oracle.source(p, mua, mus, kind=oracle.SRC_FIM)
    if stale is None:
        out, _, _ = oracle.neumann(p, mua, mus, src, src, 1, oracle.STOP_REFERENCE, n0=2)
        return p, mua, mus, out, mua, mus
    ka, ks = np.asarray(stale[0])[tiss], np.asarray(stale[1])[tiss]
    out, _, _ = oracle.neumann(p, ka, ks, src, src, 1, oracle.STOP_REFERENCE, n0=2, mut_self=mua + mus)
    return p, mua, mus, out, ka, ks


def _fim_axes(g):
    """The mains' voxel-centre coordinates: every axis built from the x extent
    (rte_fim.cu:160-170, rte_snr.cu likewise)."""
    nx, ny, nz = (int(g[k]) for k in ("nx", "ny", "nz"))
    fov = nx * float(g["delX"])
    X = np.arange(nx) * fov / nx - fov / 2 + fov / (2 * nx)
    Y = np.arange(ny) * fov / ny - fov / 2 + fov / (2 * ny)
    Z = np.arange(nz) * fov / nz + fov / (2 * nz)
    return fov, X, Y, Z


def test_fim_fisher_main(oracle):
    """The reference's Fisher main (rte_fim.cu, run in fim_fisher) against its restatement on the oracle:
    tissue map ignored (every voxel tissue 1, mu_a 0.01, mu_s 1), one region of radius fov/(2 nX)
    (a float, squared in float) about (nX/2, nY/2, z index 1), tangent source -C mask(out), Poisson
    F = sum dg^2 / g over the reflection image.  The main prints F with 7 significant digits."""
    run = np.load(os.path.join(GOLD, "fim_fisher_main_10x10x20_L2.npz"))
    g = np.load(os.path.join(GOLD, str(run["base"]) + ".npz"))
    F_ref = float(re.search(r"(\S+) is fisher abs", str(run["stdout"])).group(1))
    nx, ny, nz = (int(g[k]) for k in ("nx", "ny", "nz"))
    tiss = np.ones(nx * ny * nz, np.int64)
    p, mua, mus, out, _, _ = _fim_main_setup(oracle, g, [0.0, 0.01, 0.01, 0.01], [0.0, 1.0, 1.0, 1.0], tiss)
    mag = float(g["mag"])
    _, gref = oracle.images(p, mua, mus, out, 1, mag=mag)
    fov, X, Y, Z = _fim_axes(g)
    rad = np.float32(fov / (2 * nx))
    d2 = (X[None, None, :] - X[nx // 2]) ** 2 + (Y[None, :, None] - Y[ny // 2]) ** 2 + (Z[:, None, None] - Z[1]) ** 2
    mask = ~(d2 > float(rad * rad)).ravel()
    src = np.where(mask[:, None], -out, 0)
    o, _, _ = oracle.neumann(p, mua, mus, src, src, 1, oracle.STOP_REFERENCE, n0=2)
    _, dref = oracle.images(p, mua, mus, o, 1, mag=mag, with_ballistic=0)
    gr, dr = gref.real.ravel(), dref.real.ravel()
    nzp = gr != 0
    F = float(np.sum(dr[nzp] ** 2 / gr[nzp]))
    assert abs(F - F_ref) <= 1e-6 * abs(F_ref), (F, F_ref)


def test_fim_snr_main(oracle):
    """The reference's SNR main (rte_snr.cu, run in fim_snr) against its restatement on the oracle at the
    first lesion depth: a lesion (tissue 2, radius 3 fov/(2 nX) in float) at (nX/2, nY/2, z index 2),
    mu_a 0.35 (signal present) or 0.25 (absent), mu_s 1, on the stale device tissue table;
    SNR^2 = sum (g1 - g0)^2 / g0 over the reflection image, printed with 7 digits.  Two more quirks:
    the z coordinate array is filled only below nX (rte_snr.cu:175-179; the rest read as 0 in this
    run, which puts the deep part of the centre column inside the lesion), and the program never
    reaches the next depth (its loop step `loc_indz = loc_indz++`, rte_snr.cu:219, leaves the index
    unchanged under gcc)."""
    run = np.load(os.path.join(GOLD, "fim_snr_main_10x10x20_L2.npz"))
    g = np.load(os.path.join(GOLD, str(run["base"]) + ".npz"))
    m = re.match(r"(\S+) is snr_sq for (\d+) as z index", str(run["first_line"]))
    snr_ref, lz = float(m.group(1)), int(m.group(2))
    assert lz == 2
    nx, ny = int(g["nx"]), int(g["ny"])
    fov, X, Y, Z = _fim_axes(g)
    Z[nx:] = 0.0
    rad = np.float32(3 * fov / (2 * nx))
    mua_t, mus_t = np.array(g["mua_t"], float), np.array(g["mus_t"], float)
    d2 = (X[None, None, :] - X[nx // 2]) ** 2 + (Y[None, :, None] - Y[ny // 2]) ** 2 + (Z[:, None, None] - Z[lz]) ** 2
    tiss = np.where(d2 < float(rad * rad), 2, 1).ravel()
    imgs = []
    for hyp in (1, 0):
        a, s = mua_t.copy(), mus_t.copy()
        a[2], s[2] = 0.25 + 0.1 * hyp, 1.0
        p, mua, mus, out, _, _ = _fim_main_setup(oracle, g, a, s, tiss, stale=(mua_t, mus_t))
        imgs.append(oracle.images(p, mua, mus, out, 1, mag=float(g["mag"]))[1].real.ravel())
    snr = float(np.sum((imgs[0] - imgs[1]) ** 2 / imgs[1]))
    assert abs(snr - snr_ref) <= 1e-6 * abs(snr_ref), (snr, snr_ref)


def test_fim_region_gradient_main(oracle):
    """The reference's region-gradient main (compute_grad_rte.cu, run in fim_grad, one iteration) against
    its restatement on the oracle: iteration 0 sets tissue 1 to mu_a 0.008, mu_s 0.8; per tissue a tangent
    solve of -C mask(out) (mu_a) and of mask((g^l - 1) out) with the stale-index mask (mu_s) projected to
    the transmission image without the ballistic term, all on the stale device tissue table (the
    .par values; the source, the self-voxel table and the images take the new ones); grad1 = -2 av sum dg/(g - gbar), grad2 = -2 av
    sum (g - gbar) dg over pixels with g or gbar non-zero (av 0.01 as a float for mu_a, 1 for mu_s);
    Residual.out = sum log((gbar - g)^2).  Printed values carry 7 digits; Residual.out is binary."""
    run = np.load(os.path.join(GOLD, "fim_grad_main_10x10x20_L2.npz"))
    g = np.load(os.path.join(GOLD, str(run["base"]) + ".npz"))
    text = str(run["stdout"])
    got1 = [tuple(float(x) for x in m) for m in re.findall(r"mua grad1 = (\S+) musgrad1 = (\S+)", text)]
    got2 = [tuple(float(x) for x in m) for m in re.findall(r"mua grad2 = (\S+) musgrad2 = (\S+)", text)]
    nx, ny = int(g["nx"]), int(g["ny"])
    meas = g["trans"].real.reshape(ny, nx) * float(run["measured_scale"])
    mua_t, mus_t = np.array(g["mua_t"], float), np.array(g["mus_t"], float)
    mua_t[1], mus_t[1] = 0.008, 0.8
    tiss = g["tiss"].astype(np.int64)
    p, mua, mus, out, ka, ks = _fim_main_setup(oracle, g, mua_t, mus_t, tiss,
                                               stale=(np.array(g["mua_t"], float), np.array(g["mus_t"], float)))
    mag = float(g["mag"])
    gbar, _ = oracle.images(p, mua, mus, out, 1, mag=mag)
    gb, gm = gbar.real.ravel(), meas.ravel()
    use = (gm != 0) | (gb != 0)
    L = int(g["nL"])
    lof = np.array([int(np.floor(np.sqrt(c))) for c in range((L + 1) ** 2)])

    def tangent(src):
        o, _, _ = oracle.neumann(p, ka, ks, src, src, 1, oracle.STOP_REFERENCE, n0=2, mut_self=mua + mus)
        return oracle.images(p, mua, mus, o, 1, mag=mag, with_ballistic=0)[0].real.ravel()

    assert len(got1) == len(got2) == len(mua_t) - 1
    for t in range(1, len(mua_t)):
        m = tiss == t
        dga = tangent(np.where(m[:, None], -out, 0))
        resid = gm[use] - gb[use]
        ga = float(np.sum(-2 * np.float32(0.01) * dga[use] / resid))
        ga2 = float(np.sum(-2 * np.float32(0.01) * resid * dga[use]))
        ms = np.ones_like(m)
        if not m.all():
            ms[-1] = False  # the stale-index mu_s mask (compute_grad_rte.cu:356-363)
        dgs = tangent(np.where(ms[:, None], out * (-1.0 + float(g["g"]) ** lof)[None, :], 0))
        gs = float(np.sum(-2 * dgs[use] / resid))
        gs2 = float(np.sum(-2 * resid * dgs[use]))
        for got, want in ((got1[t - 1][0], ga), (got1[t - 1][1], gs), (got2[t - 1][0], ga2), (got2[t - 1][1], gs2)):
            assert abs(got - want) <= 1e-6 * abs(want), (t, got, want)
    diff = gb - gm
    res = float(np.sum(np.log(diff[diff != 0] ** 2)))
    assert abs(run["Residual_out"][0] - res) <= 1e-12 * abs(res)


@pytest.mark.parametrize("case", FIM_CASES[:3])
def test_fim_forward_main_files(rte, tmp_path, case):
    """The image files the reference's forward main (rte.cu, run in fim_host) writes for each case: the
    fixture's images are exactly these (so the GPU program tests compare against the main's own
    output), and rte_write_image produces the same bytes from them (header nY, nX, then the real and
    the imaginary plane, dist.cu:316-345)."""
    files = np.load(os.path.join(GOLD, "fim_forward_main_files.npz"))
    g = np.load(os.path.join(GOLD, case + ".npz"))
    nx, ny = int(g["nx"]), int(g["ny"])
    for k in ("trans", "ref"):
        raw = files[f"{case}__{k}"].tobytes()
        assert np.frombuffer(raw[:8], np.int32).tolist() == [ny, nx]
        v = np.frombuffer(raw[8:], np.float64)
        assert v.size == 2 * nx * ny
        assert np.array_equal(v[:nx * ny] + 1j * v[nx * ny:], g[k].ravel())
        path = str(tmp_path / f"{k}.out")
        rte.rte.write_image(path, g[k].reshape(ny, nx))
        assert open(path, "rb").read() == raw
