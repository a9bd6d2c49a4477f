"""The reference's programs rebuilt over the library (doi_b200/bin): rte_gpu on .par files whose
outputs the reference's own code produced (tests/golden, FisherInfo_IO run on the CPU), rte_fim and
rte_inv against the FP64 oracle's tangent solves.  FIM-model tolerance 1e-6 (the reference walks paths
with float alpha, the library with exact crossings)."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["fim_uniform_10x10x20_L2", "fim_tissues_10x10x20_L2", "fim_shipped_nonuni_20_L1"]


def _exe(rte, name):
    return os.path.join(os.path.dirname(rte.rte.LIB_PATH), "..", "bin", name)


def _par(g, d, extra="", alg=""):
    text = str(g["par"])
    text = re.sub(r"(?im)^TissMapFile\s*=.*$", f"TissMapFile = {d}/tiss.bin", text)
    for k, f in (("TransFile", "trans.out"), ("ReflectFile", "ref.out"), ("PhaseFile", "phase.out")):
        text = re.sub(rf"(?im)^{k}\s*=.*$", f"{k} = {d}/{f}", text)
    text = text.replace("[Runtime]", "[Runtime]\n" + extra, 1)
    text = text.replace("[Algorithm]", "[Algorithm]\n" + alg, 1)
    g["tiss"].astype(np.uint8).tofile(os.path.join(d, "tiss.bin"))
    p = os.path.join(d, "case.par")
    open(p, "w").write(text)
    return p


def _read_img(path):
    b = open(path, "rb").read()
    ny, nx = struct.unpack("2i", b[:8])
    v = np.frombuffer(b[8:], np.float64)
    return (v[: nx * ny] + 1j * v[nx * ny:2 * nx * ny]).reshape(ny, nx)


@pytest.mark.parametrize("case", CASES)
def test_rte_gpu_matches_reference_outputs(rte, tmp_path, case):
    g = np.load(os.path.join(GOLD, case + ".npz"))
    d = str(tmp_path)
    r = subprocess.run([_exe(rte, "rte_gpu"), _par(g, d)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    assert f"Neumann series: {int(g['terms'])} terms" in r.stdout
    tr, rf = _read_img(os.path.join(d, "trans.out")), _read_img(os.path.join(d, "ref.out"))
    assert rel(tr, g["trans"].reshape(tr.shape)) < 1e-6
    assert rel(rf, g["ref"].reshape(rf.shape)) < 1e-6
    b = open(os.path.join(d, "phase.out"), "rb").read()
    ny, nx = struct.unpack("2i", b[:8])
    ph = np.frombuffer(b[8:], np.float64).reshape(ny, nx)
    assert np.all(np.isfinite(ph)) and ph.shape == tr.shape


@pytest.mark.parametrize("case", CASES)
def test_reference_main_with_library_neumann(rte, tmp_path, case):
    """The reference's own forward main (FisherInfo_IO/src/rte.cu, unchanged: its parameter reading, source,
    images and files) linked with the library's Neumann() shim (doi_b200/shim/neumann_b200.cu) in place of
    neumann.cu, as a maintainer would build it (oracle/build.sh makes oracle/_ref/fim_shim): its TransFile /
    ReflectFile equal the images of the reference main run as shipped (the golden fixtures, pinned to that
    main's own files by test_fim_forward_main_files) to 1e-6."""
    exe = os.path.join(os.path.dirname(GOLD), "..", "oracle", "_ref", "fim_shim")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/fim_shim is built by oracle/build.sh where the reference tree is present")
    g = np.load(os.path.join(GOLD, case + ".npz"))
    d = str(tmp_path)
    r = subprocess.run([exe, _par(g, d)], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    tr, rf = _read_img(os.path.join(d, "trans.out")), _read_img(os.path.join(d, "ref.out"))
    assert rel(tr, g["trans"].reshape(tr.shape)) < 1e-6, rel(tr, g["trans"].reshape(tr.shape))
    assert rel(rf, g["ref"].reshape(rf.shape)) < 1e-6, rel(rf, g["ref"].reshape(rf.shape))


def _oracle_setup(oracle, g, mua_t, mus_t, tiss):
    nx, ny, nz, L = (int(g[k]) for k in ("nx", "ny", "nz", "nL"))
    dx = float(g["delX"])
    p = oracle.params(nx, ny, nz, dx, dx, dx, L, float(g["g"]), float(g["cm"]), float(np.float32(g["prop"])),
                      mode=oracle.MODE_FIM, ssv=1, x_min=-nx * 0.05, y_min=-ny * 0.05)
    mua, mus = np.asarray(mua_t)[tiss], np.asarray(mus_t)[tiss]
    src = oracle.source(p, mua, mus, kind=oracle.SRC_FIM)
    out, _, _ = oracle.neumann(p, mua, mus, src, src, 1, oracle.STOP_REFERENCE, n0=2)
    return p, mua, mus, out


def _tangent(oracle, p, mua, mus, src, mag):
    o, _, _ = oracle.neumann(p, mua, mus, src, src, 1, oracle.STOP_REFERENCE, n0=2)
    return oracle.images(p, mua, mus, o, 1, mag=mag, with_ballistic=0)


def test_rte_fim_matches_oracle(rte, oracle, tmp_path):
    g = np.load(os.path.join(GOLD, "fim_tissues_10x10x20_L2.npz"))
    d = str(tmp_path)
    r = subprocess.run([_exe(rte, "rte_fim"), _par(g, d)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    F = float(re.search(r"([-+0-9.eE]+) is fisher abs", r.stdout).group(1))
    # the main: tissue map ignored (all tissue 1), mu_a 0.01, mu_s 1, one-voxel region at (nX/2, nY/2, 1)
    nx, ny, nz = (int(g[k]) for k in ("nx", "ny", "nz"))
    tiss = np.ones(nx * ny * nz, np.int64)
    p, mua, mus, out = _oracle_setup(oracle, g, [0.0, 0.01, 0.01, 0.01], [0.0, 1.0, 1.0, 1.0], tiss)
    mag = float(g["mag"])
    _, gref = oracle.images(p, mua, mus, out, 1, mag=mag)
    # the main's region (rte_fim.cu:135-206): coordinates on the x extent for every axis, radius
    # fov/(2 nX) as float, squared in float
    fov = nx * float(g["delX"])
    X = np.arange(nx) * fov / nx - fov / 2 + fov / (2 * nx)
    Y = np.arange(ny) * fov / ny - fov / 2 + fov / (2 * ny)
    Z = np.arange(nz) * fov / nz + fov / (2 * nz)
    rad = np.float32(fov / (2 * nx))
    d2 = (X[None, None, :] - X[nx // 2]) ** 2 + (Y[None, :, None] - Y[ny // 2]) ** 2 + (Z[:, None, None] - Z[1]) ** 2
    mask = ~(d2 > float(rad * rad)).ravel()
    src = np.where(mask[:, None], -out, 0)
    _, dref = _tangent(oracle, p, mua, mus, src, mag)
    gr, dr = gref.real.ravel(), dref.real.ravel()
    nzp = gr != 0
    F_ref = float(np.sum(dr[nzp] ** 2 / gr[nzp]))
    assert abs(F - F_ref) <= 1e-5 * abs(F_ref)


def test_rte_inv_matches_oracle(rte, oracle, tmp_path):
    g = np.load(os.path.join(GOLD, "fim_tissues_10x10x20_L2.npz"))
    d = str(tmp_path)
    nx, ny = int(g["nx"]), int(g["ny"])
    meas = (g["trans"].real.reshape(ny, nx) * 1.05).astype(np.float64)
    with open(os.path.join(d, "g.out"), "wb") as f:
        f.write(struct.pack("2i", ny, nx))
        f.write(meas.tobytes())
    par = _par(g, d, extra=f"gFile = {d}/g.out\nnumIterations = 1\n", alg="ReferenceQuirks = 0\n")
    r = subprocess.run([_exe(rte, "rte_inv"), par], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    got = [tuple(float(x) for x in m) for m in re.findall(r"mua grad1 = (\S+) musgrad1 = (\S+)", r.stdout)]
    got2 = [tuple(float(x) for x in m) for m in re.findall(r"mua grad2 = (\S+) musgrad2 = (\S+)", r.stdout)]
    # iteration 0 of the main sets tissue 1 to mu_a 0.008, mu_s 0.8 (compute_grad_rte.cu:207-209)
    mua_t, mus_t = np.array(g["mua_t"], float), np.array(g["mus_t"], float)
    mua_t[1], mus_t[1] = 0.008, 0.8
    tiss = g["tiss"].astype(np.int64)
    p, mua, mus, out = _oracle_setup(oracle, g, mua_t, mus_t, tiss)
    mag = float(g["mag"])
    gbar, _ = oracle.images(p, mua, mus, out, 1, mag=mag)
    gb, gm = gbar.real.ravel(), meas.ravel()
    use = (gm != 0) | (gb != 0)
    L = int(g["nL"])
    lof = np.array([int(np.floor(np.sqrt(c))) for c in range((L + 1) ** 2)])
    for t in range(1, len(mua_t)):
        m = tiss == t
        dga, _ = _tangent(oracle, p, mua, mus, np.where(m[:, None], -out, 0), mag)
        resid = gm[use] - gb[use]
        ga = float(np.sum(-2 * np.float32(0.01) * dga.real.ravel()[use] / resid))
        ga2 = float(np.sum(-2 * np.float32(0.01) * resid * dga.real.ravel()[use]))
        ms = np.ones_like(m)
        if not m.all():
            ms[-1] = False  # the reference's stale-index mu_s mask
        fac = -1.0 + float(g["g"]) ** lof
        dgs, _ = _tangent(oracle, p, mua, mus, np.where(ms[:, None], out * fac[None, :], 0), mag)
        gs = float(np.sum(-2 * 1.0 * dgs.real.ravel()[use] / resid))
        gs2 = float(np.sum(-2 * 1.0 * resid * dgs.real.ravel()[use]))
        # grad2 (misfit-weighted) to 1e-5; grad1 divides by the per-pixel residual, which amplifies the
        # model's 1e-7 path-integral difference where a residual is small: 1e-3
        assert abs(got2[t - 1][0] - ga2) <= 1e-5 * abs(ga2), (t, got2[t - 1][0], ga2)
        assert abs(got2[t - 1][1] - gs2) <= 1e-5 * abs(gs2), (t, got2[t - 1][1], gs2)
        assert abs(got[t - 1][0] - ga) <= 1e-3 * abs(ga), (t, got[t - 1][0], ga)
        assert abs(got[t - 1][1] - gs) <= 1e-3 * abs(gs), (t, got[t - 1][1], gs)
    assert os.path.getsize(os.path.join(d, "Residual.out")) == 8


@pytest.mark.parametrize("case", ["cpu_uniform_11_L3", "cpu_isotropic_9_L2", "cpu_modulated_9_L2",
                                  "cpu_modulated_wide_9_L3"])
def test_rte_gpu_on_cpu_package_files(rte, tmp_path, case):
    """A CPU-package parameter file (uniform medium keys): same images, phase image, side-face files and
    printed photon number as the CPU package itself, with intensity modulation (its modulated
    continuation and CombineOuts, RTE_uniform.c:120-196) and a beam over several columns."""
    g = np.load(os.path.join(GOLD, case + ".npz"))
    d = str(tmp_path)
    text = str(g["par"])
    for k, f in (("TransFile", "trans.out"), ("ReflectFile", "ref.out"), ("PhaseFile", "phase.out")):
        text = re.sub(rf"(?im)^{k}\s*=.*$", f"{k} = {d}/{f}", text)
    par = os.path.join(d, "c.par")
    open(par, "w").write(text)
    r = subprocess.run([_exe(rte, "rte_gpu"), par], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    assert f"Neumann series: {int(g['terms'])} terms" in r.stdout
    assert rel(_read_img(os.path.join(d, "trans.out")), g["trans"]) < 1e-10
    assert rel(_read_img(os.path.join(d, "ref.out")), g["ref"]) < 1e-10
    for q, ax in ((1, "-X"), (2, "+X"), (3, "-Y"), (4, "+Y")):
        assert rel(_read_img(os.path.join(d, f"SideFace{q}({ax}).out")), g[f"side{q}"]) < 1e-10
    ph = float(re.search(r"Number of photons total: (\S+)", r.stdout).group(1))
    assert abs(ph - float(g["photons"])) < 2e-6
    b = open(os.path.join(d, "phase.out"), "rb").read()  # OutputPhaseImage: nX, nY, values x fastest
    nx, ny = struct.unpack("2i", b[:8])
    phase = np.frombuffer(b[8:], np.float64).reshape(ny, nx)
    assert np.abs(phase - g["phase"]).max() < 1e-8
    if float(g["modulation"]) != 0.0:
        assert f"Neumann series (modulated): {int(g['terms_mod'])} terms" in r.stdout


def test_rte_snr_matches_oracle(rte, oracle, tmp_path):
    g = np.load(os.path.join(GOLD, "fim_tissues_10x10x20_L2.npz"))
    d = str(tmp_path)
    nx, ny, nz = (int(g[k]) for k in ("nx", "ny", "nz"))
    with open(os.path.join(d, "g.out"), "wb") as f:  # the program insists on a measured image
        f.write(struct.pack("2i", ny, nx) + np.zeros(nx * ny).tobytes())
    par = _par(g, d, extra=f"gFile = {d}/g.out\n", alg="ReferenceQuirks = 0\n")
    r = subprocess.run([_exe(rte, "rte_snr"), par], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    snr = np.fromfile(os.path.join(d, "snr_terms.dat"), np.float64)
    # depths 2..15 are filled (the reflection image of this model can be negative, and so can the
    # sums); the rest of the file stays zero
    assert snr.size == nz - 2 and np.all(snr[:14] != 0) and np.all(snr[14:] == 0)
    fov = nx * float(g["delX"])
    X = np.arange(nx) * fov / nx - fov / 2 + fov / (2 * nx)
    Y = np.arange(ny) * fov / ny - fov / 2 + fov / (2 * ny)
    Z = np.arange(nz) * fov / nz + fov / (2 * nz)
    rad = np.float32(3 * fov / (2 * nx))
    mua_t, mus_t = np.array(g["mua_t"], float), np.array(g["mus_t"], float)
    for lz in (2, 5):
        d2 = (X[None, None, :] - X[nx // 2]) ** 2 + (Y[None, :, None] - Y[ny // 2]) ** 2 + (Z[:, None, None] - Z[lz]) ** 2
        tiss = np.where(d2 < float(rad * rad), 2, 1).ravel()
        imgs = []
        for hyp in (1, 0):
            a, s = mua_t.copy(), mus_t.copy()
            a[2], s[2] = 0.25 + 0.1 * hyp, 1.0
            p, mua, mus, out = _oracle_setup(oracle, g, a, s, tiss)
            imgs.append(oracle.images(p, mua, mus, out, 1, mag=float(g["mag"]))[1].real.ravel())
        ref = float(np.sum((imgs[0] - imgs[1]) ** 2 / imgs[1]))
        assert abs(snr[lz - 2] - ref) <= 1e-5 * abs(ref), (lz, snr[lz - 2], ref)


def test_rte_inv_reproduces_reference_main(rte, tmp_path):
    """rte_inv with its defaults (ReferenceQuirks = 1: kernels on the .par tissue table, the rest on the swept
    values, as the reference's main leaves its device table) prints the values the reference's own
    region-gradient main (compute_grad_rte.cu, run unchanged on the CPU for the fixture) printed for the same
    .par file and measured image, and writes the same Residual.out.  grad2 to 1e-5, grad1 (which divides by
    per-pixel residuals, amplifying the 1e-7 path-integral difference of the table model) to 1e-3."""
    run = np.load(os.path.join(GOLD, "fim_grad_main_10x10x20_L2.npz"))
    g = np.load(os.path.join(GOLD, str(run["base"]) + ".npz"))
    d = str(tmp_path)
    nx, ny = int(g["nx"]), int(g["ny"])
    meas = (g["trans"].real.reshape(ny, nx) * float(run["measured_scale"])).astype(np.float64)
    with open(os.path.join(d, "g.out"), "wb") as f:
        f.write(struct.pack("2i", ny, nx) + meas.tobytes())
    par = _par(g, d, extra=f"gFile = {d}/g.out\nnumIterations = 1\n")
    r = subprocess.run([_exe(rte, "rte_inv"), par], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    pat1, pat2 = r"mua grad1 = (\S+) musgrad1 = (\S+)", r"mua grad2 = (\S+) musgrad2 = (\S+)"
    got1 = [tuple(float(x) for x in m) for m in re.findall(pat1, r.stdout)]
    got2 = [tuple(float(x) for x in m) for m in re.findall(pat2, r.stdout)]
    ref1 = [tuple(float(x) for x in m) for m in re.findall(pat1, str(run["stdout"]))]
    ref2 = [tuple(float(x) for x in m) for m in re.findall(pat2, str(run["stdout"]))]
    assert len(got1) == len(ref1) > 0 and len(got2) == len(ref2)
    for a, b in zip(got2, ref2):
        for x, y in zip(a, b):
            assert abs(x - y) <= 1e-5 * abs(y), (x, y)
    for a, b in zip(got1, ref1):
        for x, y in zip(a, b):
            assert abs(x - y) <= 1e-3 * abs(y), (x, y)
    res = np.fromfile(os.path.join(d, "Residual.out"), np.float64)
    assert abs(res[0] - run["Residual_out"][0]) <= 1e-6 * abs(run["Residual_out"][0])


def test_rte_snr_reproduces_reference_main(rte, tmp_path):
    """rte_snr with its defaults (ReferenceQuirks = 1: kernels on the .par tissue table, and z coordinates from
    index nX on read as 0, as in the reference's run) gives at the first lesion depth the SNR^2 the
    reference's own SNR main printed (the only depth it reaches: its loop step never advances) to 1e-5."""
    run = np.load(os.path.join(GOLD, "fim_snr_main_10x10x20_L2.npz"))
    g = np.load(os.path.join(GOLD, str(run["base"]) + ".npz"))
    m = re.match(r"(\S+) is snr_sq for (\d+) as z index", str(run["first_line"]))
    snr_ref, lz = float(m.group(1)), int(m.group(2))
    d = str(tmp_path)
    nx, ny = int(g["nx"]), int(g["ny"])
    with open(os.path.join(d, "g.out"), "wb") as f:
        f.write(struct.pack("2i", ny, nx) + np.zeros(nx * ny).tobytes())
    par = _par(g, d, extra=f"gFile = {d}/g.out\n")
    r = subprocess.run([_exe(rte, "rte_snr"), par], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout
    snr = np.fromfile(os.path.join(d, "snr_terms.dat"), np.float64)
    assert abs(snr[lz - 2] - snr_ref) <= 1e-5 * abs(snr_ref), (snr[lz - 2], snr_ref)
