"""The reference's parameter-file dialect and file formats through the library (no GPU needed):
iniparser rules (FisherInfo_IO/src/iniparser.cu:455-620), the loaders' derived inputs
(FisherInfo_IO/src/inits.cu:22-269, rte.cu:116-119; CPU package/src/Inits.c:24-131), and the image
file layouts (dist.cu:291-345, CPU package/src/Dist.c:16-40, compute_grad_rte.cu:151-161)."""
import os
import struct

import numpy as np
import pytest


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_ini_dialect(rte, tmp_path):
    path = _write(tmp_path, "a.par", """# comment line
[Geometry]
nX = 0x10          ; hex as strtol base 0
NY=012
nZ = 7 # trailing comment
xMin = -1.5
[ALGORITHM]
nL = 3
name = "quoted ; value"
other = 'single # quoted'
empty =
long = 1\\
2
nL = 4
""")
    par = rte.rte.ParFile(path)
    assert par.get_int("Geometry:nX") == 16
    assert par.get_int("geometry:ny") == 10       # octal, case-insensitive lookup
    assert par.get_int("Geometry:nZ") == 7
    assert par.get_double("GEOMETRY:XMIN") == -1.5
    assert par.get("Algorithm:name") == "quoted ; value"
    assert par.get("Algorithm:other") == "single # quoted"
    assert par.get("Algorithm:empty") == ""
    assert par.get("Algorithm:long") == "12"
    assert par.get_int("Algorithm:nL") == 4        # last repeat wins
    assert par.get("Algorithm:missing", "dflt") == "dflt"
    assert par.get_double("Source:posX", 0.25) == 0.25


FIM_PAR = """[Runtime]
TransFile = {d}/trans.out
ReflectFile = {d}/ref.out
gFile = {d}/g.out
numIterations = 3
[Algorithm]
nL = 2
[Geometry]
nX = 10
nY = 10
nZ = 20
xMin = -0.5
xMax = 0.5
yMin = -0.5
yMax = 0.5
zMin = 0
zMax = 2.0
propThresh = 10.1
[Phantom]
NoTiss = 2
TissMapFile = {d}/map.bin
TissAbs1 = 0.02
TissSc2 = 1.5
g = 0.8
n = 1.4
[Source]
posX = 0.1
magnitude = 2.0
"""


def test_fim_style_problem(rte, tmp_path):
    d = str(tmp_path)
    tiss = np.random.default_rng(0).integers(0, 3, 2000).astype(np.uint8)
    tiss.tofile(os.path.join(d, "map.bin"))
    pr = rte.rte.ParFile(_write(tmp_path, "f.par", FIM_PAR.format(d=d))).problem()
    assert (pr["nx"], pr["ny"], pr["nz"], pr["nL"]) == (10, 10, 20, 2)
    assert pr["style"] == 0 and pr["model"] == rte.MODEL_FIM and pr["source"]["kind"] == rte.SRC_FIM
    assert pr["x_min"] == np.float32(-0.5) and pr["z_max"] == np.float32(2.0)
    assert pr["prop_thresh"] == float(np.float32(10.1))            # float in the reference's Geometry
    assert pr["g"] == 0.8 and pr["n"] == 1.4 and pr["c"] == 1.0 and pr["self_sub_vox"] == 1
    assert pr["ntypes"] == 3
    assert list(pr["mua_tab"]) == [0.0, 0.02, 0.01] and list(pr["mus_tab"]) == [0.0, 1.0, 1.5]  # defaults 0.01 / 1.0
    assert np.array_equal(pr["tiss"], tiss)
    mut = (pr["mua_tab"] + pr["mus_tab"])[tiss].mean()
    assert abs(pr["mut_mean"] - mut) < 1e-14
    # rte.cu:116-119: mu_t mean * depth > 4 -> propThresh = -log(0.01) / mu_t mean (float)
    expect = float(np.float32(-np.log(0.01) / mut)) if mut * 2.0 > 4 else pr["prop_thresh"]
    assert pr["diffuse_prop_thresh"] == expect
    assert pr["source"]["pos_x"] == 0.1 and pr["source"]["mag"] == 2.0 and pr["source"]["diam"] == 0.2
    assert pr["stop"]["rule"] == rte.STOP_REFERENCE and pr["num_iterations"] == 3
    assert pr["trans_file"] == os.path.join(d, "trans.out") and pr["g_file"] == os.path.join(d, "g.out")
    # LoadPhantom(ini, 0): no map, every voxel tissue 1
    pr0 = rte.rte.ParFile(_write(tmp_path, "f0.par", FIM_PAR.format(d=d + "/missing"))).problem(read_map=False)
    assert (pr0["tiss"] == 1).all()
    with pytest.raises(rte.RteError):
        rte.rte.ParFile(_write(tmp_path, "f1.par", FIM_PAR.format(d=d + "/missing"))).problem()


def test_cpu_style_and_new_keys(rte, tmp_path):
    text = """[Algorithm]
nL = 3
Precision = mixed
StopRule = rel_l2
MaxTerms = 30
Tol = 1e-7
DetectorBins = 11
[Geometry]
nX = 11
nY = 11
nZ = 11
xMin = -0.55
xMax = 0.55
yMin = -0.55
yMax = 0.55
zMin = 0
zMax = 1.1
propThresh = 10
[Phantom]
mua = 0.01
mus = 1.0
g = 0.8
n = 1.0
[Source]
diam = 0.1
Kind = point
Face = 3
modulation = 0.25
"""
    pr = rte.rte.ParFile(_write(tmp_path, "c.par", text)).problem()
    assert pr["style"] == 1 and pr["model"] == rte.MODEL_CPU and pr["c"] == 2.9979e10
    assert pr["x_min"] == -0.55 and pr["self_sub_vox"] == 1 and pr["precision"] == rte.PREC_MIXED
    assert pr["stop"] == {"rule": rte.STOP_REL_L2, "max_terms": 30, "tol": 1e-7} and pr["detector_bins"] == 11
    assert pr["source"]["kind"] == rte.SRC_POINT and pr["source"]["face"] == 3
    assert pr["source"]["modulation"] == 0.25
    assert (pr["tiss"] == 1).all() and list(pr["mua_tab"]) == [0.0, 0.01]


def test_image_files(rte, tmp_path):
    rng = np.random.default_rng(1)
    img = rng.standard_normal((4, 6)) + 1j * rng.standard_normal((4, 6))  # ny = 4, nx = 6
    for cpu in (False, True):
        p = str(tmp_path / f"i{int(cpu)}.out")
        rte.rte.write_image(p, img, cpu_layout=cpu)
        b = open(p, "rb").read()
        assert struct.unpack("2i", b[:8]) == ((6, 4) if cpu else (4, 6))
        v = np.frombuffer(b[8:], np.float64)
        assert np.array_equal(v[:24], img.real.ravel()) and np.array_equal(v[24:], img.imag.ravel())
    g = rte.rte.read_image(str(tmp_path / "i0.out"), 6, 4)  # a measured image: the real plane
    assert np.array_equal(g, img.real)
    for cpu in (False, True):  # phase images: dist.cu:291-314 (nY, nX) and Dist.c:47-65 (nX, nY)
        p = str(tmp_path / f"p{int(cpu)}.out")
        rte.rte.write_phase_image(p, img.real, cpu_layout=cpu)
        b = open(p, "rb").read()
        assert struct.unpack("2i", b[:8]) == ((6, 4) if cpu else (4, 6)) and len(b) == 8 + 24 * 8
        assert np.array_equal(np.frombuffer(b[8:], np.float64), img.real.ravel())


@pytest.mark.parametrize("nx,ny,ds", [(20, 20, 2), (20, 20, 5), (21, 21, 4), (12, 18, 3), (7, 9, 1), (5, 5, 5)])
def test_downsample_image(rte, oracle, nx, ny, ds):
    """downsample_image (FisherInfo_IO/src/dist.cu:271-289) through the C ABI: bit-exact against the
    oracle's loop restatement, including the reference's row-length-nY indexing on non-square images
    and the dropped ragged edge; on square images whose side ds divides, the block sums keep the total."""
    rng = np.random.default_rng(nx * 100 + ny * 10 + ds)
    img = rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))
    got = rte.downsample_image(img, ds)
    ref = oracle.downsample_image(img, nx, ny, ds)
    assert got.shape == (nx // ds, ny // ds)
    assert np.array_equal(got.ravel(), ref)
    if nx == ny and nx % ds == 0:
        blocks = img.reshape(ny // ds, ds, nx // ds, ds).sum(axis=(1, 3))
        assert np.allclose(got, blocks, rtol=1e-13, atol=1e-13)
        assert abs(got.sum() - img.sum()) < 1e-11
    if ds == 1:
        assert np.array_equal(got.ravel(), img.ravel())


def test_downsample_image_rejects_bad_factor(rte):
    img = np.ones((4, 6), np.complex128)
    for ds in (0, -1, 5, 7):
        with pytest.raises(rte.RteError):
            rte.downsample_image(img, ds)


def test_cli_usage_without_device(rte):
    import subprocess
    exe = os.path.join(os.path.dirname(rte.rte.LIB_PATH), "..", "bin", "rte_gpu")
    r = subprocess.run([exe], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 1 and "file.ini" in r.stdout
    r = subprocess.run([exe, "/nonexistent.par"], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 1 and "cannot read parameter file" in r.stdout
