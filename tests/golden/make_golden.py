"""Generate the golden fixtures of tests/golden/ by running the reference's own code.

The reference ships no tests or golden outputs.  This script builds (oracle/build.sh) and runs:
  * oracle/_ref/fim_host -- the FisherInfo_IO sources compiled as host C++, its GPU kernels
    (kernels.cu:151-418) executed once per emulated CUDA thread, its own Neumann()/StopIteration,
    source, diag-term and image code;
  * oracle/_ref/rte_cpu  -- the CPU package built from its own sources;
on small inputs (.par files written below; tissue maps generated with a fixed seed, plus the two
20^3 maps shipped in `GPU package/utility/`), and stores the outputs as .npz files.  It needs the
reference tree: $RTE_REFERENCE_DIR, else a `reference` directory beside the repository; the
fixtures it writes are committed so the tests run without it.

    python tests/golden/make_golden.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("RTE_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))

FIM_PAR = """[Runtime]
TransFile = trans.out
ReflectFile = ref.out
PhaseFile = phase.out
[Algorithm]
nL = {nL}
nTerms = 5
[Geometry]
nX = {nx}
nY = {ny}
nZ = {nz}
xMin = {xmin}
xMax = {xmax}
yMin = {ymin}
yMax = {ymax}
zMin = 0
zMax = {zmax}
propThresh = {prop}
selfsubVox = 1
[Phantom]
NoTiss = {ntiss}
TissMapFile = {tiss}
{tissue_lines}
g = {g}
n = {n}
[Source]
posX = 0
posY = 0
magnitude = {mag}
"""

CPU_PAR = """[Runtime]
TransFile = trans.out
ReflectFile = ref.out
PhaseFile = phase.out
[Algorithm]
nL = {nL}
nTerms = 30
[Geometry]
nX = {n}
nY = {n}
nZ = {n}
xMin = {lo}
xMax = {hi}
yMin = {lo}
yMax = {hi}
zMin = 0
zMax = {zmax}
propThresh = 10
[Phantom]
mua = {mua}
mus = {mus}
g = {g}
n = 1.0
c = 1.0
[Source]
posX = 0
posY = 0
diam = {diam}
magnitude = {mag}
modulation = {modulation}
"""


def run(cmd, cwd):
    # errors="replace": compute_grad_rte.cu:155 prints a FILE* with %s
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, errors="replace")
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed:\n{r.stdout[-2000:]}")
    return r.stdout


def fim_case(name, nx, ny, nz, nL, tiss, mua_t, mus_t, g=0.8, n=1.0, prop=10.0, mag=1.0, apply_seed=None):
    d = tempfile.mkdtemp(prefix="golden_")
    tiss.astype(np.uint8).tofile(os.path.join(d, "tiss.bin"))
    lines = "\n".join(f"TissAbs{t} = {mua_t[t]!r}\nTissSc{t} = {mus_t[t]!r}" for t in range(1, len(mua_t)))
    par = FIM_PAR.format(nL=nL, nx=nx, ny=ny, nz=nz, xmin=-nx * 0.05, xmax=nx * 0.05, ymin=-ny * 0.05,
                         ymax=ny * 0.05, zmax=nz * 0.1, prop=prop, ntiss=len(mua_t) - 1, tiss="tiss.bin",
                         tissue_lines=lines, g=g, n=n, mag=mag)
    open(os.path.join(d, "t.par"), "w").write(par)
    exe = os.path.join(ROOT, "oracle", "_ref", "fim_host")
    N, C = nx * ny * nz, (nL + 1) ** 2
    out = dict(nx=nx, ny=ny, nz=nz, nL=nL, g=g, n=n, prop=prop, mag=mag, tiss=tiss.astype(np.uint8),
               mua_t=np.array(mua_t), mus_t=np.array(mus_t), par=par)
    run([exe, "forward", "t.par", "res"], d)
    rd = lambda f, k: np.fromfile(os.path.join(d, f), np.complex128).reshape(k)
    out["src"] = rd("res_src.bin", (N, C))
    out["out"] = rd("res_out.bin", (N, C))
    out["trans"] = rd("res_trans.bin", (ny, nx))
    out["ref"] = rd("res_ref.bin", (ny, nx))
    meta = dict(l.split() for l in open(os.path.join(d, "res_meta.txt")))
    out["terms"] = int(meta["terms"])
    out["cm"] = float(meta["cm"])
    out["delX"] = float(meta["delX"])
    run([exe, "diag", "t.par", "diag.bin"], d)
    out["diag"] = np.fromfile(os.path.join(d, "diag.bin"), np.complex128).reshape(25, 25, 4)[:C, :C, :]
    if apply_seed is not None:
        rng = np.random.default_rng(apply_seed)
        W = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
        W.tofile(os.path.join(d, "in.bin"))
        for flag, fs in ((1, 1), (1, 0), (0, 1)):
            run([exe, "apply", "t.par", "in.bin", str(flag), str(fs), f"o{flag}{fs}.bin"], d)
            out[f"apply_{flag}{fs}"] = rd(f"o{flag}{fs}.bin", (N, C))
        out["apply_seed"] = apply_seed
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name, "terms", out["terms"])


def fim_downsample_case(name, nx, ny, factors, seed):
    """downsample_image (dist.cu:271-289) of a seeded complex nX x nY image, run by the reference's own
    function inside fim_host (the geometry comes from a .par file, as there; the solver is not run).
    tcache off, so that every block the function allocates gets the allocator's zero fill."""
    d = tempfile.mkdtemp(prefix="golden_")
    nz = 2
    np.ones(nx * ny * nz, np.uint8).tofile(os.path.join(d, "tiss.bin"))
    par = FIM_PAR.format(nL=0, nx=nx, ny=ny, nz=nz, xmin=-nx * 0.05, xmax=nx * 0.05, ymin=-ny * 0.05,
                         ymax=ny * 0.05, zmax=nz * 0.1, prop=1.0, ntiss=1, tiss="tiss.bin",
                         tissue_lines="TissAbs1 = 0.01\nTissSc1 = 1.0", g=0.8, n=1.0, mag=1.0)
    open(os.path.join(d, "t.par"), "w").write(par)
    rng = np.random.default_rng(seed)
    img = rng.standard_normal(nx * ny) + 1j * rng.standard_normal(nx * ny)
    img.tofile(os.path.join(d, "img.bin"))
    exe = os.path.join(ROOT, "oracle", "_ref", "fim_host")
    env = dict(os.environ, GLIBC_TUNABLES="glibc.malloc.tcache_count=0")
    out = dict(nx=nx, ny=ny, img=img, factors=np.array(factors), seed=seed)
    for ds in factors:
        r = subprocess.run([exe, "downsample", "t.par", "img.bin", str(ds), f"ds{ds}.bin"], cwd=d, env=env,
                           stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"fim_host downsample {ds} failed:\n{r.stdout[-2000:]}")
        out[f"ds{ds}"] = np.fromfile(os.path.join(d, f"ds{ds}.bin"), np.complex128)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name)


def fim_program_case(name, base, exe_name, files=(), measured_scale=0.0, runtime_keys=""):
    """Run one of the reference's FisherInfo_IO mains (rte_fim.cu in fim_fisher, rte_snr.cu in
    fim_snr, compute_grad_rte.cu in fim_grad), compiled for the host, on the .par file and tissue map
    of the fixture `base`.  The measured image (gFile) these mains read is the base fixture's
    transmission image times measured_scale (0: zeros).  Stores the program's standard output and
    the binary files it writes."""
    g = np.load(os.path.join(HERE, base + ".npz"))
    d = tempfile.mkdtemp(prefix="golden_")
    nx, ny = int(g["nx"]), int(g["ny"])
    g["tiss"].astype(np.uint8).tofile(os.path.join(d, "tiss.bin"))
    meas = (g["trans"].real.reshape(ny, nx) * measured_scale).astype(np.float64)
    with open(os.path.join(d, "g.out"), "wb") as f:
        f.write(np.array([ny, nx], np.int32).tobytes() + meas.tobytes())
    par = str(g["par"]).replace("[Runtime]", "[Runtime]\ngFile = g.out\n" + runtime_keys, 1)
    open(os.path.join(d, "t.par"), "w").write(par)
    stdout = run([os.path.join(ROOT, "oracle", "_ref", exe_name), "program", "t.par"], d)
    out = dict(base=base, par=par, stdout=stdout, measured_scale=measured_scale)
    for f in files:
        out[f.replace(".", "_")] = np.fromfile(os.path.join(d, f), np.float64)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name)


def fim_forward_main_files(name, bases):
    """The reference's forward main (rte.cu, run in fim_host) on each base fixture's .par file: the raw
    bytes of the TransFile and ReflectFile it writes (dist.cu:316-345 layout)."""
    out = {}
    for base in bases:
        g = np.load(os.path.join(HERE, base + ".npz"))
        d = tempfile.mkdtemp(prefix="golden_")
        g["tiss"].astype(np.uint8).tofile(os.path.join(d, "tiss.bin"))
        open(os.path.join(d, "t.par"), "w").write(str(g["par"]))
        run([os.path.join(ROOT, "oracle", "_ref", "fim_host"), "program", "t.par"], d)
        for f, k in (("trans.out", "trans"), ("ref.out", "ref")):
            out[f"{base}__{k}"] = np.frombuffer(open(os.path.join(d, f), "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print("wrote", name)


def fim_snr_first_depth(name, base):
    """The reference's SNR main (rte_snr.cu) never leaves its first depth: its loop step
    `loc_indz = loc_indz++` (rte_snr.cu:219) leaves the index unchanged as gcc, the host compiler,
    evaluates it, so the program prints the SNR^2 of depth 2 again and again and never writes
    snr_terms.dat.  Run it with line-buffered output until the first value is printed, then stop it,
    and store that line."""
    g = np.load(os.path.join(HERE, base + ".npz"))
    d = tempfile.mkdtemp(prefix="golden_")
    nx, ny = int(g["nx"]), int(g["ny"])
    g["tiss"].astype(np.uint8).tofile(os.path.join(d, "tiss.bin"))
    with open(os.path.join(d, "g.out"), "wb") as f:
        f.write(np.array([ny, nx], np.int32).tobytes() + np.zeros(nx * ny).tobytes())
    par = str(g["par"]).replace("[Runtime]", "[Runtime]\ngFile = g.out", 1)
    open(os.path.join(d, "t.par"), "w").write(par)
    exe = os.path.join(ROOT, "oracle", "_ref", "fim_snr")
    proc = subprocess.Popen(["stdbuf", "-oL", exe, "program", "t.par"], cwd=d, stdout=subprocess.PIPE,
                            stderr=subprocess.STDOUT, text=True)
    line = None
    try:
        for ln in proc.stdout:
            if "is snr_sq for" in ln:
                line = ln.strip()
                break
    finally:
        proc.kill()
        proc.wait()
    if line is None:
        raise RuntimeError("fim_snr printed no SNR value")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), base=base, par=par, first_line=line)
    print("wrote", name, line)


def read_img(path):
    b = open(path, "rb").read()
    nx, ny = np.frombuffer(b[:8], np.int32)
    v = np.frombuffer(b[8:], np.float64)
    return (v[: nx * ny] + 1j * v[nx * ny: 2 * nx * ny]).reshape(ny, nx)


def read_phase(path):
    """The CPU package's phase image (OutputPhaseImage, Dist.c:47-65): nX, nY, then nX*nY doubles."""
    b = open(path, "rb").read()
    nx, ny = np.frombuffer(b[:8], np.int32)
    return np.frombuffer(b[8:], np.float64)[: nx * ny].reshape(ny, nx)


def cpu_case(name, n, nL, mua, mus, g, diam, modulation=0.0, mag=1.0):
    d = tempfile.mkdtemp(prefix="golden_")
    par = CPU_PAR.format(nL=nL, n=n, lo=-n * 0.05, hi=n * 0.05, zmax=n * 0.1, mua=mua, mus=mus, g=g, diam=diam,
                         mag=mag, modulation=modulation)
    open(os.path.join(d, "c.par"), "w").write(par)
    log = run([os.path.join(ROOT, "oracle", "_ref", "rte_cpu"), "c.par"], d)
    # "Neumann series: n" after the steady-state loop (n = terms + 1), after the modulated loop and
    # once more at the end (RTE_uniform.c:111, 159, 186)
    counts = [int(l.split()[-1]) for l in log.splitlines() if l.startswith("Neumann series:")]
    terms = counts[0] - 1
    terms_mod = counts[1] - 1 if modulation != 0.0 else 0
    photons = float([l for l in log.splitlines() if l.startswith("Number of photons total")][-1].split()[-1])
    # the four side-face images, same file layout as the z-face images (Dist.c:353-532)
    side = {f"side{q}": read_img(os.path.join(d, f"SideFace{q}({ax}).out"))
            for q, ax in ((1, "-X"), (2, "+X"), (3, "-Y"), (4, "+Y"))}
    np.savez_compressed(os.path.join(HERE, name + ".npz"), n=n, nL=nL, mua=mua, mus=mus, g=g, diam=diam,
                        mag=mag, modulation=modulation,
                        trans=read_img(os.path.join(d, "trans.out")), ref=read_img(os.path.join(d, "ref.out")),
                        phase=read_phase(os.path.join(d, "phase.out")), terms=terms, terms_mod=terms_mod,
                        photons=photons, par=par, **side)
    print("wrote", name, "terms", terms)


def main():
    if not os.path.isdir(REF):
        sys.exit(f"reference tree {REF} not found")
    subprocess.run(["bash", os.path.join(ROOT, "oracle", "build.sh")], check=True)
    if "--cpu-only" not in sys.argv:
        fim_cases()
    # 4. the CPU package on the 11^3, L=3 configuration (uniform, g = 0.8)
    cpu_case("cpu_uniform_11_L3", 11, 3, 0.01, 1.0, 0.8, 0.1)
    # 5. the CPU package, isotropic scattering (g = 0: only l = 0 propagated), 9^3, L=2
    cpu_case("cpu_isotropic_9_L2", 9, 2, 0.05, 2.0, 0.0, 0.1)
    # 5b. the benchmark's order L = 5 on a 9^3 uniform medium
    cpu_case("cpu_uniform_9_L5", 9, 5, 0.01, 1.0, 0.8, 0.1)
    # 6. intensity modulation (mu_a + i modulation/(c/n), RTE_uniform.c:120-176), 9^3, L=2
    cpu_case("cpu_modulated_9_L2", 9, 2, 0.02, 1.5, 0.8, 0.1, modulation=0.5)
    # 7. a beam over nine columns (the magnitude normalised per column, twice when modulated), L=3
    cpu_case("cpu_modulated_wide_9_L3", 9, 3, 0.03, 1.2, 0.5, 0.35, modulation=1.0, mag=2.0)


def fim_cases():
    rng = np.random.default_rng(2024)
    # 1. uniform medium, 10x10x20, L=2, the reference stop rule (FIM forward)
    fim_case("fim_uniform_10x10x20_L2", 10, 10, 20, 2, np.ones(2000, np.uint8), [0.0, 0.01], [0.0, 1.0],
             apply_seed=1)
    # 2. three tissues at random plus 5% air voxels (never on the source column: mu_s/mu_t of air is
    #    0/0 in the source term), L=2, g = 0.9, n = 1.4 (cm = float(1/n)), magnitude 2
    tiss = rng.integers(1, 4, 2000).astype(np.uint8)
    air = rng.random(2000) < 0.05
    col = (np.arange(2000) % 10 == 5) & ((np.arange(2000) // 10) % 10 == 5)
    tiss[air & ~col] = 0
    fim_case("fim_tissues_10x10x20_L2", 10, 10, 20, 2, tiss, [0.0, 0.01, 0.05, 0.02], [0.0, 1.0, 1.5, 0.7],
             g=0.9, n=1.4, prop=1.5, mag=2.0, apply_seed=2)
    # 3. the shipped non-uniform 20^3 tissue map, L=1
    shipped = np.fromfile(os.path.join(REF, "GPU package", "utility", "tiss_map_nonuni.bin"), np.uint8)
    fim_case("fim_shipped_nonuni_20_L1", 20, 20, 20, 1, shipped, [0.0, 0.01, 0.02, 0.03], [0.0, 1.0, 1.2, 0.8])
    # 4. two tissues at L = 4, the highest order the reference's diag_terms indexing allows (MAX_NL 5)
    tiss4 = np.random.default_rng(77).integers(1, 3, 2000).astype(np.uint8)
    fim_case("fim_tissues_10x10x20_L4", 10, 10, 20, 4, tiss4, [0.0, 0.02, 0.08], [0.0, 1.0, 2.0], g=0.8, prop=10.0,
             apply_seed=4)
    # 5. the forward main itself (rte.cu): the image files it writes for the first three cases
    fim_forward_main_files("fim_forward_main_files", ["fim_uniform_10x10x20_L2", "fim_tissues_10x10x20_L2",
                                                      "fim_shipped_nonuni_20_L1"])
    # 5b. the Fisher, SNR and region-gradient mains on the random-tissue case
    fim_program_case("fim_fisher_main_10x10x20_L2", "fim_tissues_10x10x20_L2", "fim_fisher")
    fim_snr_first_depth("fim_snr_main_10x10x20_L2", "fim_tissues_10x10x20_L2")
    fim_program_case("fim_grad_main_10x10x20_L2", "fim_tissues_10x10x20_L2", "fim_grad", files=("Residual.out",),
                     measured_scale=1.05, runtime_keys="numIterations = 1\n")
    # 6. downsample_image on a square and on a non-square image (its rows are nY long), ragged factors
    fim_downsample_case("fim_downsample_20x20", 20, 20, [1, 2, 3, 4, 5, 7], 31)
    fim_downsample_case("fim_downsample_24x18", 24, 18, [2, 3, 4, 5], 32)


if __name__ == "__main__":
    main()
