"""Build the sm_100a shared library doi_b200/lib/librte_b200.so with nvcc (in-tree).

Usage: python -m doi_b200.build [-v]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "librte_b200.so")
BINDIR = os.path.join(HERE, "bin")
SOURCES = ["rte_kernels.cu", "rte_noalloc.cu", "rte_host.cpp", "rte_server.cpp", "rte_par.cpp", "rte_faces.cpp",
           "rte_fft.cpp"]
CLI = "rte_cli.cpp"  # built into bin/ by build_cli, not into the library
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    if not os.path.exists(os.path.join(BINDIR, "rte_gpu")):
        return True
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "rte_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose=False, force=False, ptxas_verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objs = []
    for src in SOURCES:
        obj = os.path.join(LIBDIR, src + ".o")
        cmd = [nvcc()] + ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
               "-I", os.path.join(HERE, "..", "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cu"):
            cmd[1:1] = ["--expt-relaxed-constexpr"]
            if ptxas_verbose:
                cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc(), "-shared"] + ARCH + ["-o", LIB] + objs + ["-lcufft", "-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    build_cli(verbose)
    return LIB


def build_cli(verbose=False):
    """The reference's program names (rte_gpu, rte_inv, rte_test, rte_fim, rte_snr) as one executable over the
    library, in doi_b200/bin (run-time path to ../lib)."""
    os.makedirs(BINDIR, exist_ok=True)
    exe = os.path.join(BINDIR, "rte_gpu")
    cmd = [nvcc()] + ARCH + ["-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), os.path.join(CSRC, CLI),
           "-o", exe, "-L", LIBDIR, "-lrte_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../lib"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    for name in ("rte_inv", "rte_test", "rte_fim", "rte_snr"):
        link = os.path.join(BINDIR, name)
        if os.path.lexists(link):
            os.remove(link)
        os.symlink("rte_gpu", link)


if __name__ == "__main__":
    v = "-v" in sys.argv
    print(build(verbose=v, force=True, ptxas_verbose="--ptxas" in sys.argv))
