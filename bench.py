#!/usr/bin/env python
"""Forward-solve throughput of the B200 Neumann-series RTE solver.

Workload (one step = one forward solve): 33x33x33 voxels of 0.1 cm, SH order L=5 (36 coefficients),
uniform background mu_a=0.01, mu_s=1 cm^-1, g=0.8, n=1, plus 3 seeded spherical inclusions
(radius U[0.2,0.6] cm, mu_a x U[2,10], mu_s x U[0.5,2]); collimated pencil at the centre of the z=0
face; 20 Neumann terms plus the final attenuation pass; exitance images of both z faces.  Every
step solves a different seeded phantom, so the voxel-pair kernel is recomputed inside every step.

`value`  : solves/s with the media already resident in HBM (rte_set_medium_device + rte_forward).
`e2e`    : the same through the C ABI with pinned HOST buffers: medium H2D, full distribution + images D2H.
Multi-GPU: replicas only (one process per GPU, independent solves, max-over-ranks device time).
--impl reference: the FP64 CPU port of the reference path (oracle/, OpenMP on all host cores) on a
bounded sample of the same workload, extrapolated to solves/s.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd solves/s @33³ L=5 (mixed+batched vs FP64, ≤1e-5 rel); serve p50/p99 ms"
N_SIDE, L, TERMS, DX = 33, 5, 20, 0.1


def phantom(seed):
    from doi_b200.phantoms import sphere_phantom
    mua, mus, _ = sphere_phantom(N_SIDE, dx=DX, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=seed)
    return mua, mus


def algorithmic_counts(n=N_SIDE, Lo=L):
    """Coupled ordered pairs and the summed Siddon step count sum(|dx|+|dy|+|dz|) over them (all pairs
    couple at propThresh > diagonal)."""
    N = n ** 3
    C = (Lo + 1) ** 2
    pairs = N * (N - 1)
    # sum over ordered pairs of |di| for one axis = n^2 * n^2 * sum_{a,b} |a-b| = n^4 * (n^3 - n)/3
    s1 = (n ** 4) * (n ** 3 - n) / 3.0
    steps = 3 * s1
    # FLOP per launch of the one-source pair-apply kernel: 7C (SH recurrence 3C + two C-length MACs
    # 4C) + 10 (direction) per coupled pair; the precompute: 2 per Siddon step + 25 (geometry, exp).
    apply_flop = pairs * (7 * C + 10)
    store_flop = 2 * steps + 25 * pairs
    # canonical per-solve count (flops_term = pairs(7C + 2S + 25) + N(2C^2 + 4C), (terms+1) terms)
    term = pairs * (7 * C + 25) + 2 * steps + N * (2 * C * C + 4 * C)
    return dict(N=N, C=C, pairs=pairs, steps=steps, apply_flop=apply_flop, store_flop=store_flop,
                solve_flop=(TERMS + 1) * term)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-i", str(index), "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip() == "Active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(value, device=None):
    """Max of a per-rank scalar over the process group (device time of a multi-GPU run)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def throughput(world, steps, ms_max):
    """Whole-job solves/s: every rank solves `steps` phantoms; the job takes the slowest rank's time."""
    return world * steps / (ms_max / 1e3)


def cpu_baseline(seconds=10.0, seed=0):
    """The FP64 oracle (CPU port of the reference path) on a bounded sample: the operator for a set of
    destination voxels against all sources, extrapolated to a full solve (21 applications)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build.sh")], check=True,
                       env=dict(os.environ, RTE_REFERENCE_DIR="/nonexistent"))
    mua, mus = phantom(seed)
    N = N_SIDE ** 3
    p = O.params(N_SIDE, N_SIDE, N_SIDE, DX, DX, DX, L, 0.8, 1.0, 100.0, mode=O.MODE_EXACT)
    rng = np.random.default_rng(0)
    W = O.source(p, mua, mus, kind=O.SRC_COLUMN)
    W = W + 1e-3 * rng.standard_normal(W.shape)  # dense input so every pair does full work
    O.apply_subset(p, mua, mus, W, rng.choice(N, 4, replace=False))  # builds the self-term tables
    nd = 16
    t = time.perf_counter()
    O.apply_subset(p, mua, mus, W, rng.choice(N, nd, replace=False))
    dt = time.perf_counter() - t
    nd2 = max(nd, int(nd * seconds / max(dt, 1e-3)))
    t = time.perf_counter()
    O.apply_subset(p, mua, mus, W, rng.choice(N, nd2, replace=False))
    dt = time.perf_counter() - t
    per_app = dt * N / nd2
    solve_s = per_app * (TERMS + 1)
    cores = os.cpu_count()
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"operator D*A for {nd2} random destination voxels ({100.0 * nd2 / N:.1f} % of the {N}) x all "
                      f"sources of the 33^3 L=5 phantom ({dt:.1f} s), extrapolated x{N / nd2:.0f} voxels x{TERMS + 1} "
                      "applications",
            "what": "the unoptimised FP64 oracle port (a restatement of the reference algorithm in the complex "
                    "SH basis, OpenMP over destination voxels): a reported baseline, not a target; the reference "
                    "has no CPU code for non-uniform media (the CPU package's own run is config1_plain_fp64)",
            "seconds_per_solve": solve_s}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return 0
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(seconds=args.ref_seconds)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(seconds=args.ref_seconds))
    wall = time.perf_counter() - t0
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "33^3 voxels, L=5, 3-sphere phantom, 20 Neumann terms + final A, images",
                       "parallelism": "host OpenMP"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                                        "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


SERVE_GRIDS, SERVE_ORDERS = (17, 25, 33, 41), (3, 5, 7)


def serve_requests(count, seed):
    """The seeded request mix of the serving stream: grid from {17,25,33,41}^3 (0.1 cm), SH order from
    {3,5,7}, background mu_a=0.01 / mu_s=1 plus 0-3 inclusions as in the phantom above, one source:
    collimated beam or isotropic point on a random face at a uniform-random position."""
    from doi_b200.phantoms import sphere_phantom
    import doi_b200 as R
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        n = int(rng.choice(SERVE_GRIDS))
        Lq = int(rng.choice(SERVE_ORDERS))
        mua, mus, _ = sphere_phantom(n, dx=DX, mua_bg=0.01, mus_bg=1.0, nspheres=int(rng.integers(0, 4)),
                                     seed=seed * 100003 + q)
        face = int(rng.integers(0, 6))
        kind = R.SRC_BEAM if rng.random() < 0.5 else R.SRC_POINT
        a, b = rng.uniform(-n * DX / 2, n * DX / 2, 2)
        src = R.Source(pos_x=float(a), pos_y=float(b), pos_z=float(b + n * DX / 2), kind=kind, face=face)
        out.append((n, Lq, mua, mus, src))
    return out


def serve_stream(srv, reqs, gaps):
    """Submit reqs (n, L, mua, mus, src) at the given inter-arrival gaps, wait for all; returns (wall s,
    latencies ms, summed device ms)."""
    t0 = time.perf_counter()
    tickets, t_next = [], t0
    for (n, Lq, mua, mus, src), gap in zip(reqs, gaps):
        t_next += gap
        d = t_next - time.perf_counter()
        if d > 0:
            time.sleep(d)
        tickets.append(srv.submit(mua, mus, [src], n, dx=DX, nL=Lq, g=0.8, terms=TERMS))
    lat, dev_ms = [], 0.0
    for t in tickets:
        _, _, info = srv.wait(t, timeout=3600)
        lat.append(info["latency_ms"])
        dev_ms += info["device_ms"]
    return time.perf_counter() - t0, np.array(lat), dev_ms


def serve_measure(srv, reqs, rate, seed):
    """Saturated capacity (every request submitted at once: completed / wall), then the same requests
    with seeded Poisson arrivals at `rate` (0: 0.7 x the capacity) for p50 / p99 latency."""
    wall_sat, _, _ = serve_stream(srv, reqs, np.zeros(len(reqs)))
    capacity = len(reqs) / wall_sat
    rate = rate if rate > 0 else 0.7 * capacity
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, len(reqs))
    wall, lat, dev_ms = serve_stream(srv, reqs, gaps)
    return {"requests": len(reqs), "capacity_solves_per_s": capacity, "saturated_wall_s": wall_sat,
            "arrival_rate_per_s": rate, "solves_per_s": len(reqs) / wall, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()), "wall_s": wall,
            "device_ms_sum": dev_ms}


def run_serve(args, dev):
    """Continuous-batching streams through rte_server_*.  (1) BASELINE config 3's request mix (grids
    {17,25,33,41}^3, orders {3,5,7}, 0-3 inclusions, beam or isotropic point on a random face); (2) the
    benchmark's own shape: single-source 33^3 L=5 requests, each on a new 3-sphere phantom with a
    collimated beam at a random z=0 position, the form the >= 5x target is stated for.  Each stream:
    saturated capacity, then Poisson arrivals at 0.7 x capacity for p50 / p99 latency."""
    import doi_b200 as R
    from doi_b200.phantoms import sphere_phantom
    mix = serve_requests(args.serve_requests, seed=17)
    rng = np.random.default_rng(29)
    bench_shape = []
    for q in range(args.serve_requests_33):
        mua, mus, _ = sphere_phantom(N_SIDE, dx=DX, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=50000 + q)
        a, b = rng.uniform(-N_SIDE * DX / 2, N_SIDE * DX / 2, 2)
        bench_shape.append((N_SIDE, L, mua, mus, R.Source(pos_x=float(a), pos_y=float(b), kind=R.SRC_COLUMN)))
    out = {}
    with R.Server(device=dev, workers=args.serve_workers) as srv:
        # one request of every shape first (context creation, self-term tables, graph capture) so the
        # streams measure steady-state serving; these are not counted
        N0 = [(n, Lq) for n in SERVE_GRIDS for Lq in SERVE_ORDERS]
        warm = [srv.submit(np.full(n ** 3, 0.01), np.full(n ** 3, 1.0), [R.Source(kind=R.SRC_BEAM)], n, dx=DX,
                           nL=Lq, g=0.8, terms=TERMS) for n, Lq in N0]
        for t in warm:
            srv.wait(t, timeout=1800)
        st0 = srv.stats()
        if mix:
            out = serve_measure(srv, mix, args.serve_rate, 23)
            out["mix"] = ("grid {17,25,33,41}^3, L {3,5,7}, 0-3 inclusions, beam or isotropic point on a random "
                          "face; warm-up: one uncounted request of every (grid, order) shape")
            out["subset"] = (f"{len(mix)} of the 2,000 requests of the full stream (the full stream takes ~20 min "
                             "of device time, beyond the bench's time budget; run it with --serve-requests 2000)")
        if bench_shape:
            b = serve_measure(srv, bench_shape, 0.0, 31)
            b["workload"] = (f"{len(bench_shape)} single-source {N_SIDE}^3 L={L} requests, each a new 3-sphere phantom, "
                             "collimated z=0 beam at a random position, 20 terms, mixed precision")
            out["bench_shape"] = b
        st = srv.stats()
    out.update({"workers": args.serve_workers, "terms": TERMS,
                "precision": "mixed (stored FP32 pair kernel; FFT convolution for uniform media)",
                "contexts": st["contexts"], "hbm_reserved_gb": st["hbm_reserved"] / 1e9,
                "failed": st["failed"] - st0["failed"]})
    return out


CFG1_PAR = """[Runtime]
TransFile = trans.out
ReflectFile = ref.out
PhaseFile = phase.out
[Algorithm]
nL = 3
nTerms = 30
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
c = 1.0
[Source]
posX = 0
posY = 0
diam = 0.1
magnitude = 1.0
"""


def run_cfg1(dev):
    """The plain FP64 method on the uniform 11^3, L=3 case: GPU solve with the relative-L2 rule (1e-7 or
    30 terms) plus the 6-face flux, and the CPU package itself (oracle/_ref/rte_cpu, built from the
    reference sources) on the same input with its own stop rule, timed on the host cores; the GPU run
    with the package's stop rule is compared with the package's images."""
    import doi_b200 as R
    n, L = 11, 3
    N = n ** 3
    ctx = R.Context(n, n, n, dx=0.1, nL=L, g=0.8, n=1.0, c=1.0, prop_thresh=10.0, model=R.MODEL_CPU,
                    precision=R.PREC_FP64, device=dev)
    ctx.set_medium_voxel(np.full(N, 0.01), np.full(N, 1.0))
    src = R.Source(diam=0.1, kind=R.SRC_CPU)
    out = {"workload": "11^3 uniform (mu_a 0.01, mu_s 1, g 0.8), L=3, centre pencil, CPU-package model, FP64"}
    ctx.forward(src, R.Stop(R.STOP_REL_L2, 30, 1e-7))  # warm-up
    t = time.perf_counter()
    r = ctx.forward(src, R.Stop(R.STOP_REL_L2, 30, 1e-7))
    flux = ctx.detector_flux([src], R.Stop(R.STOP_REL_L2, 30, 1e-7), R.Detector(nbins=n, faces=63))
    out["gpu_wall_ms"] = (time.perf_counter() - t) * 1e3
    out["gpu_solve_ms_device"] = r["ms_device"]
    out["gpu_terms_rel_l2_1e-7"] = r["terms"]
    out["six_face_flux_total"] = float(flux.sum())
    ref_rule = ctx.forward(src, R.Stop(R.STOP_REFERENCE))
    ctx.close()
    exe = os.path.join(ROOT, "oracle", "_ref", "rte_cpu")
    if not os.path.exists(exe):
        out["cpu_package"] = None
        return out
    d = tempfile.mkdtemp(prefix="cfg1_")
    open(os.path.join(d, "c.par"), "w").write(CFG1_PAR)
    t = time.perf_counter()
    pr = subprocess.run([exe, "c.par"], cwd=d, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    wall = time.perf_counter() - t
    if pr.returncode != 0:
        out["cpu_package"] = {"error": pr.stdout[-300:]}
        return out

    def img(path):
        b = open(path, "rb").read()
        nx, ny = np.frombuffer(b[:8], np.int32)
        v = np.frombuffer(b[8:], np.float64)
        return (v[: nx * ny] + 1j * v[nx * ny: 2 * nx * ny]).reshape(ny, nx)

    terms = [ln for ln in pr.stdout.splitlines() if ln.startswith("Neumann series:")]
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    out["cpu_package"] = {"wall_s": wall, "cores": os.cpu_count(), "threads": "OpenMP, all host cores",
                          "terms_own_rule": int(terms[-1].split()[-1]) - 1 if terms else None,
                          "gpu_terms_same_rule": ref_rule["terms"],
                          "rel_l2_trans": rel(ref_rule["trans"], img(os.path.join(d, "trans.out"))),
                          "rel_l2_ref": rel(ref_rule["ref"], img(os.path.join(d, "ref.out")))}
    return out


def grad_problem(dev, n=N_SIDE, prec=None, kernel_mode=None, terms=TERMS):
    """Config 4: the n^3 L=5 phantom (3 spheres, seed 4), 4 collimated z=0 sources at (+-0.825, +-0.825) cm
    scaled to the grid, 8x8 bins on each of the 6 faces, target flux from the phantom with every sphere's
    coefficients scaled by (1 + 0.05 N(0,1))."""
    import doi_b200 as R
    from doi_b200.phantoms import sphere_phantom
    mua, mus, sph = sphere_phantom(n, dx=DX, mua_bg=0.01, mus_bg=1.0, nspheres=3, seed=4)
    rng = np.random.default_rng(44)
    pa, ps = mua.copy(), mus.copy()
    for sp in sph:  # perturb each inclusion's values
        ka, ks = 1 + 0.05 * rng.standard_normal(2)
        pa[mua == sp["mua"]] *= ka
        ps[mus == sp["mus"]] *= ks
    prec = R.PREC_MIXED if prec is None else prec
    ctx = R.Context(n, n, n, dx=DX, nL=L, g=0.8, precision=prec, device=dev,
                    kernel_mode=R.KERNEL_STORE if kernel_mode is None else kernel_mode)
    off = 0.825 * n / 33.0
    srcs = [R.Source(pos_x=x, pos_y=y, kind=R.SRC_COLUMN) for x, y in ((-off, -off), (off, -off), (-off, off), (off, off))]
    stop = R.Stop(R.STOP_FIXED, terms)
    det = R.Detector(nbins=8, faces=63)
    ctx.set_medium_voxel(pa, ps)
    target = ctx.detector_flux(srcs, stop, det)
    ctx.set_medium_voxel(mua, mus)
    return ctx, srcs, stop, det, target


def run_grad(dev):
    """Adjoint gradient at config 4 (33^3, L=5): cost of the mixed-precision rte_gradient against the
    forward solves it differentiates, and its error against the FP64 method's gradient (stored FP64 pair
    kernel) of the same 20-term model."""
    import doi_b200 as R
    ctx, srcs, stop, det, target = grad_problem(dev)
    ctx.detector_flux(srcs[:1], stop, det)
    ctx.gradient(srcs[:1], stop, det, target[:1])  # warm-up (autotuner, buffers)
    t = time.perf_counter()
    ctx.detector_flux(srcs, stop, det)
    t_fwd = time.perf_counter() - t
    t = time.perf_counter()
    loss, ga, gs = ctx.gradient(srcs, stop, det, target)
    t_grad = time.perf_counter() - t
    ctx.close()
    c64, srcs, stop, det, target = grad_problem(dev, prec=R.PREC_FP64, kernel_mode=R.KERNEL_STORE)
    t = time.perf_counter()
    loss64, ga64, gs64 = c64.gradient(srcs, stop, det, target)
    t64 = time.perf_counter() - t
    c64.close()
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    return {"workload": "33^3 L=5 phantom, 4 z=0 sources, 8x8 bins x 6 faces, 20 terms, mixed precision",
            "forward_s_4src": t_fwd, "gradient_s_4src": t_grad, "ratio_gradient_over_forward": t_grad / t_fwd,
            "loss": loss, "grad_norm_mua": float(np.linalg.norm(ga)), "grad_norm_mus": float(np.linalg.norm(gs)),
            "fp64_rel_err": {"loss": abs(loss - loss64) / loss64, "g_mua": rel(ga, ga64), "g_mus": rel(gs, gs64),
                             "against": "FP64 method (stored FP64 pair kernel) on the same 20-term model"},
            "fp64_gradient_s_4src": t64,
            "check": "central finite differences at this size in FP64 (10 + 10 voxels, 40 terms): "
                     "tests/test_gpu_fullsize.py::test_gradient_finite_differences_at_config4_size"}


def fisher_problem(dev, n, Lq, prec, kernel_mode):
    """Config 5's medium at n^3: background mu_a 0.02, mu_s 2, g 0.9, 8 seeded inclusions rasterised with a
    one-voxel partial-volume ramp (derivatives of x, y, z and mu_a contrast each: 32 parameters), six
    collimated beams at the face centres."""
    import doi_b200 as R
    sph = R.random_spheres(n, 8, seed=55, dx=DX)
    mua, mus, dmua, dmus = R.smooth_sphere_phantom(n, sph, dx=DX, mua_bg=0.02, mus_bg=2.0)
    ctx = R.Context(n, n, n, dx=DX, nL=Lq, g=0.9, precision=prec, kernel_mode=kernel_mode, device=dev)
    ctx.set_medium_voxel(mua, mus)
    h = n * DX / 2
    srcs = [R.Source(kind=R.SRC_BEAM, face=0), R.Source(kind=R.SRC_BEAM, face=1, pos_z=n * DX),
            R.Source(kind=R.SRC_BEAM, face=2, pos_z=h), R.Source(kind=R.SRC_BEAM, face=3, pos_z=h),
            R.Source(kind=R.SRC_BEAM, face=4, pos_z=h), R.Source(kind=R.SRC_BEAM, face=5, pos_z=h)]
    return ctx, srcs, dmua, dmus


def run_fisher_case(dev, n, Lq, nbins, terms, nsrc=6, P=32, kernel_mode=None, prec=None, want_J=False):
    """One rte_fisher call of nsrc sources x P parameters; returns (F, J, seconds, forward seconds of the
    same sources, stats).  The forward seconds are those of the FP64 method with path integrals
    recomputed, which is how rte_fisher runs its forward solves in either precision (the Poisson weights)."""
    import doi_b200 as R
    ctx, srcs, dmua, dmus = fisher_problem(dev, n, Lq, R.PREC_MIXED if prec is None else prec,
                                           R.KERNEL_RECOMPUTE if kernel_mode is None else kernel_mode)
    stop = R.Stop(R.STOP_FIXED, terms)
    det = R.Detector(nbins=nbins, faces=63)
    ctx.stats()
    ctx.set_profiling(True)
    t = time.perf_counter()
    res = ctx.fisher(srcs[:nsrc], stop, det, dmua[:P], dmus[:P], want_J=want_J)
    sec = time.perf_counter() - t
    st = ctx.stats()
    ctx.close()
    c64, srcs, _, _ = fisher_problem(dev, n, Lq, R.PREC_FP64, R.KERNEL_RECOMPUTE)
    c64.detector_flux(srcs[:1], R.Stop(R.STOP_FIXED, 1), det)  # warm-up: buffers, tables
    t = time.perf_counter()
    c64.detector_flux(srcs[:nsrc], stop, det)
    t_fwd = time.perf_counter() - t
    c64.close()
    F, J = res if want_J else (res, None)
    return F, J, sec, t_fwd, st


def run_fisher(dev, full_matrix_at_49=False):
    """Fisher information of 8 seeded inclusions x (x, y, z, mu_a contrast) = 32 parameters (BASELINE config
    5), Poisson noise, path integrals recomputed along every pair in every term (no stored pair kernel):
    (1) the full configuration, 49^3, L=7, 16x16 bins, on a bounded leg of 1 source x 4 parameters (one
    four-right-hand-side tangent series), extrapolated to 6 sources x 32 parameters; (2) the whole 32 x 32
    matrix at 25^3, L=5; (3) its FP64 error on 6 sources x 4 parameters against the FP64 method."""
    import doi_b200 as R
    out = {"workload": "8 inclusions x 4 = 32 parameters, 6 face-centre beams, 16x16 bins x 6 faces, 20 terms, "
                       "mixed precision, path integrals recomputed (no stored pair kernel)"}
    # (1) the full configuration, bounded
    run_fisher_case(dev, 49, 7, 16, 2, nsrc=1, P=4)  # warm-up: split autotuning, buffers
    if full_matrix_at_49:
        F, _, sec, t_fwd, st = run_fisher_case(dev, 49, 7, 16, TERMS)
        out["full_49_L7"] = {"seconds": sec, "measured": "6 sources x 32 parameters", "pair_kernel_ms": st["ms_pair"]}
    else:
        F, _, sec, t_fwd, st = run_fisher_case(dev, 49, 7, 16, TERMS, nsrc=1, P=4)
        t_tan = max(sec - t_fwd, 0.0)
        out["full_49_L7"] = {
            "measured": "1 source x 4 parameters (the FP64 forward solve and one four-right-hand-side tangent series)",
            "seconds": sec, "forward_s_1src": t_fwd, "tangent_s_4params": t_tan,
            "extrapolated_s_6src_32params": 6 * t_fwd + 6 * 8 * t_tan,
            "extrapolation": "6 FP64 forward solves (timed alone: forward_s_1src) + 6 x 8 four-parameter tangent "
                             "series (the rest of the measured call) at the measured rates",
            "pair_kernel_ms": st["ms_pair"], "launches": st["launches"]}
    # (2) the whole matrix at 25^3, L=5
    F, _, sec, t_fwd, st = run_fisher_case(dev, 25, 5, 16, TERMS)
    ev = np.linalg.eigvalsh(F)
    out["matrix_25_L5"] = {"seconds": sec, "tangent_solves": 6 * 32, "forward_solves_6src_fp64_s": t_fwd,
                           "pair_kernel_ms": st["ms_pair"], "launches": st["launches"], "F_trace": float(np.trace(F)),
                           "F_cond": float(ev.max() / max(ev.min(), 1e-300)), "F_min_eig": float(ev.min())}
    # (3) FP64 error of F and J (all 6 sources x 4 parameters at 25^3 L=5)
    Fm, Jm, _, _, _ = run_fisher_case(dev, 25, 5, 16, TERMS, nsrc=6, P=4, want_J=True)
    F64, J64, _, _, _ = run_fisher_case(dev, 25, 5, 16, TERMS, nsrc=6, P=4, want_J=True, prec=R.PREC_FP64,
                                        kernel_mode=R.KERNEL_STORE)
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    out["fp64_rel_err"] = {"F": rel(Fm, F64), "J": rel(Jm, J64), "case": "25^3 L=5, 6 sources x 4 parameters",
                           "note": "F weights each bin by 1/flux; bins of near-zero flux amplify the mixed solve's "
                                   "relative flux error there, so F's error exceeds J's"}
    return out


def run_uniform(dev):
    """A uniform 33^3, L=5 medium (the background of the phantom): forward solves through the FFT
    convolution path (automatic kernel mode) against the stored-kernel pair path, FP64 error of each."""
    import doi_b200 as R
    N = N_SIDE ** 3
    mua, mus = np.full(N, 0.01), np.full(N, 1.0)
    src = R.Source(kind=R.SRC_COLUMN)
    stop = R.Stop(R.STOP_FIXED, TERMS)
    out = {"workload": f"{N_SIDE}^3 uniform (mu_a 0.01, mu_s 1, g 0.8), L={L}, centre beam, {TERMS} terms"}
    res = {}
    for name, prec, km in (("fft", R.PREC_MIXED, R.KERNEL_AUTO), ("pair_stored", R.PREC_MIXED, R.KERNEL_STORE),
                           ("fp64_pairs", R.PREC_FP64, R.KERNEL_RECOMPUTE)):
        ctx = R.Context(N_SIDE, N_SIDE, N_SIDE, dx=DX, nL=L, g=0.8, precision=prec, kernel_mode=km, device=dev)
        ctx.set_medium_voxel(mua, mus)
        ctx.forward(src, stop, want_W=False)  # warm-up: tables, plans, stored kernel
        t = time.perf_counter()
        r = ctx.forward(src, stop, want_W=True)
        res[name] = r
        out[name + "_ms"] = (time.perf_counter() - t) * 1e3
        out[name + "_ms_device"] = r["ms_device"]
        ctx.close()
    rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
    out["fft_rel_err_vs_fp64"] = rel(res["fft"]["W"], res["fp64_pairs"]["W"])
    out["pair_rel_err_vs_fp64"] = rel(res["pair_stored"]["W"], res["fp64_pairs"]["W"])
    out["speedup_fft_over_pairs"] = out["pair_stored_ms_device"] / out["fft_ms_device"]
    return out


def hbm_line(traffic, avg_ms):
    """The pair kernel's DRAM bytes per launch (ncu) over its live launch time, against the measured
    HBM copy bandwidth: how far the kernel is from being memory-bound."""
    if not traffic:
        return None
    peak = None
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        peak = json.load(open(mp)).get("hbm_gbs")
    gbs = traffic / (avg_ms * 1e-3) / 1e9
    return {"achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak if peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peak else None}


def run_ours(args):
    import torch
    import doi_b200 as R
    ws, rank, local = dist_setup()
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)
    prec = R.PREC_MIXED if args.precision == "mixed" else R.PREC_FP64
    kmode = R.KERNEL_STORE if prec == R.PREC_MIXED else R.KERNEL_RECOMPUTE
    ctx = R.Context(N_SIDE, N_SIDE, N_SIDE, dx=DX, nL=L, g=0.8, n=1.0, precision=prec, kernel_mode=kmode,
                    device=dev)
    src = R.Source(pos_x=0.0, pos_y=0.0, kind=R.SRC_COLUMN)
    stop = R.Stop(R.STOP_FIXED, TERMS)
    # batched form: B of the four collimated z=0 sources at (+-0.825, +-0.825) cm of the adjoint
    # configuration, solved together on each phantom (each pair's direction, spherical harmonics and
    # kernel value serve all B sources)
    B = args.batch
    srcs = [R.Source(pos_x=x, pos_y=y, kind=R.SRC_COLUMN) for x, y in
            ((-0.825, -0.825), (0.825, -0.825), (-0.825, 0.825), (0.825, 0.825))][:B] if B > 1 else [src]
    nsteps = args.steps + args.warmup
    seeds = [1000 * rank + s for s in range(nsteps)]
    media = [phantom(s) for s in seeds]
    dmedia = [(torch.tensor(a, dtype=torch.float64, device=f"cuda:{dev}"),
               torch.tensor(b, dtype=torch.float64, device=f"cuda:{dev}")) for a, b in media]
    peak32 = R.rte.measure_fma_peak(False, dev)
    peak64 = R.rte.measure_fma_peak(True, dev)
    streams = {k: R.rte.measure_fma_peak(device=dev, stream=k)
               for k in ("fp32_scalar", "fp32_packed", "fp32_packed_fresh")}
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")
    counts = algorithmic_counts(N_SIDE, L)

    def step(k):
        a, b = dmedia[k]
        ctx.set_medium_device(a.data_ptr(), b.data_ptr())
        if B > 1:
            return ctx.forward_batch(srcs, stop, want_W=False, want_images=True)
        return ctx.forward(src, stop, want_W=False, want_images=True)

    for k in range(args.warmup):
        step(k)
    ctx.stats()  # reset counters
    ctx.set_profiling(True)
    torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    clk = Clocks(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.warmup, nsteps):
        step(k)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    st = ctx.stats()
    ctx.set_profiling(False)
    if ws > 1:
        ms = max_over_ranks(ms, f"cuda:{dev}")
        torch.distributed.barrier()
    value = throughput(ws, args.steps * B, ms)

    # e2e through the C ABI with host buffers (medium H2D, distribution + images D2H), all in pinned
    # host memory allocated before the timed region, as a serving process would hold them
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    h2d = 2 * counts["N"] * 8
    d2h = B * (counts["N"] * counts["C"] * 16 + 2 * N_SIDE * N_SIDE * 16)

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype).pin_memory().numpy()

    pmedia = []
    for a, b in media[args.warmup:]:
        pa, pb = pinned(a.shape, torch.float64), pinned(b.shape, torch.float64)
        pa[...], pb[...] = a, b
        pmedia.append((pa, pb))
    lead = (B,) if B > 1 else ()
    img = (B, N_SIDE, N_SIDE) if B > 1 else (N_SIDE * N_SIDE,)
    pout = {"W": pinned(lead + (counts["N"], counts["C"]), torch.complex128),
            "trans": pinned(img, torch.complex128), "ref": pinned(img, torch.complex128)}
    torch.cuda.synchronize(dev)
    e2.record(stream)
    for pa, pb in pmedia:
        ctx.set_medium_voxel(pa, pb)
        if B > 1:
            ctx.forward_batch(srcs, stop, want_W=True, want_images=True, out=pout)
        else:
            ctx.forward(src, stop, want_W=True, want_images=True, out=pout)
    e3.record(stream)
    e3.synchronize()
    ms_e2e = e2.elapsed_time(e3)
    if ws > 1:
        ms_e2e = max_over_ranks(ms_e2e, f"cuda:{dev}")
    e2e = throughput(ws, args.steps * B, ms_e2e)

    out = None
    if rank == 0:
        # accuracy of this precision against the plain FP64 method (itself held to the oracle by the
        # parity tests) on the first timed phantom, and the plain method's own speed
        ctx.set_medium_voxel(*media[args.warmup])
        r_mixed = ctx.forward_batch(srcs, stop, want_W=True) if B > 1 else ctx.forward(src, stop, want_W=True)
        if B > 1:
            r_mixed = {k: r_mixed[k][0] for k in ("W", "trans", "ref")}
        ref_err, plain, plain_stored = None, None, None
        if prec == R.PREC_MIXED and not args.skip_fp64_check:
            # the plain FP64 method as the reference computes it (every path integral recomputed every
            # term), and the same method with its FP64 pair kernel stored (8 N^2 bytes, precompute included)
            c64 = R.Context(N_SIDE, N_SIDE, N_SIDE, dx=DX, nL=L, g=0.8, precision=R.PREC_FP64, device=dev)
            c64.set_medium_voxel(*media[args.warmup])
            r64 = c64.forward(srcs[0], stop, want_W=True)
            rel = lambda x, y: float(np.linalg.norm(x - y) / np.linalg.norm(y))
            ref_err = {"W": rel(r_mixed["W"], r64["W"]), "trans": rel(r_mixed["trans"], r64["trans"]),
                       "ref": rel(r_mixed["ref"], r64["ref"]), "against": "plain FP64 method on the same phantom "
                       "and source (itself within 1e-11 of the FP64 oracle: tests/test_gpu_fullsize.py)"}
            plain = 1e3 / r64["ms_device"]
            c64.close()
            c64 = R.Context(N_SIDE, N_SIDE, N_SIDE, dx=DX, nL=L, g=0.8, precision=R.PREC_FP64,
                            kernel_mode=R.KERNEL_STORE, device=dev)
            c64.set_medium_voxel(*media[0])
            c64.forward(srcs[0], stop, want_W=False)  # warm-up on another phantom
            c64.set_medium_voxel(*media[args.warmup])
            r64s = c64.forward(srcs[0], stop, want_W=True)
            ref_err["fp64_stored_vs_recomputed_W"] = rel(r64s["W"], r64["W"])
            plain_stored = 1e3 / r64s["ms_device"]
            c64.close()
        avg_pair_ms = st["ms_pair"] / max(st["n_pair"], 1)
        nbk = 1 if B == 1 else (2 if B <= 2 else 4)  # right-hand sides per launch
        # algorithmic FLOP per launch: per coupled pair 3C (SH) + 4C per right-hand side + 10 (direction)
        apply_flop = counts["pairs"] * (3 * counts["C"] + 4 * counts["C"] * B + 10)
        achieved = apply_flop / (avg_pair_ms * 1e-3) / 1e12
        peak = peak32 if prec == R.PREC_MIXED else peak64
        # DRAM bytes of one pair launch from the ncu capture in profiles/ (per pair, scaled to this grid)
        traffic = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp) and prec == R.PREC_MIXED:
            bpp = json.load(open(tp)).get("bytes_per_pair", {}).get(str(nbk))
            traffic = bpp * counts["pairs"] if bpp else None
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64acc" if prec == R.PREC_MIXED else "f64", "data": "synthetic",
            "config": {"workload": (f"33^3 voxels (0.1 cm), L=5, 3-sphere seeded phantom per step, {B} collimated "
                                    "z=0 sources from (+-0.825, +-0.825) cm solved as one batch" if B > 1 else
                                    "33^3 voxels (0.1 cm), L=5, 3-sphere seeded phantom per step, collimated "
                                    "centre source") + ", 20 Neumann terms + final A, z-face images",
                       "batch": B,
                       "precision": args.precision, "pair_kernel": "stored FP32 (recomputed per solve)"
                       if prec == R.PREC_MIXED else "recomputed per term",
                       "grid": N_SIDE, "L": L, "terms": TERMS,
                       "l2": f"inputs larger than L2: {counts['N'] ** 2 * 4 / 1e9:.1f} GB pair kernel streamed per term",
                       "parallelism": f"replicas x{ws}"},
            "roofline": {"bound": "fp32-cuda-core" if prec == R.PREC_MIXED else "fp64-cuda-core",
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": traffic, "kernel": f"k_pair_mixed_tk<5,{nbk}> (stored FP32 kernel staged by bulk copy)"
                         if prec == R.PREC_MIXED else "k_pair_fp64<5>", "avg_launch_ms": avg_pair_ms,
                         "flop_per_launch": apply_flop, "rhs_per_launch": nbk,
                         "peak_source": ("measured in this run by rte_measure_fma_peak (8 independent FMA chains "
                                         "per thread on every SM), of measured; theoretical FP32 148 SMs x 128 "
                                         "FMA/clk x 2 x 1.965 GHz = 74.4 TFLOP/s, FP64 half of it (37.2); "
                                         "MEASURED_PEAKS.json holds HBM and bf16 only"),
                         "hbm": hbm_line(traffic, avg_pair_ms)},
            "cpu_baseline": None,
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": st["launches"],
            "clocks": clocks,
            "fp64_rel_err": ref_err,
            "plain_fp64_solves_per_s": plain,
            "plain_fp64_stored_kernel_solves_per_s": plain_stored,
            "speedup_over_plain_fp64": {"recomputed": value / plain if plain else None,
                                        "stored_kernel": value / plain_stored if plain_stored else None},
            "kernel_ms_per_step": {"pair": st["ms_pair"] / args.steps, "store": st["ms_store"] / args.steps,
                                   "epilogue": st["ms_epi"] / args.steps},
            "solve_tflops_canonical": B * counts["solve_flop"] / (ms / args.steps / 1e3) / 1e12,
            "peaks_tflops": {"fp32": peak32, "fp64": peak64, **streams,
                             "streams": "fp32_* time one FP32 stream alone: scalar FMA, packed f32x2 FMA with "
                                        "reused operands, packed with three distinct operand registers"},
        }
        if ws == 1 and not args.skip_cpu:
            line["cpu_baseline"] = cpu_baseline(args.ref_seconds)
        if not args.skip_extras:
            line["config1_plain_fp64"] = run_cfg1(dev)
            line["config4_gradient"] = run_grad(dev)
            line["config5_fisher"] = run_fisher(dev, full_matrix_at_49=args.fisher_full)
            line["uniform_fft"] = run_uniform(dev)
        if args.serve_requests > 0 or args.serve_requests_33 > 0:
            line["serve"] = run_serve(args, dev)
            bs = line["serve"].get("bench_shape")
            if bs and plain:
                bs["vs_plain_fp64"] = {"recomputed": bs["capacity_solves_per_s"] / plain,
                                       "stored_kernel": bs["capacity_solves_per_s"] / plain_stored if plain_stored else None}
        out = line
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


def run_profile(args):
    """Small single-purpose runs for ncu captures (no timing line): --profile-grad N runs one mixed-
    precision gradient of the config-4 problem at N^3 (4 sources, 8x8 bins, 20 terms); --profile-fisher N
    one mixed-precision Fisher information at N^3, L=5 (1 face beam, 8 parameters, 16x16 bins, path
    integrals recomputed; --profile-order 7: L=7 and 4 parameters); --profile-uniform N three forward solves of a uniform N^3, L=5 medium through
    the FFT convolution path."""
    import doi_b200 as R
    if args.profile_grad:
        ctx, srcs, stop, det, target = grad_problem(0, n=args.profile_grad)
        loss, ga, gs = ctx.gradient(srcs, stop, det, target)
        ctx.close()
        print(json.dumps({"profile": "gradient", "n": args.profile_grad, "loss": loss}))
    if args.profile_fisher:
        Lq = args.profile_order
        F = run_fisher_case(0, args.profile_fisher, Lq, 16, TERMS, nsrc=1, P=8 if Lq <= 5 else 4,
                            kernel_mode=R.KERNEL_RECOMPUTE)[0]
        print(json.dumps({"profile": "fisher", "n": args.profile_fisher, "L": Lq, "F_trace": float(np.trace(F))}))
    if args.profile_uniform:
        n = args.profile_uniform
        with R.Context(n, n, n, dx=DX, nL=L, g=0.8, precision=R.PREC_MIXED, kernel_mode=R.KERNEL_AUTO) as ctx:
            ctx.set_medium_voxel(np.full(n ** 3, 0.01), np.full(n ** 3, 1.0))
            for _ in range(3):  # the first solve builds the table spectra and the transform plans
                r = ctx.forward(R.Source(kind=R.SRC_COLUMN), R.Stop(R.STOP_FIXED, TERMS), want_W=False)
        print(json.dumps({"profile": "uniform", "n": n, "ms_device": r["ms_device"]}))
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-fp64-check", action="store_true")
    ap.add_argument("--n", type=int, default=33, help="grid side (33 = the benchmark; smaller for profiling)")
    ap.add_argument("--batch", type=int, default=4, choices=[1, 2, 3, 4],
                    help="sources per phantom solved together (1 = one source per solve)")
    ap.add_argument("--skip-extras", action="store_true", help="skip the config-1, gradient and Fisher measurements")
    ap.add_argument("--fisher-full", action="store_true",
                    help="the whole 32 x 32 Fisher matrix at 49^3, L=7 instead of the bounded leg (long)")
    ap.add_argument("--serve-requests", type=int, default=64,
                    help="requests in the serving stream (0 = skip; 2000 = the full stream)")
    ap.add_argument("--profile-grad", type=int, default=0, help="one config-4 gradient at this grid side, then exit")
    ap.add_argument("--profile-fisher", type=int, default=0, help="one Fisher information at this grid side, then exit")
    ap.add_argument("--profile-order", type=int, default=5, choices=[5, 7],
                    help="SH order of --profile-fisher (5: 8 parameters; 7: 4 parameters, one four-RHS series)")
    ap.add_argument("--profile-uniform", type=int, default=0,
                    help="three uniform-medium solves (FFT convolution path) at this grid side, then exit")
    ap.add_argument("--serve-requests-33", type=int, default=32,
                    help="requests in the single-shape 33^3 L=5 serving stream (0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="Poisson arrival rate (requests/s); 0 = 0.7 x the capacity measured first")
    ap.add_argument("--serve-workers", type=int, default=4, help="requests in flight at most")
    args = ap.parse_args()
    global N_SIDE
    N_SIDE = args.n
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_grad or args.profile_fisher or args.profile_uniform:
        return run_profile(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
