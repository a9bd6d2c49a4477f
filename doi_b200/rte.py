"""Python binding of the C ABI in include/rte_b200.h (ctypes over doi_b200/lib/librte_b200.so).

Mirrors the reference entry points for the Neumann-series RTE path:
  Context.prop_abs      <- prop_abs()            FisherInfo_IO/src/kernels.cu:704-808
  Context.neumann       <- Neumann(src,out,flag)  FisherInfo_IO/src/neumann.cu:23-120
  Context.source_beam   <- generate_source_beam  FisherInfo_IO/src/dist.cu:66-101
  Context.images        <- generate_trans_image / generate_ref_image (dist.cu:103-268)
  Context.forward       <- the forward main      FisherInfo_IO/src/rte.cu:92-236
Distributions are complex128 arrays of shape (N, C), N = nX*nY*nZ (x fastest), C = (nL+1)^2.
Every failure raises RteError with the library's message; there is no CPU fallback: the library
must be built (python -m doi_b200.build) and a CUDA device present.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "librte_b200.so")

MODEL_EXACT, MODEL_FIM, MODEL_CPU = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
KERNEL_AUTO, KERNEL_STORE, KERNEL_RECOMPUTE = 0, 1, 2
SRC_COLUMN, SRC_FIM, SRC_CPU, SRC_BEAM, SRC_POINT = 0, 1, 2, 3, 4
STOP_REFERENCE, STOP_FIXED, STOP_REL_L2 = 0, 1, 2
DERIV_EXACT, DERIV_REFERENCE = 0, 1

# exported symbols of include/rte_b200.h (checked by the CPU tests)
EXPORTS = ("rte_create", "rte_destroy", "rte_last_error", "rte_device_bytes", "rte_set_medium_tissue",
           "rte_set_medium_voxel", "rte_set_medium_device", "rte_source_beam", "rte_prop_abs", "rte_neumann",
           "rte_images", "rte_forward", "rte_forward_batch", "rte_detector_flux", "rte_gradient",
           "rte_measure_fma_peak", "rte_get_stream", "rte_set_profiling", "rte_get_stats", "rte_forward_graph",
           "rte_server_create", "rte_server_submit", "rte_server_wait", "rte_server_cancel", "rte_server_stats",
           "rte_server_destroy", "rte_par_load", "rte_par_free", "rte_par_get_string", "rte_par_get_int",
           "rte_par_get_double", "rte_par_problem", "rte_problem_free", "rte_write_image", "rte_write_phase_image",
           "rte_read_image", "rte_region_gradient", "rte_fisher_regions", "rte_fisher",
           "rte_cpu_face_outputs", "rte_set_modulation", "rte_downsample_image", "rte_image_gradient",
           "rte_set_medium_tissue_split", "rte_prop_abs_adjoint")


class RteError(RuntimeError):
    pass


class _Config(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("x_min", ctypes.c_double), ("x_max", ctypes.c_double),
                ("y_min", ctypes.c_double), ("y_max", ctypes.c_double),
                ("z_min", ctypes.c_double), ("z_max", ctypes.c_double),
                ("nL", ctypes.c_int), ("prop_thresh", ctypes.c_double), ("self_sub_vox", ctypes.c_int),
                ("g", ctypes.c_double), ("n", ctypes.c_double), ("c", ctypes.c_double),
                ("model", ctypes.c_int), ("precision", ctypes.c_int), ("kernel_mode", ctypes.c_int),
                ("device", ctypes.c_int)]


class _Source(ctypes.Structure):
    _fields_ = [("pos_x", ctypes.c_double), ("pos_y", ctypes.c_double), ("pos_z", ctypes.c_double),
                ("diam", ctypes.c_double), ("theta", ctypes.c_double), ("phi", ctypes.c_double),
                ("mag", ctypes.c_double), ("modulation", ctypes.c_double), ("kind", ctypes.c_int),
                ("face", ctypes.c_int)]


class _Stop(ctypes.Structure):
    _fields_ = [("rule", ctypes.c_int), ("max_terms", ctypes.c_int), ("tol", ctypes.c_double)]


class _Detector(ctypes.Structure):
    _fields_ = [("nbins", ctypes.c_int), ("faces", ctypes.c_int)]


@dataclass
class Detector:
    """nbins x nbins bins on each face in the `faces` bit mask (1 z=0, 2 z=nZ-1, 4 y=0, 8 y=nY-1,
    16 x=0, 32 x=nX-1)."""
    nbins: int = 8
    faces: int = 63

    def c(self):
        return _Detector(self.nbins, self.faces)


class _Stats(ctypes.Structure):
    _fields_ = [("launches", ctypes.c_longlong), ("ms_pair", ctypes.c_double), ("n_pair", ctypes.c_longlong),
                ("ms_store", ctypes.c_double), ("n_store", ctypes.c_longlong), ("ms_epi", ctypes.c_double),
                ("n_epi", ctypes.c_longlong)]


class _Report(ctypes.Structure):
    _fields_ = [("terms", ctypes.c_int), ("last_rel", ctypes.c_double), ("ms_device", ctypes.c_double),
                ("ms_setup", ctypes.c_double)]


@dataclass
class Source:
    pos_x: float = 0.0
    pos_y: float = 0.0
    pos_z: float = 0.0
    diam: float = 0.2
    theta: float = 0.0
    phi: float = 0.0
    mag: float = 1.0
    modulation: float = 0.0
    kind: int = SRC_COLUMN
    face: int = 0

    def c(self):
        return _Source(self.pos_x, self.pos_y, self.pos_z, self.diam, self.theta, self.phi, self.mag,
                       self.modulation, self.kind, self.face)


@dataclass
class Stop:
    rule: int = STOP_FIXED
    max_terms: int = 20
    tol: float = 1e-7

    def c(self):
        return _Stop(self.rule, self.max_terms, self.tol)


class _Request(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("dx", ctypes.c_double), ("nL", ctypes.c_int), ("g", ctypes.c_double),
                ("n_index", ctypes.c_double), ("precision", ctypes.c_int), ("terms", ctypes.c_int),
                ("nsrc", ctypes.c_int), ("src", _Source * 4), ("mua", ctypes.c_void_p), ("mus", ctypes.c_void_p)]


class _Problem(ctypes.Structure):
    _fields_ = [("cfg", _Config), ("src", _Source), ("stop", _Stop), ("style", ctypes.c_int), ("ntypes", ctypes.c_int),
                ("mua", ctypes.c_double * 256), ("mus", ctypes.c_double * 256), ("tiss", ctypes.c_void_p),
                ("mua_vox", ctypes.c_void_p), ("mus_vox", ctypes.c_void_p), ("mut_mean", ctypes.c_double),
                ("diffuse_prop_thresh", ctypes.c_double), ("nterms", ctypes.c_int), ("detector_bins", ctypes.c_int),
                ("num_iterations", ctypes.c_int), ("step_a", ctypes.c_double), ("step_s", ctypes.c_double),
                ("trans_file", ctypes.c_char * 1024), ("ref_file", ctypes.c_char * 1024),
                ("phase_file", ctypes.c_char * 1024), ("g_file", ctypes.c_char * 1024),
                ("flux_file", ctypes.c_char * 1024)]


class _ResultInfo(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("service_ms", ctypes.c_double), ("device_ms", ctypes.c_double)]


class _ServerInfo(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("cancelled", ctypes.c_longlong), ("inflight", ctypes.c_longlong), ("pending", ctypes.c_longlong),
                ("contexts", ctypes.c_int), ("hbm_reserved", ctypes.c_size_t), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("wall_s", ctypes.c_double)]


_LIB = None


def load_library():
    """Load librte_b200.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RteError(f"{LIB_PATH} is missing: build it with `python -m doi_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    dp = ctypes.c_void_p
    L.rte_create.argtypes = [ctypes.POINTER(_Config), ctypes.POINTER(ctypes.c_void_p)]
    L.rte_destroy.argtypes = [P]
    L.rte_destroy.restype = None
    L.rte_last_error.argtypes = [P]
    L.rte_last_error.restype = ctypes.c_char_p
    L.rte_device_bytes.argtypes = [P]
    L.rte_device_bytes.restype = ctypes.c_size_t
    L.rte_set_medium_tissue.argtypes = [P, dp, ctypes.c_int, dp, dp]
    L.rte_set_medium_tissue_split.argtypes = [P, dp, ctypes.c_int, dp, dp, dp, dp]
    L.rte_set_medium_voxel.argtypes = [P, dp, dp]
    L.rte_set_medium_device.argtypes = [P, dp, dp]
    L.rte_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.rte_get_stream.argtypes = [P]
    L.rte_get_stream.restype = ctypes.c_void_p
    L.rte_set_profiling.argtypes = [P, ctypes.c_int]
    L.rte_get_stats.argtypes = [P, ctypes.POINTER(_Stats)]
    L.rte_source_beam.argtypes = [P, ctypes.POINTER(_Source), dp]
    L.rte_prop_abs.argtypes = [P, dp, dp, ctypes.c_int, ctypes.c_int]
    L.rte_prop_abs_adjoint.argtypes = [P, dp, dp, ctypes.c_int]
    L.rte_neumann.argtypes = [P, dp, dp, ctypes.c_int, ctypes.POINTER(_Stop), ctypes.POINTER(ctypes.c_int)]
    L.rte_images.argtypes = [P, dp, ctypes.POINTER(_Source), dp, dp]
    L.rte_forward.argtypes = [P, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), dp, dp, dp,
                              ctypes.POINTER(_Report)]
    L.rte_detector_flux.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Source), ctypes.POINTER(_Stop),
                                    ctypes.POINTER(_Detector), dp]
    L.rte_gradient.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Source), ctypes.POINTER(_Stop),
                               ctypes.POINTER(_Detector), dp, ctypes.POINTER(ctypes.c_double), dp, dp]
    L.rte_image_gradient.argtypes = [P, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), ctypes.c_int, ctypes.c_int, dp,
                                     ctypes.POINTER(ctypes.c_double), dp, dp]
    L.rte_forward_batch.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), dp, dp, dp,
                                    ctypes.POINTER(_Report)]
    L.rte_forward_graph.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Source), ctypes.c_int, dp, dp,
                                    ctypes.POINTER(_Report)]
    L.rte_server_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.rte_server_submit.argtypes = [P, ctypes.POINTER(_Request), ctypes.POINTER(ctypes.c_longlong)]
    L.rte_server_wait.argtypes = [P, ctypes.c_longlong, ctypes.c_double, dp, dp, ctypes.POINTER(_ResultInfo)]
    L.rte_server_cancel.argtypes = [P, ctypes.c_longlong]
    L.rte_server_stats.argtypes = [P, ctypes.POINTER(_ServerInfo)]
    L.rte_server_destroy.argtypes = [P]
    L.rte_server_destroy.restype = None
    L.rte_par_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]
    L.rte_par_free.argtypes = [P]
    L.rte_par_free.restype = None
    L.rte_par_get_string.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p]
    L.rte_par_get_string.restype = ctypes.c_char_p
    L.rte_par_get_int.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
    L.rte_par_get_double.argtypes = [P, ctypes.c_char_p, ctypes.c_double]
    L.rte_par_get_double.restype = ctypes.c_double
    L.rte_par_problem.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Problem)]
    L.rte_problem_free.argtypes = [ctypes.POINTER(_Problem)]
    L.rte_problem_free.restype = None
    L.rte_write_image.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
    L.rte_write_phase_image.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int]
    L.rte_set_modulation.argtypes = [P, ctypes.c_double]
    L.rte_read_image.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, dp]
    L.rte_downsample_image.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp]
    L.rte_region_gradient.argtypes = [P, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), dp, dp, ctypes.c_int,
                                      ctypes.c_int, dp, dp, dp, dp, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double)]
    L.rte_cpu_face_outputs.argtypes = [ctypes.POINTER(_Config), dp, ctypes.POINTER(_Source), ctypes.c_double,
                                       ctypes.c_double, dp, dp, dp, dp, dp]
    L.rte_fisher.argtypes = [P, ctypes.c_int, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), ctypes.POINTER(_Detector),
                             ctypes.c_int, dp, dp, dp, dp]
    L.rte_fisher_regions.argtypes = [P, ctypes.POINTER(_Source), ctypes.POINTER(_Stop), ctypes.c_int, dp, ctypes.c_int,
                                     dp]
    _LIB = L
    return L


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


FMA_STREAMS = {"fp32": 0, "fp64": 1, "fp32_scalar": 2, "fp32_packed": 3, "fp32_packed_fresh": 4}


def measure_fma_peak(fp64=False, device=0, stream=None):
    """Measured FMA throughput (TFLOP/s) of the device's CUDA cores: FP32 (the faster of the scalar and
    packed streams) or FP64, or one named stream of FMA_STREAMS."""
    lib = load_library()
    v = ctypes.c_double(0.0)
    mode = FMA_STREAMS[stream] if stream is not None else int(bool(fp64))
    rc = lib.rte_measure_fma_peak(device, mode, ctypes.byref(v))
    if rc != 0:
        raise RteError(f"rte_measure_fma_peak failed ({rc})")
    return v.value


class Context:
    """One solver context on one GPU (rte_create / rte_destroy)."""

    def __init__(self, nx, ny, nz, dx=0.1, dy=None, dz=None, nL=3, g=0.8, n=1.0, c=1.0, prop_thresh=None,
                 model=MODEL_EXACT, precision=PREC_FP64, kernel_mode=KERNEL_AUTO, self_sub_vox=1, device=0,
                 x_min=None, x_max=None, y_min=None, y_max=None, z_min=0.0, z_max=None):
        dy = dx if dy is None else dy
        dz = dx if dz is None else dz
        x_min = -nx * dx / 2 if x_min is None else x_min
        x_max = x_min + nx * dx if x_max is None else x_max
        y_min = -ny * dy / 2 if y_min is None else y_min
        y_max = y_min + ny * dy if y_max is None else y_max
        z_max = z_min + nz * dz if z_max is None else z_max
        if prop_thresh is None:  # couple every pair
            prop_thresh = 2.0 * np.sqrt((nx * dx) ** 2 + (ny * dy) ** 2 + (nz * dz) ** 2)
        self.lib = load_library()
        self.nx, self.ny, self.nz, self.nL = nx, ny, nz, nL
        self.N = nx * ny * nz
        self.C = (nL + 1) ** 2
        cfg = _Config(nx, ny, nz, x_min, x_max, y_min, y_max, z_min, z_max, nL, prop_thresh, self_sub_vox,
                      g, n, c, model, precision, kernel_mode, device)
        h = ctypes.c_void_p()
        rc = self.lib.rte_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise RteError(f"rte_create failed ({rc}): {self.lib.rte_last_error(None).decode()}")
        self.h = h
        self.cfg = cfg

    def close(self):
        if getattr(self, "h", None):
            self.lib.rte_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc, what):
        if rc != 0:
            raise RteError(f"{what} failed ({rc}): {self.lib.rte_last_error(self.h).decode()}")

    def stream_ptr(self):
        """cudaStream_t of this context (wrap with torch.cuda.ExternalStream to time on it)."""
        return int(self.lib.rte_get_stream(self.h) or 0)

    def set_profiling(self, on=True):
        self._check(self.lib.rte_set_profiling(self.h, int(bool(on))), "rte_set_profiling")

    def stats(self):
        """Launch count and per-class kernel times since the last call (synchronises)."""
        st = _Stats()
        self._check(self.lib.rte_get_stats(self.h, ctypes.byref(st)), "rte_get_stats")
        return {k: getattr(st, k) for k, _ in _Stats._fields_}

    def device_bytes(self):
        return int(self.lib.rte_device_bytes(self.h))

    def set_medium_voxel(self, mua, mus):
        mua = np.ascontiguousarray(mua, np.float64).ravel()
        mus = np.ascontiguousarray(mus, np.float64).ravel()
        if mua.size != self.N or mus.size != self.N:
            raise RteError("medium arrays must have nX*nY*nZ entries")
        self._check(self.lib.rte_set_medium_voxel(self.h, _ptr(mua), _ptr(mus)), "rte_set_medium_voxel")

    def set_medium_device(self, mua_ptr, mus_ptr):
        """Medium from device pointers (e.g. torch.Tensor.data_ptr() of float64 CUDA tensors)."""
        self._check(self.lib.rte_set_medium_device(self.h, ctypes.c_void_p(mua_ptr), ctypes.c_void_p(mus_ptr)),
                    "rte_set_medium_device")

    def set_medium_tissue(self, tiss, mua_tab, mus_tab):
        tiss = np.ascontiguousarray(tiss, np.uint8).ravel()
        a = np.ascontiguousarray(mua_tab, np.float64)
        s = np.ascontiguousarray(mus_tab, np.float64)
        self._check(self.lib.rte_set_medium_tissue(self.h, _ptr(tiss), len(a), _ptr(a), _ptr(s)),
                    "rte_set_medium_tissue")

    def set_medium_tissue_split(self, tiss, mua_tab, mus_tab, mua_kernel, mus_kernel):
        """Tissue map with two tables: the self-voxel term, source and ballistic beam take (mua_tab, mus_tab),
        the pair kernels and the scatter (mua_kernel, mus_kernel), as in the reference's SNR and
        region-gradient mains (rte_set_medium_tissue_split)."""
        tiss = np.ascontiguousarray(tiss, np.uint8).ravel()
        tabs = [np.ascontiguousarray(t, np.float64) for t in (mua_tab, mus_tab, mua_kernel, mus_kernel)]
        n = len(tabs[0])
        if any(len(t) != n for t in tabs):
            raise ValueError("the four tables must have the same length")
        self._check(self.lib.rte_set_medium_tissue_split(self.h, _ptr(tiss), n, *[_ptr(t) for t in tabs]),
                    "rte_set_medium_tissue_split", "rte_prop_abs_adjoint")

    def set_modulation(self, modulation):
        """Intensity modulation: mu_a -> mu_a + i*modulation/(c/n) (the reference's [Source] modulation);
        0 restores the steady state.  rte_forward solves at its source's own modulation."""
        self._check(self.lib.rte_set_modulation(self.h, float(modulation)), "rte_set_modulation")

    def _dist(self, W):
        W = np.ascontiguousarray(W, np.complex128).reshape(self.N, self.C)
        return W

    def source_beam(self, src):
        out = np.zeros((self.N, self.C), np.complex128)
        s = src.c()
        self._check(self.lib.rte_source_beam(self.h, ctypes.byref(s), _ptr(out)), "rte_source_beam")
        return out

    def prop_abs(self, W, flag=1, flag_scat=1):
        W = self._dist(W)
        out = np.zeros_like(W)
        self._check(self.lib.rte_prop_abs(self.h, _ptr(W), _ptr(out), flag, flag_scat), "rte_prop_abs")
        return out

    def prop_abs_adjoint(self, W, flag=1):
        """A^H W: the adjoint of prop_abs without scatter (rte_prop_abs_adjoint)."""
        W = self._dist(W)
        out = np.zeros_like(W)
        self._check(self.lib.rte_prop_abs_adjoint(self.h, _ptr(W), _ptr(out), flag), "rte_prop_abs_adjoint")
        return out

    def neumann(self, src, out, flag=1, stop=None):
        stop = stop or Stop()
        src = self._dist(src)
        o = np.array(self._dist(out), copy=True)
        nt = ctypes.c_int(0)
        st = stop.c()
        self._check(self.lib.rte_neumann(self.h, _ptr(src), _ptr(o), flag, ctypes.byref(st), ctypes.byref(nt)),
                    "rte_neumann")
        return o, nt.value

    def images(self, out, src=None):
        out = self._dist(out)
        tr = np.zeros(self.nx * self.ny, np.complex128)
        rf = np.zeros(self.nx * self.ny, np.complex128)
        s = src.c() if src is not None else None
        self._check(self.lib.rte_images(self.h, _ptr(out), ctypes.byref(s) if s is not None else None,
                                        _ptr(tr), _ptr(rf)), "rte_images")
        return tr.reshape(self.ny, self.nx), rf.reshape(self.ny, self.nx)

    def detector_flux(self, srcs, stop, det):
        """Binned exitant flux, shape (len(srcs), 6, nbins, nbins)."""
        B = len(srcs)
        out = np.zeros((B, 6, det.nbins, det.nbins))
        arr = (_Source * B)(*[s.c() for s in srcs])
        st, d = stop.c(), det.c()
        self._check(self.lib.rte_detector_flux(self.h, B, arr, ctypes.byref(st), ctypes.byref(d), _ptr(out)),
                    "rte_detector_flux")
        return out

    def gradient(self, srcs, stop, det, target):
        """(loss, dL/dmu_a, dL/dmu_s) for loss = sum (flux - target)^2, by the adjoint method."""
        B = len(srcs)
        target = np.ascontiguousarray(target, np.float64).reshape(B, 6, det.nbins, det.nbins)
        ga = np.zeros(self.N)
        gs = np.zeros(self.N)
        loss = ctypes.c_double(0.0)
        arr = (_Source * B)(*[s.c() for s in srcs])
        st, d = stop.c(), det.c()
        self._check(self.lib.rte_gradient(self.h, B, arr, ctypes.byref(st), ctypes.byref(d), _ptr(target),
                                          ctypes.byref(loss), _ptr(ga), _ptr(gs)), "rte_gradient")
        return loss.value, ga, gs

    def image_gradient(self, src, stop, g, image=0, deriv=DERIV_EXACT):
        """(loss, dL/dmu_a, dL/dmu_s) for the reference's image misfit loss = sum (gbar - g)^2 of one
        source's transmission (image=0) or reflection (image=1) image, from one forward and one adjoint
        series; deriv=DERIV_REFERENCE gives the reference's tangent model (rte_image_gradient)."""
        g = np.ascontiguousarray(g, np.float64).ravel()
        if g.size != self.nx * self.ny:
            raise ValueError("g must hold nX*nY values")
        ga = np.zeros(self.N)
        gs = np.zeros(self.N)
        loss = ctypes.c_double(0.0)
        s, st = src.c(), stop.c()
        self._check(self.lib.rte_image_gradient(self.h, ctypes.byref(s), ctypes.byref(st), int(image), int(deriv),
                                                _ptr(g), ctypes.byref(loss), _ptr(ga), _ptr(gs)), "rte_image_gradient")
        return loss.value, ga, gs

    def _outputs(self, out, shapes):
        """Result arrays: those given in out (C-contiguous complex128 of the right shape, e.g. views of
        pinned host memory, written in place), else fresh zeros."""
        res = []
        for key, shape in shapes:
            if shape is None:
                res.append(None)
                continue
            a = (out or {}).get(key)
            if a is None:
                a = np.zeros(shape, np.complex128)
            elif (not isinstance(a, np.ndarray) or a.dtype != np.complex128 or a.shape != shape
                  or not a.flags.c_contiguous):
                raise RteError(f"out[{key!r}] must be a C-contiguous complex128 array of shape {shape}")
            res.append(a)
        return res

    def forward_batch(self, srcs, stop=None, want_W=True, want_images=True, out=None):
        """Several sources on the current medium in one batched solve; returns the per-source results
        stacked along a leading axis.  out may hold preallocated arrays "W", "trans", "ref" to write."""
        stop = stop or Stop()
        B = len(srcs)
        W, tr, rf = self._outputs(out, (("W", (B, self.N, self.C) if want_W else None),
                                        ("trans", (B, self.ny, self.nx) if want_images else None),
                                        ("ref", (B, self.ny, self.nx) if want_images else None)))
        arr = (_Source * B)(*[s.c() for s in srcs])
        rep = _Report()
        st = stop.c()
        self._check(self.lib.rte_forward_batch(self.h, B, arr, ctypes.byref(st), _ptr(W), _ptr(tr), _ptr(rf),
                                               ctypes.byref(rep)), "rte_forward_batch")
        res = dict(terms=rep.terms, last_rel=rep.last_rel, ms_device=rep.ms_device, ms_setup=rep.ms_setup)
        if want_W:
            res["W"] = W
        if want_images:
            res["trans"], res["ref"] = tr, rf
        return res

    def region_gradient(self, src, stop, g, tiss, ntypes, compat=True):
        """Region derivatives of the reference's inverse main: (grada, grada2, grads, grads2, residual,
        residual2) with one entry per tissue type."""
        g = np.ascontiguousarray(g, np.float64).ravel()
        tiss = np.ascontiguousarray(tiss, np.uint8).ravel()
        out = [np.zeros(ntypes) for _ in range(4)]
        r1, r2 = ctypes.c_double(0), ctypes.c_double(0)
        s, st = src.c(), stop.c()
        self._check(self.lib.rte_region_gradient(self.h, ctypes.byref(s), ctypes.byref(st), _ptr(g), _ptr(tiss), ntypes,
                                                 int(bool(compat)), *[_ptr(o) for o in out], ctypes.byref(r1),
                                                 ctypes.byref(r2)), "rte_region_gradient")
        return (*out, r1.value, r2.value)

    def fisher(self, srcs, stop, det, dmua, dmus, want_J=False):
        """Poisson Fisher information (P x P) of the parameters whose per-voxel derivatives are
        dmua, dmus (P x N), from tangent solves; with want_J also J, shape
        (len(srcs), 6, nbins, nbins, P)."""
        dmua = np.ascontiguousarray(np.asarray(dmua, np.float64).reshape(-1, self.N))
        dmus = np.ascontiguousarray(np.asarray(dmus, np.float64).reshape(-1, self.N))
        P = dmua.shape[0]
        B = len(srcs)
        F = np.zeros((P, P))
        J = np.zeros((B, 6, det.nbins, det.nbins, P)) if want_J else None
        arr = (_Source * B)(*[x.c() for x in srcs])
        st, d = stop.c(), det.c()
        self._check(self.lib.rte_fisher(self.h, B, arr, ctypes.byref(st), ctypes.byref(d), P, _ptr(dmua), _ptr(dmus),
                                        _ptr(J), _ptr(F)), "rte_fisher")
        return (F, J) if want_J else F

    def fisher_regions(self, src, stop, masks, image=1):
        """Poisson Fisher information of the mu_a of each region in masks (P x N booleans)."""
        masks = np.ascontiguousarray(np.asarray(masks).reshape(-1, self.N), np.uint8)
        P = masks.shape[0]
        F = np.zeros((P, P))
        s, st = src.c(), stop.c()
        self._check(self.lib.rte_fisher_regions(self.h, ctypes.byref(s), ctypes.byref(st), P, _ptr(masks), image,
                                                _ptr(F)), "rte_fisher_regions")
        return F

    def forward_graph(self, srcs, nterms):
        """Fixed-term forward solve of up to 4 sources, replayed from a CUDA graph recorded on the
        first call; returns (trans, ref) stacked per source and the device time in ms."""
        B = len(srcs)
        tr = np.zeros((B, self.ny, self.nx), np.complex128)
        rf = np.zeros((B, self.ny, self.nx), np.complex128)
        arr = (_Source * B)(*[s.c() for s in srcs])
        rep = _Report()
        self._check(self.lib.rte_forward_graph(self.h, B, arr, int(nterms), _ptr(tr), _ptr(rf), ctypes.byref(rep)),
                    "rte_forward_graph")
        return tr, rf, rep.ms_device

    def forward(self, src, stop=None, want_W=True, want_images=True, out=None):
        stop = stop or Stop()
        W, tr, rf = self._outputs(out, (("W", (self.N, self.C) if want_W else None),
                                        ("trans", (self.nx * self.ny,) if want_images else None),
                                        ("ref", (self.nx * self.ny,) if want_images else None)))
        rep = _Report()
        s, st = src.c(), stop.c()
        self._check(self.lib.rte_forward(self.h, ctypes.byref(s), ctypes.byref(st), _ptr(W), _ptr(tr), _ptr(rf),
                                         ctypes.byref(rep)), "rte_forward")
        res = dict(terms=rep.terms, last_rel=rep.last_rel, ms_device=rep.ms_device, ms_setup=rep.ms_setup)
        if want_W:
            res["W"] = W
        if want_images:
            res["trans"] = tr.reshape(self.ny, self.nx)
            res["ref"] = rf.reshape(self.ny, self.nx)
        return res


class Server:
    """Continuous-batching forward-solve server on one GPU (rte_server_*).

    submit() copies the request and returns a ticket at once; requests of any grid / order / medium
    run concurrently as HBM and worker slots allow; wait() returns (trans, ref, info)."""

    def __init__(self, device=0, hbm_budget_gb=0.0, workers=4):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.rte_server_create(device, float(hbm_budget_gb), int(workers), ctypes.byref(h))
        if rc != 0:
            raise RteError(f"rte_server_create failed ({rc}): {self.lib.rte_last_error(None).decode()}")
        self.h = h
        self._shape = {}

    def submit(self, mua, mus, srcs, n, dx=0.1, nL=3, g=0.8, n_index=1.0, precision=PREC_MIXED, terms=12):
        mua = np.ascontiguousarray(mua, np.float64).ravel()
        mus = np.ascontiguousarray(mus, np.float64).ravel()
        if mua.size != n ** 3 or mus.size != n ** 3:
            raise RteError("medium arrays must have n^3 entries")
        if not 1 <= len(srcs) <= 4:
            raise RteError("1 to 4 sources per request")
        rq = _Request()
        rq.n, rq.dx, rq.nL, rq.g, rq.n_index = n, dx, nL, g, n_index
        rq.precision, rq.terms, rq.nsrc = precision, terms, len(srcs)
        for i, s in enumerate(srcs):
            rq.src[i] = s.c()
        rq.mua, rq.mus = mua.ctypes.data, mus.ctypes.data
        t = ctypes.c_longlong(0)
        rc = self.lib.rte_server_submit(self.h, ctypes.byref(rq), ctypes.byref(t))
        if rc != 0:
            raise RteError(f"rte_server_submit failed ({rc}): {self.lib.rte_last_error(None).decode()}")
        self._shape[t.value] = (len(srcs), n)
        return t.value

    def wait(self, ticket, timeout=600.0):
        B, n = self._shape[ticket]
        tr = np.zeros((B, n, n), np.complex128)
        rf = np.zeros((B, n, n), np.complex128)
        info = _ResultInfo()
        rc = self.lib.rte_server_wait(self.h, ticket, float(timeout), _ptr(tr), _ptr(rf), ctypes.byref(info))
        if rc == 7:  # RTE_ERR_TIMEOUT: the ticket stays valid
            raise TimeoutError(f"request {ticket} still running")
        del self._shape[ticket]
        if rc != 0:
            raise RteError(f"request {ticket} failed ({rc}): {self.lib.rte_last_error(None).decode()}")
        return tr, rf, {k: getattr(info, k) for k, _ in _ResultInfo._fields_}

    def cancel(self, ticket):
        return self.lib.rte_server_cancel(self.h, ticket) == 0

    def stats(self):
        st = _ServerInfo()
        if self.lib.rte_server_stats(self.h, ctypes.byref(st)) != 0:
            raise RteError("rte_server_stats failed")
        return {k: getattr(st, k) for k, _ in _ServerInfo._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.rte_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ParFile:
    """A reference .par file read by the library's parser (section:key lookups, iniparser rules)."""

    def __init__(self, path):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.rte_par_load(os.fsencode(path), ctypes.byref(h))
        if rc != 0:
            raise RteError(f"rte_par_load({path}) failed ({rc})")
        self.h = h

    def get(self, key, default=None):
        v = self.lib.rte_par_get_string(self.h, key.encode(), None)
        return default if v is None else v.decode()

    def get_int(self, key, default=0):
        return self.lib.rte_par_get_int(self.h, key.encode(), default)

    def get_double(self, key, default=0.0):
        return self.lib.rte_par_get_double(self.h, key.encode(), default)

    def problem(self, read_map=True):
        """The solver inputs the reference mains derive from this file (a dict)."""
        pr = _Problem()
        rc = self.lib.rte_par_problem(self.h, int(bool(read_map)), ctypes.byref(pr))
        if rc != 0:
            raise RteError(f"rte_par_problem failed ({rc})")
        try:
            c = pr.cfg
            N = c.nx * c.ny * c.nz
            out = {k: getattr(c, k) for k, _ in _Config._fields_}
            out["source"] = {k: getattr(pr.src, k) for k, _ in _Source._fields_}
            out["stop"] = {k: getattr(pr.stop, k) for k, _ in _Stop._fields_}
            for k in ("style", "ntypes", "mut_mean", "diffuse_prop_thresh", "nterms", "detector_bins",
                      "num_iterations", "step_a", "step_s"):
                out[k] = getattr(pr, k)
            for k in ("trans_file", "ref_file", "phase_file", "g_file", "flux_file"):
                out[k] = getattr(pr, k).decode()
            out["mua_tab"] = np.array(pr.mua[:pr.ntypes])
            out["mus_tab"] = np.array(pr.mus[:pr.ntypes])
            out["tiss"] = np.ctypeslib.as_array(ctypes.cast(pr.tiss, ctypes.POINTER(ctypes.c_uint8)), (N,)).copy() \
                if pr.tiss else None
            return out
        finally:
            self.lib.rte_problem_free(ctypes.byref(pr))

    def close(self):
        if getattr(self, "h", None):
            self.lib.rte_par_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_image(path, img, cpu_layout=False):
    img = np.ascontiguousarray(img, np.complex128)
    ny, nx = img.shape
    rc = load_library().rte_write_image(os.fsencode(path), nx, ny, _ptr(img), int(bool(cpu_layout)))
    if rc != 0:
        raise RteError(f"rte_write_image failed ({rc})")


def write_phase_image(path, phase, cpu_layout=False):
    """Phase image: FisherInfo_IO layout (nY, nX header) or the CPU package's (nX, nY header)."""
    phase = np.ascontiguousarray(phase, np.float64)
    ny, nx = phase.shape
    rc = load_library().rte_write_phase_image(os.fsencode(path), nx, ny, _ptr(phase), int(bool(cpu_layout)))
    if rc != 0:
        raise RteError(f"rte_write_phase_image failed ({rc})")


def read_image(path, nx, ny):
    out = np.zeros(nx * ny)
    rc = load_library().rte_read_image(os.fsencode(path), nx, ny, _ptr(out))
    if rc != 0:
        raise RteError(f"rte_read_image failed ({rc})")
    return out.reshape(ny, nx)


def downsample_image(img, ds):
    """Block sums of an nY x nX image (the reference's downsample_image, FisherInfo_IO/src/dist.cu:271-289):
    returns an (nX//ds) x (nY//ds) complex array; rows/columns beyond the last whole block are dropped."""
    img = np.ascontiguousarray(img, np.complex128)
    ny, nx = img.shape
    if ds < 1 or ds > nx or ds > ny:
        raise RteError(f"rte_downsample_image: bad factor {ds} for a {nx} x {ny} image")
    out = np.zeros((nx // ds, ny // ds), np.complex128)
    rc = load_library().rte_downsample_image(_ptr(img), nx, ny, int(ds), _ptr(out))
    if rc != 0:
        raise RteError(f"rte_downsample_image failed ({rc})")
    return out


def cpu_face_outputs(W, nx, ny, nz, nL, x_min, x_max, y_min, y_max, z_min, z_max, src, mu_t, c=1.0, n=1.0):
    """The CPU package's side-face images (-x, +x, -y, +y; x faces (nY, nZ), y faces (nX, nZ)) and
    photon number of a final distribution W (N x C complex, reference layout); host computation.
    mu_t may be complex (intensity modulation: mu_t + i*modulation/(c/n))."""
    lib = load_library()
    cfg = _Config(nx, ny, nz, x_min, x_max, y_min, y_max, z_min, z_max, nL, 0.0, 1, 0.0, n, c, MODEL_CPU, 0, 0, 0)
    W = np.ascontiguousarray(W, np.complex128)
    sx0 = np.zeros(nz * ny, np.complex128)
    sx1 = np.zeros(nz * ny, np.complex128)
    sy0 = np.zeros(nz * nx, np.complex128)
    sy1 = np.zeros(nz * nx, np.complex128)
    ph = np.zeros(1, np.complex128)
    s = src.c()
    mu_t = complex(mu_t)
    rc = lib.rte_cpu_face_outputs(ctypes.byref(cfg), _ptr(W), ctypes.byref(s), mu_t.real, mu_t.imag, _ptr(sx0),
                                  _ptr(sx1), _ptr(sy0), _ptr(sy1), _ptr(ph))
    if rc != 0:
        raise RteError(f"rte_cpu_face_outputs failed ({rc})")
    return [sx0.reshape(ny, nz), sx1.reshape(ny, nz), sy0.reshape(nx, nz), sy1.reshape(nx, nz)], ph[0]
