"""The C-ABI library without a GPU: it loads, exports every function include/rte_b200.h declares, and
fails with a status code and a message (never a crash, never a CPU fallback) when no device exists."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "rte_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rte_[a-z0-9_]+)\s*\(", src)))


def test_header_parses():
    names = _declared()
    assert "rte_neumann" in names and "rte_prop_abs" in names and "rte_attenuate_noalloc" in names


def test_library_exports_every_declared_symbol(rte):
    lib = rte.load_library()
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing
    assert set(rte.rte.EXPORTS) <= set(_declared())


def test_create_without_device_fails_loudly(rte):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(rte.RteError) as e:
        rte.Context(5, 5, 5, nL=2)
    assert "rte_create failed" in str(e.value)


def test_bad_config_rejected(rte):
    lib = rte.load_library()
    from doi_b200.rte import _Config
    h = ctypes.c_void_p()
    cfg = _Config(0, 5, 5, -1, 1, -1, 1, 0, 1, 3, 10.0, 1, 0.8, 1.0, 1.0, 0, 0, 0, 0)
    assert lib.rte_create(ctypes.byref(cfg), ctypes.byref(h)) == 1  # RTE_ERR_ARG
    assert b"grid" in lib.rte_last_error(None)
    cfg = _Config(5, 5, 5, -1, 1, -1, 1, 0, 1, 9, 10.0, 1, 0.8, 1.0, 1.0, 0, 0, 0, 0)
    assert lib.rte_create(ctypes.byref(cfg), ctypes.byref(h)) == 6  # RTE_ERR_UNSUPPORTED (nL > 7)


def test_noalloc_rejects_bad_arguments_without_device(rte):
    lib = rte.load_library()
    f = lib.rte_attenuate_noalloc
    f.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                                 ctypes.c_void_p]
    assert f(0, 4, 4, 0.1, 0.1, 0.1, 2, 1.0, 1.0, None, None, None, None) == 1
    # too large for the built-in scratch: rejected before any device work
    assert f(128, 128, 128, 0.1, 0.1, 0.1, 7, 1.0, 1.0, 1, 1, 1, None) == 6
    assert b"scratch" in lib.rte_last_error(None)


NULL_IS_ERROR = ["rte_set_medium_tissue", "rte_set_medium_tissue_split", "rte_set_medium_voxel", "rte_set_medium_device", "rte_set_modulation",
                 "rte_source_beam", "rte_prop_abs", "rte_prop_abs_adjoint", "rte_neumann", "rte_images", "rte_forward",
                 "rte_detector_flux", "rte_gradient", "rte_image_gradient", "rte_region_gradient", "rte_fisher_regions", "rte_fisher",
                 "rte_forward_batch", "rte_forward_graph", "rte_server_submit", "rte_server_wait",
                 "rte_server_cancel", "rte_server_stats", "rte_set_profiling", "rte_get_stats", "rte_par_load",
                 "rte_par_problem", "rte_write_image", "rte_write_phase_image", "rte_read_image",
                 "rte_downsample_image", "rte_cpu_face_outputs", "rte_server_create", "rte_attenuate_noalloc",
                 "rte_measure_fma_peak"]
NULL_IS_NOOP = ["rte_destroy", "rte_device_bytes", "rte_server_destroy", "rte_get_stream", "rte_par_free",
                "rte_problem_free", "rte_last_error"]


def test_null_arguments_give_status_codes(rte):
    """Every entry point given null pointers (and zero sizes) returns an error status or does nothing;
    none dereferences them.  Run in a child process so that a crash is a test failure."""
    import subprocess
    import sys
    lib_path = rte.rte.LIB_PATH
    code = f"""
import ctypes
lib = ctypes.CDLL({lib_path!r})
for name in {NULL_IS_ERROR + NULL_IS_NOOP!r}:
    f = getattr(lib, name)
    f.restype = ctypes.c_longlong
    print(name, f(*([None] * 12)))
"""
    r = subprocess.run([sys.executable, "-c", code], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout[-2000:]
    got = dict(line.split() for line in r.stdout.split("\n") if line.strip())
    for name in NULL_IS_ERROR:
        assert int(got[name]) != 0, name
    assert all(name in got for name in NULL_IS_NOOP)


def test_server_errors_carry_messages(rte):
    """rte_server_create failures (bad worker count; no device here) leave a reason for
    rte_last_error(NULL), which the Python mirror puts in its exception."""
    import torch
    with pytest.raises(rte.RteError) as e:
        rte.Server(device=0, workers=0)
    assert "nworkers" in str(e.value)
    if not torch.cuda.is_available():
        with pytest.raises(rte.RteError) as e:
            rte.Server(device=0, workers=2)
        msg = str(e.value).split("):", 1)[1].strip()
        assert msg


def test_preallocated_outputs_are_checked(rte):
    """forward / forward_batch out= arrays: used as given when complex128, C-contiguous and of the
    result's shape; anything else is refused before the library is called."""
    import numpy as np
    shapes = (("W", (2, 8, 4)), ("trans", None), ("ref", (2, 3, 3)))
    w = np.zeros((2, 8, 4), np.complex128)
    got = rte.Context._outputs(None, {"W": w}, shapes)
    assert got[0] is w and got[1] is None and got[2].shape == (2, 3, 3)
    for bad in (np.zeros((2, 8, 4)), np.zeros((2, 8, 5), np.complex128),
                np.zeros((2, 4, 8), np.complex128).transpose(0, 2, 1)):
        with pytest.raises(rte.RteError):
            rte.Context._outputs(None, {"W": bad}, shapes)


def test_fma_peak_rejects_unknown_stream(rte):
    """rte_measure_fma_peak takes modes 0-4 only; others are refused before any device call."""
    lib = rte.load_library()
    v = ctypes.c_double(0.0)
    for mode in (-1, 5):
        assert lib.rte_measure_fma_peak(0, mode, ctypes.byref(v)) == 1  # RTE_ERR_ARG
