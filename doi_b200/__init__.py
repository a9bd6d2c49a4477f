"""doi_b200: B200-native (sm_100a) Neumann-series radiative transport solver.

The compute path is the CUDA library doi_b200/lib/librte_b200.so (C ABI in include/rte_b200.h);
this package holds its build script, the ctypes binding and the phantom helpers.
"""
from .rte import (Context, RteError, Server, Source, Stop, Detector, load_library, MODEL_EXACT, MODEL_FIM, MODEL_CPU,
                  PREC_FP64, PREC_MIXED, KERNEL_AUTO, KERNEL_STORE, KERNEL_RECOMPUTE, SRC_COLUMN, SRC_FIM,
                  SRC_CPU, SRC_BEAM, SRC_POINT, STOP_REFERENCE, STOP_FIXED, STOP_REL_L2, DERIV_EXACT, DERIV_REFERENCE,
                  downsample_image)
from .inverse import reconstruct
from .phantoms import sphere_phantom, uniform_phantom, smooth_sphere_phantom, random_spheres

__all__ = ["reconstruct", "downsample_image", "Context", "RteError", "Server", "Source", "Stop", "Detector", "load_library", "sphere_phantom", "uniform_phantom",
           "MODEL_EXACT", "MODEL_FIM", "MODEL_CPU", "PREC_FP64", "PREC_MIXED", "KERNEL_AUTO", "KERNEL_STORE",
           "KERNEL_RECOMPUTE", "SRC_COLUMN", "SRC_FIM", "SRC_CPU", "SRC_BEAM", "SRC_POINT", "STOP_REFERENCE", "STOP_FIXED",
           "STOP_REL_L2", "DERIV_EXACT", "DERIV_REFERENCE"]
