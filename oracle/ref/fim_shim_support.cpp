// fim_shim_support.cpp -- the two host-emulation definitions the reference's FisherInfo_IO objects need
// when they are linked with the library's Neumann() shim (doi_b200/shim/neumann_b200.cu) instead of
// fim_host.cpp.  TEST INFRASTRUCTURE ONLY: oracle/build.sh links it into oracle/_ref/fim_shim, the
// reference's forward main (rte.cu) with Neumann() running on the GPU through librte_b200.
#include <math.h>

#include "rte.h"

thread_local emu_dim3 threadIdx, blockIdx;

// CUDA fast-math intrinsics named by complex_arith.cu's cexp_dev (not called on this path)
extern "C" float __powf(float a, float b) { return powf(a, b); }
extern "C" float __cosf(float a) { return cosf(a); }
extern "C" float __sinf(float a) { return sinf(a); }
