/* fim_emu.h -- forced-include header that lets the reference's FisherInfo_IO CUDA sources
 * compile as host C++ (g++) so its kernels can run on the CPU as the oracle's pin.
 * Test infrastructure only.  Kernel launches are replaced by oracle/ref/fim_host.cpp, which
 * sets threadIdx/blockIdx and calls each kernel body once per emulated thread. */
#pragma once
#include <math.h>
#include <stdlib.h>
#include <string.h>
#define __host__
#define __device__
#define __global__
#define __constant__
#define __shared__
#define __align__(x) __attribute__((aligned(x)))
struct emu_dim3 { unsigned int x, y, z; };
extern thread_local emu_dim3 threadIdx, blockIdx;
static inline void __syncthreads() {}
/* CUDA's __int2double_rn takes an int: a double argument is truncated on the way in, as on
 * the device (this is what turns g = 0.8 into 0 in prop_scat_dev). */
static inline double __int2double_rn(int x) { return (double)x; }
static inline float __int2float_ru(int x) { return (float)x; }
