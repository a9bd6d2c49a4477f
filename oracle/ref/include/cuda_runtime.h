/* Host-only stand-in for <cuda_runtime.h>: the few runtime names the reference's host
 * files mention.  Every call reports failure; the harness never takes those paths. */
#pragma once
#include <stddef.h>
#include "vector_types.h"
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorNotSupported = 801 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
static inline const char* cudaGetErrorString(cudaError_t) { return "cuda runtime not available (host emulation)"; }
template <class T> static inline cudaError_t cudaMalloc(T**, size_t) { return cudaErrorNotSupported; }
static inline cudaError_t cudaFree(void*) { return cudaErrorNotSupported; }
static inline cudaError_t cudaMemcpy(void*, const void*, size_t, cudaMemcpyKind) { return cudaErrorNotSupported; }
static inline cudaError_t cudaMemset(void*, int, size_t) { return cudaErrorNotSupported; }
static inline cudaError_t cudaGetLastError() { return cudaSuccess; }
static inline cudaError_t cudaThreadSynchronize() { return cudaSuccess; }
