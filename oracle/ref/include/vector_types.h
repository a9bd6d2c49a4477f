/* Host-only stand-in for CUDA's vector_types.h (only double2 is needed). */
#pragma once
typedef struct __attribute__((aligned(16))) { double x, y; } double2;
