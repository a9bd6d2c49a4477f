// Exact path integrals along voxel-centre segments (host and device): the walks the pair kernels,
// the kernel precompute and the tangent kernel share.  Host builds (the CPU checks of the walks) read
// the medium through plain loads.
#pragma once
#include <cmath>
#include <cstdlib>
#include <type_traits>

#ifdef __CUDACC__
#define RTE_WALK_FN __host__ __device__ __forceinline__
#else
#define RTE_WALK_FN inline
#endif

template <typename T>
RTE_WALK_FN T rte_walk_load(const T* p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}
RTE_WALK_FN int rte_walk_min(int a, int b) { return a < b ? a : b; }
RTE_WALK_FN int rte_walk_max(int a, int b) { return a > b ? a : b; }
RTE_WALK_FN int rte_walk_abs(int a) { return a < 0 ? -a : a; }
// fused multiply-add in the accumulator's own precision on both sides (a host call of the C fma would
// round a float sum through double)
template <typename T>
RTE_WALK_FN T rte_walk_fma(T a, T b, T c) {
#ifdef __CUDA_ARCH__
  return fma(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
RTE_WALK_FN float rte_walk_fmin(float a, float b) {
#ifdef __CUDA_ARCH__
  return fminf(a, b);
#else
  return std::fmin(a, b);
#endif
}

// Radiological path sum_v mu_t(v) len(v) between the centres of voxels (i,j,k) and (ip,jp,kp).
// Axis crossings are compared as integers: with m_a = max(D_a, 1) and Q = 2 m_x m_y m_z, the
// n-th crossing on axis a is at alpha*Q = (2n+1) * Q / (2 m_a).  Ties step z, then y, then x
// (as mu_int); a tie leaves a zero-length segment, so the order does not change the sum.
template <typename A, typename MU>
RTE_WALK_FN A path_sum(int i, int j, int k, int ip, int jp, int kp, const MU* __restrict__ mu, int nx, int plane,
                       int& Q) {
  const int Dz = rte_walk_abs(ip - i), Dy = rte_walk_abs(jp - j), Dx = rte_walk_abs(kp - k);
  const int mz = rte_walk_max(Dz, 1), my = rte_walk_max(Dy, 1), mx = rte_walk_max(Dx, 1);
  Q = 2 * mx * my * mz;
  if constexpr (std::is_same<A, float>::value) {
    // FP32 sums: the crossing parameters are integers below 2^24 and so exact in FP32, which gives the
    // same segments and the same sum without an integer-to-float conversion per step
    if (Q < (1 << 24)) {
      const float incz = (float)(2 * mx * my), incy = (float)(2 * mx * mz), incx = (float)(2 * my * mz);
      float Az = Dz ? (float)(mx * my) : 3.0e38f, Ay = Dy ? (float)(mx * mz) : 3.0e38f,
            Ax = Dx ? (float)(my * mz) : 3.0e38f;
      const int stz = ip > i ? plane : -plane, sty = jp > j ? nx : -nx, stx = kp > k ? 1 : -1;
      int v = i * plane + j * nx + k;
      float prev = 0.f, acc = 0.f;
      const int steps = Dx + Dy + Dz;
      for (int s = 0; s < steps; ++s) {
        const float m = rte_walk_fmin(Az, rte_walk_fmin(Ay, Ax));
        acc = rte_walk_fma((float)rte_walk_load(mu + v), m - prev, acc);
        prev = m;
        const bool bz = Az == m;
        const bool by = !bz && (Ay == m);
        const bool bx = !bz && !by;
        v += bz ? stz : (by ? sty : stx);
        Az += bz ? incz : 0.f;
        Ay += by ? incy : 0.f;
        Ax += bx ? incx : 0.f;
      }
      acc = rte_walk_fma((float)rte_walk_load(mu + v), (float)Q - prev, acc);
      return acc;
    }
  }
  const int BIG = 0x3fffffff;
  const int incz = 2 * mx * my, incy = 2 * mx * mz, incx = 2 * my * mz;
  int Az = Dz ? mx * my : BIG, Ay = Dy ? mx * mz : BIG, Ax = Dx ? my * mz : BIG;
  const int stz = ip > i ? plane : -plane, sty = jp > j ? nx : -nx, stx = kp > k ? 1 : -1;
  int v = i * plane + j * nx + k;
  int prev = 0;
  A acc = A(0);
  const int steps = Dx + Dy + Dz;
  for (int s = 0; s < steps; ++s) {
    const int m = rte_walk_min(Az, rte_walk_min(Ay, Ax));
    const A muv = (A)rte_walk_load(mu + v);
    acc = rte_walk_fma(muv, (A)(m - prev), acc);
    prev = m;
    const bool bz = Az == m;
    const bool by = !bz && (Ay == m);
    const bool bx = !bz && !by;
    v += bz ? stz : (by ? sty : stx);
    Az += bz ? incz : 0;
    Ay += by ? incy : 0;
    Ax += bx ? incx : 0;
  }
  acc = rte_walk_fma((A)rte_walk_load(mu + v), (A)(Q - prev), acc);
  return acc;
}

// path_sum over a field that is zero outside the voxel box [lo, hi] (x, y, z order): the walk starts at
// the last crossing at or before the path enters the box and stops where it leaves, so the segments it
// skips are exactly the zero terms of the whole walk and the sum is the same, bit for bit (the entry and
// exit parameters are found per axis from the crossing counts, crossing n of axis a lying at
// (2n + 1) h_a).  0 when the path never has all three coordinates inside the box.
template <typename A, typename MU>
RTE_WALK_FN A path_sum_box(int i, int j, int k, int ip, int jp, int kp, const MU* __restrict__ mu, int nx,
                           int plane, const int* lo, const int* hi, int& Q) {
  const int D[3] = {rte_walk_abs(ip - i), rte_walk_abs(jp - j), rte_walk_abs(kp - k)};  // z, y, x
  const int st[3] = {i, j, k};
  const int sg[3] = {ip > i ? 1 : -1, jp > j ? 1 : -1, kp > k ? 1 : -1};
  const int blo[3] = {lo[2], lo[1], lo[0]}, bhi[3] = {hi[2], hi[1], hi[0]};
  const int mz = rte_walk_max(D[0], 1), my = rte_walk_max(D[1], 1), mx = rte_walk_max(D[2], 1);
  Q = 2 * mx * my * mz;
  const int h[3] = {mx * my, mx * mz, my * mz};
  const int BIG = 0x3fffffff;
  int tin = 0, tout = Q;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    int enter = 0;  // crossings of this axis before its coordinate is inside [lo, hi]
    if (st[q] < blo[q]) enter = sg[q] > 0 && D[q] > 0 ? blo[q] - st[q] : BIG;
    else if (st[q] > bhi[q]) enter = sg[q] < 0 && D[q] > 0 ? st[q] - bhi[q] : BIG;
    if (enter > D[q]) return A(0);
    if (enter > 0) tin = rte_walk_max(tin, (2 * enter - 1) * h[q]);
    const int ex = sg[q] > 0 ? bhi[q] - st[q] + 1 : st[q] - blo[q] + 1;  // crossings until outside again
    if (D[q] > 0 && ex <= D[q]) tout = rte_walk_min(tout, (2 * ex - 1) * h[q]);
  }
  if (tin >= tout) return A(0);
  int n[3], Ax[3];  // crossings at or before tin, and each axis' next crossing
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    n[q] = rte_walk_min(D[q], (tin + h[q]) / (2 * h[q]));
    Ax[q] = n[q] < D[q] ? (2 * n[q] + 1) * h[q] : BIG;
  }
  int az = Ax[0], ay = Ax[1], ax = Ax[2];
  const int incz = 2 * h[0], incy = 2 * h[1], incx = 2 * h[2];
  const int stz = sg[0] * plane, sty = sg[1] * nx, stx = sg[2];
  int v = (i + sg[0] * n[0]) * plane + (j + sg[1] * n[1]) * nx + (k + sg[2] * n[2]);
  int prev = tin;
  A acc = A(0);
  for (;;) {
    const int m = rte_walk_min(az, rte_walk_min(ay, ax));
    if (m >= tout) {
      acc = rte_walk_fma((A)rte_walk_load(mu + v), (A)(tout - prev), acc);
      break;
    }
    acc = rte_walk_fma((A)rte_walk_load(mu + v), (A)(m - prev), acc);
    prev = m;
    const bool bz = az == m;
    const bool by = !bz && (ay == m);
    const bool bx = !bz && !by;
    v += bz ? stz : (by ? sty : stx);
    az += bz ? incz : 0;
    ay += by ? incy : 0;
    ax += bx ? incx : 0;
  }
  return acc;
}
