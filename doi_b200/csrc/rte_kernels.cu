// rte_kernels.cu -- sm_100a kernels of the Neumann-series RTE term W <- D A W.
//
// The attenuation operator A of the reference (FisherInfo_IO/src/kernels.cu:151-418,
// compute_diagonal_abs + compute_propabs + scale_dist_dev, and prop_scat_dev for D) is
// computed here in a REAL spherical-harmonic basis (the host converts at the boundary):
//
//   out[r,c] = sum_{r' != r, |r-r'| < propThresh} R_c(w) k(r,r') sum_c' R_c'(w) W[r',c']
//            + (dV/cm) sum_c' Dself_cc'(mu_t(r)) W[r,c'],
//   w = (r - r')/|r - r'|,  k = exp(-tau(r,r')) dV / (cm |r - r'|^2),
//
// then D multiplies coefficient (l,m) by scat[l] * mu_s(r).  One CUDA thread owns one
// destination voxel and streams all source voxels through shared memory (the warp
// reads the same source at the same time, so source data is a shared-memory
// broadcast).  The source range is split over blockIdx.y (split-K); the epilogue
// kernel adds the partial sums in a fixed order, so results are deterministic.
//
// Path integrals follow mu_int (FisherInfo_IO/src/kernels.cu:50-148): a Siddon walk
// between voxel centres whose axis crossings are ordered here with exact integer
// arithmetic (crossing n on an axis with |delta| = D sits at alpha = (2n+1)/(2D)).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <string.h>

#include <algorithm>

#include <type_traits>

#include "rte_internal.h"

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two FP32 FMAs per instruction.
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
  f2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

struct ScatTab {
  double v[RTE_MAX_L + 1];
};

__constant__ ShTables c_sh;
__constant__ float c_shAf[64];
__constant__ float c_shBf[64];
__constant__ float c_shQ0f[RTE_MAX_L + 1];

cudaError_t rte_upload_sh_tables(const ShTables& t) {
  float af[64], bf[64], qf[RTE_MAX_L + 1];
  for (int i = 0; i < 64; i++) {
    af[i] = (float)t.A[i];
    bf[i] = (float)t.B[i];
  }
  for (int i = 0; i <= RTE_MAX_L; i++) qf[i] = (float)t.Q0[i];
  cudaError_t e = cudaMemcpyToSymbol(c_sh, &t, sizeof(ShTables));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_shAf, af, sizeof af);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_shBf, bf, sizeof bf);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_shQ0f, qf, sizeof qf);
  return e;
}

template <typename T> __device__ __forceinline__ T shA(int i);
template <typename T> __device__ __forceinline__ T shB(int i);
template <typename T> __device__ __forceinline__ T shQ0(int i);
template <> __device__ __forceinline__ double shA<double>(int i) { return c_sh.A[i]; }
template <> __device__ __forceinline__ double shB<double>(int i) { return c_sh.B[i]; }
template <> __device__ __forceinline__ double shQ0<double>(int i) { return c_sh.Q0[i]; }
template <> __device__ __forceinline__ float shA<float>(int i) { return c_shAf[i]; }
template <> __device__ __forceinline__ float shB<float>(int i) { return c_shBf[i]; }
template <> __device__ __forceinline__ float shQ0<float>(int i) { return c_shQ0f[i]; }

// Compile-time copies of the SH recurrence coefficients (the same formulas as the host tables in
// rte_host.cpp), so the unrolled FP32 recurrence multiplies by immediates and the l = m+1 steps
// carry no B term.
struct ShConstTab {
  double A[64], B[64], Q0[RTE_MAX_L + 1];
};
constexpr double c_sqrt(double x) {
  double r = x > 1.0 ? x : 1.0;
  for (int i = 0; i < 80; ++i) r = 0.5 * (r + x / r);
  return r;
}
constexpr double c_knorm(int l, int m) {
  double f = 1.0;
  for (int i = l - m + 1; i <= l + m; ++i) f *= (double)i;
  const double k = c_sqrt((2.0 * l + 1.0) / (4.0 * 3.14159265358979323846) / f);
  return m > 0 ? k * c_sqrt(2.0) : k;
}
constexpr ShConstTab make_sh_const() {
  ShConstTab t{};
  for (int m = 0; m <= RTE_MAX_L; ++m) {
    double dfact = 1.0;
    for (int i = 2 * m - 1; i > 0; i -= 2) dfact *= (double)i;
    t.Q0[m] = c_knorm(m, m) * ((m & 1) ? -1.0 : 1.0) * dfact;
    for (int l = m + 1; l <= RTE_MAX_L; ++l) {
      const int id = l * (l + 1) / 2 + m;
      t.A[id] = c_knorm(l, m) * (2.0 * l - 1.0) / ((double)(l - m) * c_knorm(l - 1, m));
      t.B[id] = (l - 2 >= m) ? c_knorm(l, m) * (double)(l + m - 1) / ((double)(l - m) * c_knorm(l - 2, m)) : 0.0;
    }
  }
  return t;
}
__device__ constexpr ShConstTab kShConst = make_sh_const();

// Real orthonormal SH R_lm at the unit direction (x, y, z), index l*l + l + m.
// R_l0 = q_l^0(z), R_l,+m = q_l^m(z) Re((x+iy)^m), R_l,-m = q_l^m(z) Im((x+iy)^m), with the
// normalised associated-Legendre polynomials q (Condon-Shortley phase included) from the
// upward recurrence in l.  No trigonometric calls.  FP64 reads the uploaded tables; FP32 uses
// the compile-time copies.
template <int L, typename T>
__device__ __forceinline__ void sh_eval(T x, T y, T z, T* R) {
  constexpr bool F32 = std::is_same<T, float>::value;
  T cmv = T(1), smv = T(0);
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m == 1) {
      cmv = x;
      smv = y;
    } else if (m > 1) {
      T c2 = cmv * x - smv * y;
      T s2 = cmv * y + smv * x;
      cmv = c2;
      smv = s2;
    }
    T q2 = T(0), q1 = F32 ? (T)kShConst.Q0[m] : shQ0<T>(m);
    if (m == 0) {
      R[0] = q1;
    } else {
      R[m * m + 2 * m] = q1 * cmv;
      R[m * m] = q1 * smv;
    }
#pragma unroll
    for (int l = m + 1; l <= L; ++l) {
      const int id = l * (l + 1) / 2 + m;
      const T A = F32 ? (T)kShConst.A[id] : shA<T>(id);
      T q;
      if (l == m + 1) {
        q = (A * z) * q1;
      } else {
        const T B = F32 ? (T)kShConst.B[id] : shB<T>(id);
        q = (A * z) * q1 - B * q2;
      }
      q2 = q1;
      q1 = q;
      if (m == 0) {
        R[l * l + l] = q;
      } else {
        R[l * l + l + m] = q * cmv;
        R[l * l + l - m] = q * smv;
      }
    }
  }
}

// Monic form of the same recurrence for the mixed pair kernel.  With q_l^m = s_lm u_l^m, s_mm = Q0[m]
// and s_lm = A_lm s_{l-1,m}, the polynomials u satisfy u_l = z u_{l-1} - beta_lm u_{l-2} (beta_lm =
// B_lm s_{l-2,m} / s_lm), so R_c = N_c U_c with U_{l,+-m} = u_l^m Re/Im((x+iy)^m) and N_c = s_lm.
// The kernel carries U instead of R: the factors N_c are applied once per source row (the FP32 copy
// of W holds N_c W_c) and once per destination (the partial sums), not per pair, and a recurrence
// step costs two operations instead of three.
struct MonicTab {
  double beta[64];  // index l*(l+1)/2 + m
  double N[64];     // index l*l + l + m
};
constexpr MonicTab make_monic() {
  MonicTab t{};
  const ShConstTab q = make_sh_const();
  for (int m = 0; m <= RTE_MAX_L; ++m) {
    double s[RTE_MAX_L + 1] = {};
    s[m] = q.Q0[m];
    for (int l = m + 1; l <= RTE_MAX_L; ++l) s[l] = q.A[l * (l + 1) / 2 + m] * s[l - 1];
    for (int l = m; l <= RTE_MAX_L; ++l) {
      if (l >= m + 2) t.beta[l * (l + 1) / 2 + m] = q.B[l * (l + 1) / 2 + m] * s[l - 2] / s[l];
      t.N[l * l + l + m] = s[l];
      t.N[l * l + l - m] = s[l];
    }
  }
  return t;
}
__device__ constexpr MonicTab kMonic = make_monic();

// The monic recurrence, each coefficient handed to emit(index, value) as it is made (the index is a
// compile-time constant once the loops unroll).
template <int L, typename T, typename Emit>
__device__ __forceinline__ void sh_monic_recurrence(T x, T y, T z, Emit emit) {
  T cmv = T(1), smv = T(0);
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m == 1) {
      cmv = x;
      smv = y;
    } else if (m > 1) {
      const T c2 = cmv * x - smv * y;
      const T s2 = cmv * y + smv * x;
      cmv = c2;
      smv = s2;
    }
    T c1 = cmv, s1 = smv, c0 = T(0), s0 = T(0);
    if (m == 0) {
      emit(0, T(1));
    } else {
      emit(m * m + 2 * m, cmv);
      emit(m * m, smv);
    }
#pragma unroll
    for (int l = m + 1; l <= L; ++l) {
      T cn, sn = T(0);
      if (l == m + 1) {
        cn = m == 0 ? z : z * c1;
        if (m > 0) sn = z * s1;
      } else {
        const T b = (T)kMonic.beta[l * (l + 1) / 2 + m];
        cn = fma(z, c1, -b * c0);
        if (m > 0) sn = fma(z, s1, -b * s0);
      }
      c0 = c1;
      c1 = cn;
      s0 = s1;
      s1 = sn;
      if (m == 0) {
        emit(l * l + l, cn);
      } else {
        emit(l * l + l + m, cn);
        emit(l * l + l - m, sn);
      }
    }
  }
}

template <int L, typename T>
__device__ __forceinline__ void sh_eval_monic(T x, T y, T z, T* U) {
  sh_monic_recurrence<L, T>(x, y, z, [&](int c, T v) { U[c] = v; });
}

// Direction snapped to the reference's 100x100 SH table cell (FisherInfo_IO/src/defines.h:53-56
// and kernels.cu:326-333: theta = acos(dz/dist), phi = atan2(dy,dx) NOT wrapped to [0,2pi), so a
// negative phi index reads the previous theta row of the flat table).
__device__ __forceinline__ void table_direction(double ddx, double ddy, double ddz, double dist, double& ux,
                                                double& uy, double& uz) {
  double theta = acos(ddz / dist);
  double phi = atan2(ddy, ddx);
  int ti = (int)rintf((float)((100 - 1) * (theta) / (M_PI)));
  int pj = (int)rintf((float)((100 - 1) * (phi) / (2 * M_PI)));
  int off = ti * 100 + pj;
  if (off < 0) off = 0;
  int tq = off / 100, pq = off - tq * 100;
  double th = (tq * M_PI) / (100 - 1);
  double ph = (pq * 2.0 * M_PI) / (100 - 1);
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp, &cp);
  ux = st * cp;
  uy = st * sp;
  uz = ct;
}

#include "rte_walk.cuh"

// ---------------------------------------------------------------------------------------------
// Plain FP64 method: every pair recomputed in FP64 (path integral, SH, projections).  CPLX: one
// complex right-hand side stored as (real, imaginary) rows per voxel, and the pair kernel carries the
// modulation phase exp(-i kappa |r - r'|) (complex mu_t = mu_t + i kappa, uniform imaginary part).
// STORED: the pair kernel exp(-tau) dV/(cm r^2) is read from the FP64 matrix Kmat64[source slot]
// [destination slot] instead of walking the path; sources are then visited in slot order, so the
// warp's 32 destinations read one contiguous 256-byte run of K per source.
template <int LA, bool TABLE, bool CPLX, bool STORED = false>
__global__ void __launch_bounds__(RTE_PAIR_THREADS) k_pair_fp64(PairArgs a) {
  constexpr int C = (LA + 1) * (LA + 1);
  constexpr int NP = CPLX ? 2 : 1;        // rows per voxel
  constexpr int TS = RTE_PAIR_TS / NP;    // sources per shared-memory tile
  __shared__ double sW[TS * NP * C];
  __shared__ int sxyz[STORED ? TS : 1][3];  // source coordinates (slot order)
  const int tid = threadIdx.x;
  const int slot = blockIdx.x * RTE_PAIR_THREADS + tid;
  const bool act = slot < a.N;
  const int r = act ? a.perm[slot] : 0;
  const int plane = a.nx * a.ny;
  const int i = r / plane, j = (r / a.nx) % a.ny, k = r % a.nx;
  const int vs = NP * a.Cfull;
  double acc[NP][C];
#pragma unroll
  for (int p = 0; p < NP; ++p)
#pragma unroll
    for (int c = 0; c < C; ++c) acc[p][c] = 0.0;
  const int sb = blockIdx.y * a.chunk;
  const int se = min(a.N, sb + a.chunk);
  for (int s0 = sb; s0 < se; s0 += TS) {
    const int ns = min(TS, se - s0);
    __syncthreads();
    for (int q = tid; q < ns * NP * C; q += RTE_PAIR_THREADS) {
      const int sv = q / (NP * C), e = q - sv * NP * C, p = e / C, c = e - p * C;
      const int src = STORED ? a.perm[s0 + sv] : s0 + sv;
      sW[q] = a.Win[(size_t)src * vs + (size_t)p * a.Cfull + c];
    }
    if (STORED && tid < ns) {
      const int v = a.perm[s0 + tid];
      sxyz[tid][0] = v % a.nx;
      sxyz[tid][1] = (v / a.nx) % a.ny;
      sxyz[tid][2] = v / plane;
    }
    __syncthreads();
    if (!act) continue;
    if constexpr (STORED) {
      const double* Kcol = a.Kmat64 + (size_t)s0 * a.Kld + slot;
      double knext = __ldg(Kcol);
      for (int sv = 0; sv < ns; ++sv) {
        const double kk = knext;
        if (sv + 1 < ns) knext = __ldg(Kcol + (size_t)(sv + 1) * a.Kld);
        if (kk == 0.0) continue;  // the diagonal and pairs beyond the coupling distance
        const double ddx = (double)(k - sxyz[sv][0]) * a.dx, ddy = (double)(j - sxyz[sv][1]) * a.dy,
                     ddz = (double)(i - sxyz[sv][2]) * a.dz;
        const double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
        double ux, uy, uz;
        if (TABLE) {
          // A^T: snap(source - destination), negated in integers so that a zero component stays +0.0 (the
          // table's unwrapped phi index depends on atan2's sign of zero) -- the forward kernel's exact bits
          const int sg = a.transpose ? -1 : 1;
          table_direction((double)(sg * (k - sxyz[sv][0])) * a.dx, (double)(sg * (j - sxyz[sv][1])) * a.dy,
                          (double)(sg * (i - sxyz[sv][2])) * a.dz, dist, ux, uy, uz);
        } else {
          const double inv = 1.0 / dist;
          ux = ddx * inv;
          uy = ddy * inv;
          uz = ddz * inv;
        }
        double R[C];
        sh_eval<LA, double>(ux, uy, uz, R);
        double S[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          S[p] = 0.0;
#pragma unroll
          for (int c = 0; c < C; ++c) S[p] = fma(R[c], sW[(sv * NP + p) * C + c], S[p]);
        }
        if (CPLX) {
          double sn, cs;
          sincos(a.kappa * dist, &sn, &cs);
          const double t0 = kk * (cs * S[0] + sn * S[NP - 1]), t1 = kk * (cs * S[NP - 1] - sn * S[0]);
#pragma unroll
          for (int c = 0; c < C; ++c) {
            acc[0][c] = fma(R[c], t0, acc[0][c]);
            acc[NP - 1][c] = fma(R[c], t1, acc[NP - 1][c]);
          }
        } else {
          const double t = kk * S[0];
#pragma unroll
          for (int c = 0; c < C; ++c) acc[0][c] = fma(R[c], t, acc[0][c]);
        }
      }
      continue;
    }
    int kp = s0 % a.nx, jp = (s0 / a.nx) % a.ny, ip = s0 / plane;
    for (int sv = 0; sv < ns; ++sv) {
      const int rp = s0 + sv;
      if (rp != r) {
        const double ddx = (double)(k - kp) * a.dx, ddy = (double)(j - jp) * a.dy, ddz = (double)(i - ip) * a.dz;
        const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
        const double dist = sqrt(d2);
        if (dist < a.prop_thresh) {
          double ux, uy, uz;
          if (TABLE) {
            // A^T: snap(source - destination), negated in integers (a zero component stays +0.0)
            const int sg = a.transpose ? -1 : 1;
            table_direction((double)(sg * (k - kp)) * a.dx, (double)(sg * (j - jp)) * a.dy,
                            (double)(sg * (i - ip)) * a.dz, dist, ux, uy, uz);
          } else {
            const double inv = 1.0 / dist;
            ux = ddx * inv;
            uy = ddy * inv;
            uz = ddz * inv;
          }
          double R[C];
          sh_eval<LA, double>(ux, uy, uz, R);
          double S[NP];
#pragma unroll
          for (int p = 0; p < NP; ++p) {
            S[p] = 0.0;
#pragma unroll
            for (int c = 0; c < C; ++c) S[p] = fma(R[c], sW[(sv * NP + p) * C + c], S[p]);
          }
          int Q;
          const double ps = path_sum<double, double>(i, j, k, ip, jp, kp, a.mut, a.nx, plane, Q);
          const double tau = ps * dist / (double)Q;
          const double kk = exp(-tau) * a.kscale / d2;
          if (CPLX) {  // kk exp(-i kappa dist) (S0 + i S1)
            double sn, cs;
            sincos(a.kappa * dist, &sn, &cs);
            const double t0 = kk * (cs * S[0] + sn * S[NP - 1]), t1 = kk * (cs * S[NP - 1] - sn * S[0]);
#pragma unroll
            for (int c = 0; c < C; ++c) {
              acc[0][c] = fma(R[c], t0, acc[0][c]);
              acc[NP - 1][c] = fma(R[c], t1, acc[NP - 1][c]);
            }
          } else {
            const double t = kk * S[0];
#pragma unroll
            for (int c = 0; c < C; ++c) acc[0][c] = fma(R[c], t, acc[0][c]);
          }
        }
      }
      if (++kp == a.nx) {
        kp = 0;
        if (++jp == a.ny) {
          jp = 0;
          ++ip;
        }
      }
    }
  }
  if (act) {
    double* o = a.part + ((size_t)blockIdx.y * a.N + r) * vs;
#pragma unroll
    for (int p = 0; p < NP; ++p)
#pragma unroll
      for (int c = 0; c < C; ++c) o[(size_t)p * a.Cfull + c] = acc[p][c];
  }
}

// ---------------------------------------------------------------------------------------------
// Tangent pair operator: the derivative of the off-diagonal attenuation operator along one
// parameter direction dmu_t,
//   out[r] = sum_{r' != r} -dtau(r, r') k(r, r') R(w) (R(w) . W[r']),  dtau = path integral of dmu_t,
// the same pair walk as the forward operator over the perturbation field.  Pairs whose segment misses
// the support box of dmu_t are skipped before the walk, pairs with dtau = 0 after it, so a localised
// perturbation costs far less than a forward pass.  k from the stored FP32 kernel or recomputed.
__device__ __forceinline__ bool segment_hits_box(float ax, float ay, float az, float bx, float by, float bz,
                                                 const int* lo, const int* hi) {
  const float a3[3] = {ax, ay, az}, b3[3] = {bx, by, bz};
  float t0 = 0.f, t1 = 1.f;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const float l = (float)lo[d] - 0.5001f, h = (float)hi[d] + 0.5001f, dd = b3[d] - a3[d];
    if (dd == 0.f) {
      if (a3[d] < l || a3[d] > h) return false;
    } else {
      float ta = (l - a3[d]) / dd, tb = (h - a3[d]) / dd;
      if (ta > tb) {
        const float x = ta;
        ta = tb;
        tb = x;
      }
      t0 = fmaxf(t0, ta);
      t1 = fminf(t1, tb);
      if (t0 > t1) return false;
    }
  }
  return true;
}

// Real SH of a direction for the FP32 (or FP64) pair arithmetic of type T: at L >= 7 the recurrence runs
// in FP64 (the monic form of the mixed pair kernels, normalised as each value is rounded to T).
template <int LA, typename T>
__device__ __forceinline__ void sh_eval_prec(T x, T y, T z, T* R) {
  if constexpr (LA < 7 || std::is_same<T, double>::value) {
    sh_eval<LA, T>(x, y, z, R);
  } else {  // the monic recurrence in FP64, each value normalised and rounded as it is made
    sh_monic_recurrence<LA, double>((double)x, (double)y, (double)z,
                                    [&](int c, double v) { R[c] = (T)(v * kMonic.N[c]); });
  }
}

template <int LA, bool TABLE, typename T>
__global__ void __launch_bounds__(RTE_PAIR_THREADS) k_pair_tangent(PairArgs a) {
  constexpr int C = (LA + 1) * (LA + 1);
  __shared__ T sW[RTE_PAIR_TS * C];
  const int tid = threadIdx.x;
  const int slot = blockIdx.x * RTE_PAIR_THREADS + tid;
  const bool act = slot < a.N;
  const int r = act ? a.perm[slot] : 0;
  const int plane = a.nx * a.ny;
  const int i = r / plane, j = (r / a.nx) % a.ny, k = r % a.nx;
  T acc[C];
#pragma unroll
  for (int c = 0; c < C; ++c) acc[c] = T(0);
  const int sb = blockIdx.y * a.chunk;
  const int se = min(a.N, sb + a.chunk);
  const T thr = (T)a.prop_thresh;
  for (int s0 = sb; s0 < se; s0 += RTE_PAIR_TS) {
    const int ns = min(RTE_PAIR_TS, se - s0);
    __syncthreads();
    for (int q = tid; q < ns * C; q += RTE_PAIR_THREADS) {
      const int sv = q / C, c = q - sv * C;
      sW[q] = (T)a.Win[(size_t)(s0 + sv) * a.Cfull + c];
    }
    __syncthreads();
    if (!act) continue;
    int kp = s0 % a.nx, jp = (s0 / a.nx) % a.ny, ip = s0 / plane;
    for (int sv = 0; sv < ns; ++sv) {
      const int rp = s0 + sv;
      if (rp != r && segment_hits_box((float)k, (float)j, (float)i, (float)kp, (float)jp, (float)ip, a.box_lo, a.box_hi)) {
        const T ddx = (T)(k - kp) * (T)a.dx, ddy = (T)(j - jp) * (T)a.dy, ddz = (T)(i - ip) * (T)a.dz;
        const T d2 = ddx * ddx + ddy * ddy + ddz * ddz;
        const T dist = sqrt(d2);
        if (dist < thr) {
          int Q;
          const T dps = path_sum_box<T, double>(i, j, k, ip, jp, kp, a.dmut, a.nx, plane, a.box_lo, a.box_hi, Q);
          if (dps != T(0)) {
            const T dtau = dps * dist / (T)Q;
            T kk;
            if (a.Kmat64) {
              kk = (T)__ldg(a.Kmat64 + (size_t)a.islot[rp] * a.Kld + slot);
            } else if (a.Kmat) {
              kk = (T)__ldg(a.Kmat + kmat_index(a.islot[rp], slot, a.Kld));
            } else {
              int Q2;
              const T ps = path_sum<T, double>(i, j, k, ip, jp, kp, a.mut, a.nx, plane, Q2);
              kk = exp(-ps * dist / (T)Q2) * (T)a.kscale / d2;
            }
            T R[C];
            if (TABLE) {
              double ux, uy, uz;
              table_direction((double)ddx, (double)ddy, (double)ddz, (double)dist, ux, uy, uz);
              sh_eval_prec<LA, T>((T)ux, (T)uy, (T)uz, R);
            } else {
              const T inv = T(1) / dist;
              sh_eval_prec<LA, T>(ddx * inv, ddy * inv, ddz * inv, R);
            }
            T S = T(0);
#pragma unroll
            for (int c = 0; c < C; ++c) S = fma(R[c], sW[sv * C + c], S);
            const T t = -dtau * kk * S;
#pragma unroll
            for (int c = 0; c < C; ++c) acc[c] = fma(R[c], t, acc[c]);
          }
        }
      }
      if (++kp == a.nx) {
        kp = 0;
        if (++jp == a.ny) {
          jp = 0;
          ++ip;
        }
      }
    }
  }
  if (act) {
    double* o = a.part + ((size_t)blockIdx.y * a.N + r) * a.Cfull;
#pragma unroll
    for (int c = 0; c < C; ++c) o[c] = (double)acc[c];
  }
}

// q (rows qstride apart) = scat_l (mu_s T + dmu_s out): the tangent right-hand side D dA S + dD A S
__global__ void k_tangent_rhs(double* q, int qstride, const double* T, const double* out, const double* mus,
                              const double* dmus, ScatTab sc, int N, int L) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int C = (L + 1) * (L + 1);
  if (t >= (long long)N * C) return;
  const int r = (int)(t / C), c = (int)(t % C);
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  q[(size_t)r * qstride + c] = sc.v[l] * (mus[r] * T[t] + dmus[r] * out[t]);
}

__global__ void k_scatter_add(double* dst, int dstride, const int* idx, const double* vals, int n, int C) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * C) return;
  dst[(size_t)idx[t / C] * dstride + t % C] += vals[t];
}

// dst [N][C] = a (rows astride apart) + b [N][C]
__global__ void k_strided_add(double* dst, const double* a, int astride, const double* b, int N, int C) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * C) return;
  const int r = (int)(t / C), c = (int)(t % C);
  dst[t] = a[(size_t)r * astride + c] + b[t];
}

// ---------------------------------------------------------------------------------------------
// Mixed precision: path integrals, SH and projections in FP32 (SH in FP64 for l >= 7).  NB right-
// hand sides that share the medium are propagated together: the direction, its SH and the pair
// kernel are computed once per pair and used NB times.  Sources are visited in slot order (the
// same spatially compact order as the destinations).  The FP32 source coefficients are kept in
// slot order with rows of CP floats, so a 64-source tile (and its coordinates) is one contiguous
// block: one thread issues two TMA bulk copies (cp.async.bulk, completion on an mbarrier) per tile
// into a double buffer, overlapping the next tile's copy with this tile's arithmetic.  Sums: FP32
// over one tile in registers (projections split over four accumulators), FP32 across tiles in
// shared memory, FP64 across the split-K chunks in the epilogue.  STORED reads the precomputed
// pair kernel K[source slot][destination slot] (FP32); otherwise the path is walked in FP32.
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// bounded wait on an mbarrier phase; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// shared memory: [2][TS] float4 | [2][TS][cpad] float | [NB*C][T] float | 2 mbarriers (TS sources per tile)
struct MixedLayout {
  size_t off_w, off_acc, off_bar, bytes;
  __host__ __device__ MixedLayout(int cpad, int nbc, int ts = RTE_PAIR_TS) {
    off_w = sizeof(float4) * 2 * ts;
    off_acc = off_w + sizeof(float) * 2 * ts * (size_t)cpad;
    off_bar = (off_acc + sizeof(float) * (size_t)nbc * RTE_PAIR_THREADS + 15) / 16 * 16;
    bytes = off_bar + 2 * sizeof(uint64_t);
  }
};

// CPLX (NB = 2): the two right-hand sides are the real and imaginary parts of one complex one and the
// pair kernel carries the modulation phase exp(-i kappa |r - r'|).  L = 7 with one right-hand side runs
// under a three-CTA register bound (168 registers, k_pair_mixed_3): 33^3 launch 38.3 -> 33.9 ms (the
// same bound made L = 6 slower, so it applies to L = 7 alone).
template <int LA, bool TABLE, bool STORED, int NB, bool CPLX>
__device__ __forceinline__ void pair_mixed_body(const PairArgs& a) {
  static_assert(!CPLX || NB == 2, "a complex right-hand side is a (real, imaginary) pair");
  // wide rows (NB * C >= 128: 4 RHS at L = 5, 2 RHS at L = 7): 32-source tiles, so that two CTAs (their
  // register limit) fit the shared memory
  constexpr int C = (LA + 1) * (LA + 1), TS = NB * C >= 128 ? 32 : RTE_PAIR_TS, T = RTE_PAIR_THREADS;
  const int CP = a.cpad;  // FP32 source row: nb * Cfull floats, padded to a multiple of 4
  const MixedLayout Sh(CP, NB * C, TS);
  typedef typename std::conditional<(LA >= 7), double, float>::type ShT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sP = reinterpret_cast<float4*>(smem_raw);
  float* sW = reinterpret_cast<float*>(smem_raw + Sh.off_w);
  float* sAcc = reinterpret_cast<float*>(smem_raw + Sh.off_acc);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + Sh.off_bar);
  const int tid = threadIdx.x;
  const int slot = blockIdx.x * T + tid;
  const bool act = slot < a.N;
  const float4 me = a.slot_xyz[act ? slot : 0];
  const int r = __float_as_int(me.w);
  const int plane = a.nx * a.ny;
  const int i = (int)me.z, j = (int)me.y, k = (int)me.x;
  const float dxf = (float)a.dx, dyf = (float)a.dy, dzf = (float)a.dz;
  const float kscalef = (float)a.kscale;
  const float thr = (float)a.prop_thresh;
#pragma unroll
  for (int q = 0; q < NB * C; ++q) sAcc[q * T + tid] = 0.f;
  const int sb = blockIdx.y * a.chunk;
  const int se = min(a.N, sb + a.chunk);
  const int ntile = (se - sb + TS - 1) / TS;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int t) {  // tile t -> buffer t & 1 (one thread)
    const int s0 = sb + t * TS;
    const int ns = min(TS, se - s0);
    const int b = t & 1;
    const uint32_t bw = (uint32_t)(ns * CP * sizeof(float)), bp = (uint32_t)(ns * sizeof(float4));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[b], bw + bp);
    bulk_g2s(sW + b * TS * CP, a.Winf + (size_t)s0 * CP, bw, &bar[b]);
    bulk_g2s(sP + b * TS, a.slot_xyz + s0, bp, &bar[b]);
  };
  if (tid == 0 && ntile > 0) issue(0);
  constexpr int C2 = (C + 1) / 2;  // coefficient pairs (packed f32x2 arithmetic)
  const int CS = a.cstride;        // FP32 row stride of one right-hand side (even)
  f2_t acc[NB][C2];
  for (int t = 0; t < ntile; ++t) {
    if (tid == 0 && t + 1 < ntile) issue(t + 1);
    const bool ok = mbar_wait(&bar[t & 1], (uint32_t)((t >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(a.err, 1);
      return;
    }
    const int s0 = sb + t * TS;
    const int ns = min(TS, se - s0);
    const float4* P = sP + (t & 1) * TS;
    const float* Wt = sW + (t & 1) * TS * CP;
    if (act) {
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < C2; ++c) acc[b][c] = 0ull;
      const float* Kcol = STORED ? a.Kmat + kmat_index(s0, slot, a.Kld) : nullptr;  // next source: +RTE_KBLK
      float k0 = 0.f, k1 = 0.f;
      if (STORED) {
        k0 = __ldg(Kcol);
        if (ns > 1) k1 = __ldg(Kcol + RTE_KBLK);
      }
      // stored kernel with exact SH: no per-pair branch (the diagonal and pairs beyond the coupling
      // distance carry k = 0), so two sources' SH recurrences can interleave
      constexpr bool FLAT = STORED && !TABLE;
      constexpr int UNR = FLAT ? 3 : 1;
#pragma unroll UNR
      for (int sv = 0; sv < ns; ++sv) {
        float kk = 0.f;
        if (STORED) {
          kk = k0;
          k0 = k1;
          if (sv + 2 < ns) k1 = __ldg(Kcol + (size_t)(sv + 2) * RTE_KBLK);
        }
        const float4 q = P[sv];
        const float ddx = (me.x - q.x) * dxf, ddy = (me.y - q.y) * dyf, ddz = (me.z - q.z) * dzf;
        const float d2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
        bool live;
        float dist = 0.f;
        if (STORED) {
          live = FLAT || kk != 0.f;
        } else {
          dist = sqrtf(d2);
          live = d2 > 0.f && dist < thr;
        }
        if (live) {
          ShT R[C];
          if (TABLE) {
            // A^T: snap(source - destination), negated in integers (a zero component stays +0.0)
            const int sg = a.transpose ? -1 : 1;
            const double ex = (double)(sg * (k - (int)q.x)) * a.dx, ey = (double)(sg * (j - (int)q.y)) * a.dy,
                         ez = (double)(sg * (i - (int)q.z)) * a.dz;
            double ux, uy, uz;
            table_direction(ex, ey, ez, sqrt(ex * ex + ey * ey + ez * ez), ux, uy, uz);
            sh_eval_monic<LA, ShT>((ShT)ux, (ShT)uy, (ShT)uz, R);  // A^T: snap(source - destination)
          } else {
            const float inv = FLAT ? (d2 > 0.f ? rsqrtf(d2) : 0.f) : rsqrtf(d2);
            sh_eval_monic<LA, ShT>((ShT)(ddx * inv), (ShT)(ddy * inv), (ShT)(ddz * inv), R);
          }
          if (!STORED) {
            int Q;
            const float ps = path_sum<float, float>(i, j, k, (int)q.z, (int)q.y, (int)q.x, a.mutf, a.nx, plane, Q);
            kk = __expf(-ps * dist / (float)Q) * kscalef / d2;
          }
          f2_t R2[C2];
#pragma unroll
          for (int c = 0; c < C2; ++c) R2[c] = f2_pack((float)R[2 * c], 2 * c + 1 < C ? (float)R[2 * c + 1] : 0.f);
          if constexpr (CPLX) {
            float Sv[2];
#pragma unroll
            for (int b = 0; b < 2; ++b) {
              const f2_t* w = reinterpret_cast<const f2_t*>(Wt + sv * CP + b * CS);
              f2_t Sa = 0ull, Sb = 0ull;
#pragma unroll
              for (int c = 0; c < C2; c += 2) {
                Sa = f2_fma(R2[c], w[c], Sa);
                if (c + 1 < C2) Sb = f2_fma(R2[c + 1], w[c + 1], Sb);
              }
              float a0, a1, b0, b1;
              f2_unpack(Sa, a0, a1);
              f2_unpack(Sb, b0, b1);
              Sv[b] = (a0 + a1) + (b0 + b1);
            }
            float sn, cs;
            sincosf((float)a.kappa * sqrtf(d2), &sn, &cs);
            const float t0 = kk * (cs * Sv[0] + sn * Sv[1]), t1 = kk * (cs * Sv[1] - sn * Sv[0]);
            const f2_t T0 = f2_pack(t0, t0), T1 = f2_pack(t1, t1);
#pragma unroll
            for (int c = 0; c < C2; ++c) {
              acc[0][c] = f2_fma(R2[c], T0, acc[0][c]);
              acc[NB - 1][c] = f2_fma(R2[c], T1, acc[NB - 1][c]);
            }
          } else {
#pragma unroll
          for (int b = 0; b < NB; ++b) {
            const f2_t* w = reinterpret_cast<const f2_t*>(Wt + sv * CP + b * CS);
            f2_t Sa = 0ull, Sb = 0ull;
#pragma unroll
            for (int c = 0; c < C2; c += 2) {
              Sa = f2_fma(R2[c], w[c], Sa);
              if (c + 1 < C2) Sb = f2_fma(R2[c + 1], w[c + 1], Sb);
            }
            float a0, a1, b0, b1;
            f2_unpack(Sa, a0, a1);
            f2_unpack(Sb, b0, b1);
            const float tb = kk * ((a0 + a1) + (b0 + b1));
            const f2_t T2 = f2_pack(tb, tb);
#pragma unroll
            for (int c = 0; c < C2; ++c) acc[b][c] = f2_fma(R2[c], T2, acc[b][c]);
          }
          }
        }
      }
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < C2; ++c) {
          float lo, hi;
          f2_unpack(acc[b][c], lo, hi);
          sAcc[(b * C + 2 * c) * T + tid] += lo;
          if (2 * c + 1 < C) sAcc[(b * C + 2 * c + 1) * T + tid] += hi;
        }
    }
    __syncthreads();  // buffer t & 1 is free for tile t + 2
  }
  if (act) {
    const int vstride = NB * a.Cfull;
    double* o = a.part + ((size_t)blockIdx.y * a.N + r) * vstride;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < C; ++c) o[b * a.Cfull + c] = (double)sAcc[(b * C + c) * T + tid] * kMonic.N[c];
  }
}

// Stored pair kernel with exact directions (the benchmark's form): the kernel values of each 32-source
// tile for the CTA's 128 destinations are one contiguous block of the blocked K layout (kmat_index) and
// arrive by bulk copy on the same mbarrier as the tile's FP32 rows and coordinates, so the pair loop
// reads K from shared memory instead of waiting on a global load per source.  The FP32 accumulators stay
// in registers across the chunk's tiles (the chunks are summed in FP64 by the epilogue), which frees the
// shared-memory accumulator and leaves room for the K tiles.
// The source tile size TS (32 or 64) is chosen per shape by the autotuner (PairArgs::tile).
struct TkLayout {
  size_t off_w, off_k, off_bar, bytes;
  __host__ __device__ TkLayout(int cpad, int ts) {
    off_w = sizeof(float4) * 2 * ts;
    off_k = off_w + sizeof(float) * 2 * ts * (size_t)cpad;  // cpad is a multiple of 4: 16-byte aligned
    off_bar = off_k + sizeof(float) * 2 * ts * RTE_KBLK;
    bytes = off_bar + 2 * sizeof(uint64_t);
  }
};

template <int LA, int NB, int TS>
__global__ void __launch_bounds__(RTE_PAIR_THREADS) k_pair_mixed_tk(PairArgs a) {
  static_assert(RTE_PAIR_THREADS == RTE_KBLK, "one K block per CTA");
  constexpr int C = (LA + 1) * (LA + 1), T = RTE_PAIR_THREADS;
  typedef typename std::conditional<(LA >= 7), double, float>::type ShT;
  // 16-byte source-row loads, except for wide L = 7 rows where the extra registers cost more than the
  // loads save (33^3 L=7, 2 RHS: 30.1 -> 33.8 ms per launch with them)
  constexpr bool V4 = LA < 7 || NB == 1;
  const int CP = a.cpad;
  const TkLayout Sh(CP, TS);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sP = reinterpret_cast<float4*>(smem_raw);
  float* sW = reinterpret_cast<float*>(smem_raw + Sh.off_w);
  float* sK = reinterpret_cast<float*>(smem_raw + Sh.off_k);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + Sh.off_bar);
  const int tid = threadIdx.x;
  const int slot = blockIdx.x * T + tid;
  const bool act = slot < a.N;
  const float4 me = a.slot_xyz[act ? slot : 0];
  const int r = __float_as_int(me.w);
  const float dxf = (float)a.dx, dyf = (float)a.dy, dzf = (float)a.dz;
  const int sb = blockIdx.y * a.chunk;
  const int se = min(a.N, sb + a.chunk);
  const int ntile = (se - sb + TS - 1) / TS;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const float* Kblk = a.Kmat + kmat_index(0, (size_t)blockIdx.x * T, a.Kld);  // this CTA's destination block
  auto issue = [&](int t) {  // tile t -> buffer t & 1 (one thread)
    const int s0 = sb + t * TS;
    const int ns = min(TS, se - s0);
    const int b = t & 1;
    const uint32_t bw = (uint32_t)(ns * CP * sizeof(float)), bp = (uint32_t)(ns * sizeof(float4)),
                   bk = (uint32_t)(ns * RTE_KBLK * sizeof(float));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[b], bw + bp + bk);
    bulk_g2s(sW + b * TS * CP, a.Winf + (size_t)s0 * CP, bw, &bar[b]);
    bulk_g2s(sP + b * TS, a.slot_xyz + s0, bp, &bar[b]);
    bulk_g2s(sK + b * TS * RTE_KBLK, Kblk + (size_t)s0 * RTE_KBLK, bk, &bar[b]);
  };
  if (tid == 0 && ntile > 0) issue(0);
  constexpr int C2 = (C + 1) / 2;  // coefficient pairs (packed f32x2 arithmetic)
  const int CS = a.cstride;        // FP32 row stride of one right-hand side (a multiple of 4)
  f2_t acc[NB][C2];
#pragma unroll
  for (int b = 0; b < NB; ++b)
#pragma unroll
    for (int c = 0; c < C2; ++c) acc[b][c] = 0ull;
  for (int t = 0; t < ntile; ++t) {
    if (tid == 0 && t + 1 < ntile) issue(t + 1);
    const bool ok = mbar_wait(&bar[t & 1], (uint32_t)((t >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(a.err, 1);
      return;
    }
    const int ns = min(TS, se - (sb + t * TS));
    const float4* P = sP + (t & 1) * TS;
    const float* Wt = sW + (t & 1) * TS * CP;
    const float* Kt = sK + (t & 1) * TS * RTE_KBLK + tid;
    if (act) {
      // no per-pair branch: the diagonal and pairs beyond the coupling distance carry K = 0
#pragma unroll 4
      for (int sv = 0; sv < ns; ++sv) {
        const float kk = Kt[sv * RTE_KBLK];
        const float4 q = P[sv];
        const float ddx = (me.x - q.x) * dxf, ddy = (me.y - q.y) * dyf, ddz = (me.z - q.z) * dzf;
        const float d2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
        const float inv = d2 > 0.f ? rsqrtf(d2) : 0.f;
        ShT R[C];
        sh_eval_monic<LA, ShT>((ShT)(ddx * inv), (ShT)(ddy * inv), (ShT)(ddz * inv), R);
        f2_t R2[C2];
#pragma unroll
        for (int c = 0; c < C2; ++c) R2[c] = f2_pack((float)R[2 * c], 2 * c + 1 < C ? (float)R[2 * c + 1] : 0.f);
#pragma unroll
        for (int b = 0; b < NB; ++b) {
          // broadcast loads of the source row (CS and CP are multiples of 4 floats; the padding beyond C
          // is zero)
          f2_t Sa = 0ull, Sb = 0ull;
          if constexpr (V4) {
            const float4* w4 = reinterpret_cast<const float4*>(Wt + sv * CP + b * CS);
#pragma unroll
            for (int c = 0; c < C2; c += 2) {
              const float4 v = w4[c / 2];
              Sa = f2_fma(R2[c], f2_pack(v.x, v.y), Sa);
              if (c + 1 < C2) Sb = f2_fma(R2[c + 1], f2_pack(v.z, v.w), Sb);
            }
          } else {
            const f2_t* w = reinterpret_cast<const f2_t*>(Wt + sv * CP + b * CS);
#pragma unroll
            for (int c = 0; c < C2; c += 2) {
              Sa = f2_fma(R2[c], w[c], Sa);
              if (c + 1 < C2) Sb = f2_fma(R2[c + 1], w[c + 1], Sb);
            }
          }
          float a0, a1, b0, b1;
          f2_unpack(Sa, a0, a1);
          f2_unpack(Sb, b0, b1);
          const float tb = kk * ((a0 + a1) + (b0 + b1));
          const f2_t T2 = f2_pack(tb, tb);
#pragma unroll
          for (int c = 0; c < C2; ++c) acc[b][c] = f2_fma(R2[c], T2, acc[b][c]);
        }
      }
    }
    __syncthreads();  // buffer t & 1 is free for tile t + 2
  }
  if (act) {  // the chunk's FP32 sums as they are (the epilogue applies N_c after adding the chunks in FP64)
    const int vstride = NB * a.Cfull;
    float* o = a.partf + ((size_t)blockIdx.y * a.N + r) * vstride;
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < C2; ++c) {
        float lo, hi;
        f2_unpack(acc[b][c], lo, hi);
        o[b * a.Cfull + 2 * c] = lo;
        if (2 * c + 1 < C) o[b * a.Cfull + 2 * c + 1] = hi;
      }
  }
}

// Recomputed pair kernel for four right-hand sides at L >= 6 (exact directions, real rows), where four
// right-hand sides' FP32 sums no longer fit one thread's registers: 256 threads per CTA, the 128
// destinations of a K block twice over, thread group g = tid / 128 holding right-hand sides 2g and
// 2g + 1.  The path walks are shared: the kernel values of the CTA's 128 destinations x a 32-source tile
// go to shared memory, each group walking half of the tile's sources, so every pair is walked once for
// the four right-hand sides instead of once per pair of them.  The walks for tile t + 1 are interleaved
// with the projections of tile t (one walk after every second source), so each thread's instruction
// stream mixes the integer walk with the FMA work as the one-group kernels do.  FP32 sums stay in
// registers over the source chunk (FP32 chunk partials, as k_pair_mixed_tk).
struct GrpLayout {
  size_t off_w, off_k, off_bar, bytes;
  __host__ __device__ GrpLayout(int cpad, int ts) {
    off_w = sizeof(float4) * 2 * ts;
    off_k = off_w + sizeof(float) * 2 * ts * (size_t)cpad;  // cpad is a multiple of 4: 16-byte aligned
    off_bar = off_k + sizeof(float) * 2 * ts * RTE_KBLK;
    bytes = off_bar + 2 * sizeof(uint64_t);
  }
};
#define RTE_GRP_THREADS (2 * RTE_KBLK)
#define RTE_GRP_TS 32

template <int LA>
__global__ void __launch_bounds__(RTE_GRP_THREADS, 1) k_pair_mixed_grp(PairArgs a) {
  constexpr int C = (LA + 1) * (LA + 1), C2 = (C + 1) / 2, TS = RTE_GRP_TS, NBG = 2, HALF = TS / 2;
  typedef typename std::conditional<(LA >= 7), double, float>::type ShT;
  constexpr bool V4 = LA < 7;  // 16-byte row loads (the one-group rule for two right-hand sides)
  const int CP = a.cpad;
  const GrpLayout Sh(CP, TS);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* sP = reinterpret_cast<float4*>(smem_raw);
  float* sW = reinterpret_cast<float*>(smem_raw + Sh.off_w);
  float* sK = reinterpret_cast<float*>(smem_raw + Sh.off_k);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + Sh.off_bar);
  const int tid = threadIdx.x;
  const int d = tid & (RTE_KBLK - 1), g = tid / RTE_KBLK;
  const int slot = blockIdx.x * RTE_KBLK + d;
  const bool act = slot < a.N;
  const float4 me = a.slot_xyz[act ? slot : 0];
  const int r = __float_as_int(me.w);
  const int plane = a.nx * a.ny;
  const int i = (int)me.z, j = (int)me.y, k = (int)me.x;
  const float dxf = (float)a.dx, dyf = (float)a.dy, dzf = (float)a.dz;
  const float kscalef = (float)a.kscale, thr = (float)a.prop_thresh;
  const int sb = blockIdx.y * a.chunk;
  const int se = min(a.N, sb + a.chunk);
  const int ntile = (se - sb + TS - 1) / TS;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto issue = [&](int t) {  // source rows and coordinates of tile t -> buffer t & 1 (one thread)
    const int s0 = sb + t * TS;
    const int ns = min(TS, se - s0);
    const int b = t & 1;
    const uint32_t bw = (uint32_t)(ns * CP * sizeof(float)), bp = (uint32_t)(ns * sizeof(float4));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bar[b], bw + bp);
    bulk_g2s(sW + b * TS * CP, a.Winf + (size_t)s0 * CP, bw, &bar[b]);
    bulk_g2s(sP + b * TS, a.slot_xyz + s0, bp, &bar[b]);
  };
  // the pair kernel exp(-tau) dV/(cm r^2) of this destination and source q, as the one-group kernels
  // recompute it (0 on the diagonal and beyond the coupling distance)
  auto kval = [&](const float4 q) -> float {
    const float ddx = (me.x - q.x) * dxf, ddy = (me.y - q.y) * dyf, ddz = (me.z - q.z) * dzf;
    const float d2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
    const float dist = sqrtf(d2);
    if (!(d2 > 0.f && dist < thr)) return 0.f;
    int Q;
    const float ps = path_sum<float, float>(i, j, k, (int)q.z, (int)q.y, (int)q.x, a.mutf, a.nx, plane, Q);
    return __expf(-ps * dist / (float)Q) * kscalef / d2;
  };
  f2_t acc[NBG][C2];
#pragma unroll
  for (int b = 0; b < NBG; ++b)
#pragma unroll
    for (int c = 0; c < C2; ++c) acc[b][c] = 0ull;
  if (ntile > 0) {
    if (tid == 0) issue(0);
    const bool ok = mbar_wait(&bar[0], 0u);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(a.err, 1);
      return;
    }
    if (tid == 0 && ntile > 1) issue(1);
    const int ns0 = min(TS, se - sb);
    if (act)
      for (int h = 0; h < HALF; ++h) {
        const int sv = g * HALF + h;
        if (sv < ns0) sK[sv * RTE_KBLK + d] = kval(sP[sv]);
      }
    __syncthreads();
  }
  const int CS = a.cstride;  // FP32 row stride of one right-hand side (a multiple of 4)
  for (int t = 0; t < ntile; ++t) {
    const bool has_next = t + 1 < ntile;
    bool ok = true;
    if (has_next) ok = mbar_wait(&bar[(t + 1) & 1], (uint32_t)(((t + 1) >> 1) & 1));
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicExch(a.err, 1);
      return;
    }
    const int ns = min(TS, se - (sb + t * TS));
    const int nsn = has_next ? min(TS, se - (sb + (t + 1) * TS)) : 0;
    const float4* P = sP + (t & 1) * TS;
    const float* Wt = sW + (t & 1) * TS * CP + 2 * g * CS;  // this group's two right-hand sides
    const float* Kt = sK + (t & 1) * TS * RTE_KBLK + d;
    const float4* Pn = sP + ((t + 1) & 1) * TS;
    float* Kn = sK + ((t + 1) & 1) * TS * RTE_KBLK + d;
    if (act) {
      for (int sv = 0; sv < ns; ++sv) {
        const float kk = Kt[sv * RTE_KBLK];
        const float4 q = P[sv];
        const float ddx = (me.x - q.x) * dxf, ddy = (me.y - q.y) * dyf, ddz = (me.z - q.z) * dzf;
        const float d2 = fmaf(ddx, ddx, fmaf(ddy, ddy, ddz * ddz));
        const float inv = d2 > 0.f ? rsqrtf(d2) : 0.f;
        ShT R[C];
        sh_eval_monic<LA, ShT>((ShT)(ddx * inv), (ShT)(ddy * inv), (ShT)(ddz * inv), R);
        f2_t R2[C2];
#pragma unroll
        for (int c = 0; c < C2; ++c) R2[c] = f2_pack((float)R[2 * c], 2 * c + 1 < C ? (float)R[2 * c + 1] : 0.f);
#pragma unroll
        for (int b = 0; b < NBG; ++b) {
          f2_t Sa = 0ull, Sb = 0ull;
          if constexpr (V4) {
            const float4* w4 = reinterpret_cast<const float4*>(Wt + sv * CP + b * CS);
#pragma unroll
            for (int c = 0; c < C2; c += 2) {
              const float4 v = w4[c / 2];
              Sa = f2_fma(R2[c], f2_pack(v.x, v.y), Sa);
              if (c + 1 < C2) Sb = f2_fma(R2[c + 1], f2_pack(v.z, v.w), Sb);
            }
          } else {
            const f2_t* w = reinterpret_cast<const f2_t*>(Wt + sv * CP + b * CS);
#pragma unroll
            for (int c = 0; c < C2; c += 2) {
              Sa = f2_fma(R2[c], w[c], Sa);
              if (c + 1 < C2) Sb = f2_fma(R2[c + 1], w[c + 1], Sb);
            }
          }
          float a0, a1, b0, b1;
          f2_unpack(Sa, a0, a1);
          f2_unpack(Sb, b0, b1);
          const float tb = kk * ((a0 + a1) + (b0 + b1));
          const f2_t T2 = f2_pack(tb, tb);
#pragma unroll
          for (int c = 0; c < C2; ++c) acc[b][c] = f2_fma(R2[c], T2, acc[b][c]);
        }
        if ((sv & 1) == 0) {  // one walk of the next tile after every second source
          const int svn = g * HALF + (sv >> 1);
          if (svn < nsn) Kn[svn * RTE_KBLK] = kval(Pn[svn]);
        }
      }
      // a short last tile leaves walks of the next tile undone only when there is no next tile
    }
    __syncthreads();  // tile t's buffers are free, tile t + 1's kernel values complete
    if (tid == 0 && t + 2 < ntile) issue(t + 2);
  }
  if (act) {  // the chunk's FP32 sums (the epilogue applies N_c after adding the chunks in FP64)
    const int vstride = 2 * NBG * a.Cfull;
    float* o = a.partf + ((size_t)blockIdx.y * a.N + r) * vstride + (size_t)(NBG * g) * a.Cfull;
#pragma unroll
    for (int b = 0; b < NBG; ++b)
#pragma unroll
      for (int c = 0; c < C2; ++c) {
        float lo, hi;
        f2_unpack(acc[b][c], lo, hi);
        o[b * a.Cfull + 2 * c] = lo;
        if (2 * c + 1 < C) o[b * a.Cfull + 2 * c + 1] = hi;
      }
  }
}

// Launch wrappers.  k_pair_mixed_3 carries a 3-CTA register bound and is used for L = 7 with one
// right-hand side only; an explicit minimum-block count on the others makes ptxas take more registers
// (L = 5, 2 RHS: 218 instead of 164, two CTAs per SM instead of three, 13.2 -> 17.0 ms per launch).
template <int LA, bool TABLE, bool STORED, int NB, bool CPLX>
__global__ void __launch_bounds__(RTE_PAIR_THREADS) k_pair_mixed(PairArgs a) {
  pair_mixed_body<LA, TABLE, STORED, NB, CPLX>(a);
}
template <int LA, bool TABLE, bool STORED, int NB, bool CPLX>
__global__ void __launch_bounds__(RTE_PAIR_THREADS, 3) k_pair_mixed_3(PairArgs a) {
  pair_mixed_body<LA, TABLE, STORED, NB, CPLX>(a);
}

// Pair-kernel precompute K[s][d] = exp(-tau) dV/(cm |r_d - r_s|^2) over destination slots d and
// source slots s (0 on the diagonal and beyond propThresh), path sums in FP32 (T = float, into Kmat)
// or FP64 (T = double, into Kmat64, for the FP64 method).  K is symmetric: one CTA computes a 64x64
// tile with source tile index <= destination tile index into shared memory and writes it and its
// transpose with coalesced stores (a diagonal tile once).
#define RTE_KT 64
template <typename T>
__global__ void __launch_bounds__(RTE_KT) k_store_kernel(PairArgs a) {
  constexpr bool F64 = std::is_same<T, double>::value;
  __shared__ T tile[RTE_KT][RTE_KT + 1];
  __shared__ int sxyz[RTE_KT][3];
  const int ntile = (a.N + RTE_KT - 1) / RTE_KT;
  // linear CTA index -> (bs, bd) with bs <= bd, row-major over the upper triangle
  long long t = blockIdx.x;
  int bd = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((long long)(bd + 1) * (bd + 2) / 2 <= t) ++bd;
  while ((long long)bd * (bd + 1) / 2 > t) --bd;
  const int bs = (int)(t - (long long)bd * (bd + 1) / 2);
  if (bd >= ntile) return;
  const int tid = threadIdx.x;
  const int plane = a.nx * a.ny;
  const int s0 = bs * RTE_KT, d0 = bd * RTE_KT;
  {
    const int sl = s0 + tid;
    const int v = sl < a.N ? a.perm[sl] : 0;
    sxyz[tid][0] = v % a.nx;
    sxyz[tid][1] = (v / a.nx) % a.ny;
    sxyz[tid][2] = v / plane;
  }
  __syncthreads();
  const int d = d0 + tid;
  if (d < a.N) {
    const int r = a.perm[d];
    const int k = r % a.nx, j = (r / a.nx) % a.ny, i = r / plane;
    const T dxf = (T)a.dx, dyf = (T)a.dy, dzf = (T)a.dz;
    const T kscalef = (T)a.kscale, thr = (T)a.prop_thresh;
    for (int q = 0; q < RTE_KT; ++q) {
      T kk = T(0);
      if (s0 + q < a.N) {
        const int kp = sxyz[q][0], jp = sxyz[q][1], ip = sxyz[q][2];
        const T ddx = (T)(k - kp) * dxf, ddy = (T)(j - jp) * dyf, ddz = (T)(i - ip) * dzf;
        const T d2 = fma(ddx, ddx, fma(ddy, ddy, ddz * ddz));
        const T dist = sqrt(d2);
        if (d2 > T(0) && dist < thr) {
          int Q;
          if constexpr (F64) {
            const double ps = path_sum<double, double>(i, j, k, ip, jp, kp, a.mut, a.nx, plane, Q);
            kk = exp(-ps * dist / (double)Q) * kscalef / d2;
          } else {
            const float ps = path_sum<float, float>(i, j, k, ip, jp, kp, a.mutf, a.nx, plane, Q);
            kk = __expf(-ps * dist / (float)Q) * kscalef / d2;
          }
        }
      }
      tile[tid][q] = kk;  // [destination][source]
    }
  }
  __syncthreads();
  // K(s, d): FP64 row-major [source slot][destination slot]; FP32 in 128-destination blocks
  // (kmat_index).  Either way the 64 destinations of a tile row are contiguous (d0 is a multiple of 64).
  auto at = [&](size_t sl, size_t d) -> T& {
    if constexpr (F64)
      return a.Kmat64[sl * a.Kld + d];
    else
      return a.Kmat[kmat_index(sl, d, a.Kld)];
  };
  for (int q = 0; q < RTE_KT; ++q) {
    const int sl = s0 + q;
    if (sl < a.N && d0 + tid < a.N) at(sl, d0 + tid) = tile[tid][q];
  }
  if (bs != bd) {
    // K(d, s): the destination slots of this tile acting as sources
    for (int q = 0; q < RTE_KT; ++q) {
      const int dl = d0 + q;
      if (dl < a.N && s0 + tid < a.N) at(dl, s0 + tid) = tile[q][tid];
    }
  }
}

// Weight of real coefficient c in the reference stop rule's layer sum, sum over m of Re(w_lm) in the
// complex basis (dist.cu:1143-1152): for a real function R_l0 + sqrt2 R_l,m (even m > 0); for the
// imaginary part f2 of a complex function (w = w1 + i w2, Re(i w2_lm) = -Im(w2_lm)) sqrt2 R_l,-m for
// odd m > 0.
__device__ __forceinline__ double stop_weight(int c, bool imag) {
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  const int m = c - l * l - l;
  if (imag) return (m < 0 && ((-m) & 1)) ? 1.4142135623730951 : 0.0;
  return m == 0 ? 1.0 : ((m > 0 && (m % 2) == 0) ? 1.4142135623730951 : 0.0);
}

// ---------------------------------------------------------------------------------------------
// Epilogue: add split-K partials, self-voxel term, scatter; write the next term (FP64 and FP32),
// accumulate the running sum and the norms used by the stop rules.  One thread per (voxel, right-hand
// side, coefficient) element, grid-stride, so every stream (partials, self term, outputs, running sum)
// is read and written coalesced; the four norms are reduced per block and added atomically.
// Self term: computed by k_self into selfp.  Coefficients above (LA+1)^2 are written as 0.
__global__ void __launch_bounds__(256) k_epilogue(EpiArgs a, int Cact) {
  const int nb = a.nb > 0 ? a.nb : 1;
  const int vstride = nb * a.Cfull;
  const size_t total = (size_t)a.N * vstride, NV = (size_t)a.N * vstride;
  const int plane = a.nx * a.ny;
  double w2 = 0.0, s2 = 0.0, lw = 0.0, ls = 0.0;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(t / vstride), e = (int)(t - (size_t)r * vstride);
    const int b = e / a.Cfull, c = e - b * a.Cfull;
    int l = 0;
    while ((l + 1) * (l + 1) <= c) ++l;
    double x = 0.0;
    if (c < Cact) {
      x = a.selfp ? a.selfp[t] : 0.0;
      if (a.partf) {  // FP32 chunk sums of the tile-staged kernel: FP64 sum over the chunks, then N_c
        double u = 0.0;
        for (int q = 0; q < a.S; ++q) u += (double)a.partf[(size_t)q * NV + t];
        x = fma(u, kMonic.N[c], x);
      } else {
        for (int q = 0; q < a.S; ++q) x += a.part[(size_t)q * NV + t];
      }
      if (a.flag_scat) x *= a.scat[l] * a.mus[r];
    }
    a.Wout[t] = x;
    // the mixed pair kernels read N_c W_c (monic SH, sh_eval_monic)
    if (a.Woutf) a.Woutf[(size_t)a.islot[r] * a.cpad + (size_t)b * a.cstride + c] = (float)(x * kMonic.N[c]);
    w2 += x * x;
    double sv = 0.0;
    if (a.sum) {
      sv = a.sum[t] + x;
      a.sum[t] = sv;
      s2 += sv * sv;
    }
    if (r / plane == a.nz - 1) {  // the reference stop rule's layer
      const double wgt = stop_weight(c, a.cplx && (b & 1));
      lw += wgt * x;
      ls += wgt * sv;
    }
  }
  // block reduction of the four norms
  __shared__ double red[4][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double vals[4] = {w2, s2, lw, ls};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double x = vals[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[q][wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double x = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[threadIdx.x][w];
    atomicAdd(a.red + threadIdx.x, x);
  }
}

// Self-voxel term (compute_diagonal_abs, FisherInfo_IO/src/kernels.cu:151-178, and its dV scale)
// for every voxel, right-hand side and output coefficient (one thread each):
//   out[r][b][c] = scale * sum_c' D(mu_t(r))[c][c'] W[r][b][c'],
// D from a table of the medium's distinct mu_t values (lut/idx), else by the power series
// D(mu) = sum_k mu^k M_k (Horner).  FIM model: voxels with mu_t == 0 (tissue 0) get nothing.
__global__ void k_self(SelfArgs a) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)a.N * a.nb * a.Cact;
  if (t >= total) return;
  const int c = (int)(t % a.Cact);
  const int b = (int)((t / a.Cact) % a.nb);
  const int r = (int)(t / ((long long)a.Cact * a.nb));
  const size_t base = (size_t)r * a.nb * a.Cfull + (size_t)b * a.Cfull;
  const double mu = a.mut[r];
  double u = 0.0;
  if (!(a.air_no_self && mu == 0.0)) {
    const double* w = a.W + base;
    const bool der = a.dmut != nullptr;
    if (a.idx) {
      const double* D = (der ? a.dlut : a.lut) + ((size_t)a.idx[r] * a.Cfull + c) * a.Cfull;
      for (int cp = 0; cp < a.Cact; ++cp) u = fma(__ldg(D + cp), __ldg(w + cp), u);
    } else {  // D(mu) = sum_k mu^k M_k; its derivative sum_k k mu^(k-1) M_k, both by Horner
      for (int kk = a.K - 1; kk >= (der ? 1 : 0); --kk) {
        const double* M = a.mom + ((size_t)kk * a.Cfull + c) * a.Cfull;
        double tk = 0.0;
        for (int cp = 0; cp < a.Cact; ++cp) tk = fma(__ldg(M + cp), __ldg(w + cp), tk);
        u = fma(mu, u, der ? (double)kk * tk : tk);
      }
    }
    if (der) u *= a.dmut[r];
  }
  a.out[base + c] = a.scale * u;
}

// Self-voxel term with the complex mu_t + i kappa of intensity modulation (the CPU package's
// (1 - exp(-mu_t beta)) / mu_t with complex mu_t, Kernels_selfsub.c:927-946): W holds (real,
// imaginary) row pairs; D from the complex table (lut, lut_im) or the power series in the complex
// mu_t.  One thread per voxel, complex right-hand side and output coefficient.
__global__ void k_self_cplx(SelfArgs a) {
  const int npair = a.nb / 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)a.N * npair * a.Cact;
  if (t >= total) return;
  const int c = (int)(t % a.Cact);
  const int p = (int)((t / a.Cact) % npair);
  const int r = (int)(t / ((long long)a.Cact * npair));
  const size_t base = (size_t)r * a.nb * a.Cfull + (size_t)(2 * p) * a.Cfull;
  const double* w0 = a.W + base;
  const double* w1 = w0 + a.Cfull;
  double ur = 0.0, ui = 0.0;
  if (a.idx) {
    const size_t row = ((size_t)a.idx[r] * a.Cfull + c) * a.Cfull;
    const double* Dr = a.lut + row;
    const double* Di = a.lut_im + row;
    for (int cp = 0; cp < a.Cact; ++cp) {
      const double dr = __ldg(Dr + cp), di = __ldg(Di + cp), x0 = __ldg(w0 + cp), x1 = __ldg(w1 + cp);
      ur = fma(dr, x0, fma(-di, x1, ur));
      ui = fma(dr, x1, fma(di, x0, ui));
    }
  } else {  // Horner in the complex mu: u <- mu u + M_k w
    const double mr = a.mut[r], mi = a.kappa;
    for (int kk = a.K - 1; kk >= 0; --kk) {
      const double* M = a.mom + ((size_t)kk * a.Cfull + c) * a.Cfull;
      double t0 = 0.0, t1 = 0.0;
      for (int cp = 0; cp < a.Cact; ++cp) {
        const double m = __ldg(M + cp);
        t0 = fma(m, __ldg(w0 + cp), t0);
        t1 = fma(m, __ldg(w1 + cp), t1);
      }
      const double nr = mr * ur - mi * ui + t0, ni = mr * ui + mi * ur + t1;
      ur = nr;
      ui = ni;
    }
  }
  a.out[base + c] = a.scale * ur;
  a.out[base + a.Cfull + c] = a.scale * ui;
}

// Exitance images of the z = nZ-1 and z = 0 faces from the m = 0 coefficients
// (FisherInfo_IO/src/dist.cu:103-161, 229-268; the per-l weights come from the host).
__global__ void k_images(ImgArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.nx * a.ny) return;
  const double* out_im = a.out_im;
  const size_t rt = (size_t)(a.nz - 1) * a.nx * a.ny + p, rr = (size_t)p;
  double t = 0.0, f = 0.0, ti = 0.0, fi = 0.0;
  for (int l = 0; l <= a.L; ++l) {
    const int c = l * l + l;
    t += a.wt[l] * a.out[rt * a.vstride + c];
    f += a.wr[l] * a.out[rr * a.vstride + c];
    if (out_im) {
      ti += a.wt[l] * out_im[rt * a.vstride + c];
      fi += a.wr[l] * out_im[rr * a.vstride + c];
    }
  }
  if (a.fball) {
    t += a.fball[(size_t)a.nx * a.ny + p];
    f += a.fball[p];
  }
  if (a.fball_im) {
    ti += a.fball_im[(size_t)a.nx * a.ny + p];
    fi += a.fball_im[p];
  }
  if (a.trans) {
    a.trans[2 * p] = t;
    a.trans[2 * p + 1] = ti;
  }
  if (a.ref) {
    a.ref[2 * p] = f;
    a.ref[2 * p + 1] = fi;
  }
}

// Collimated-beam source xi = D A xi_beam on the pencil columns (one thread per column), with the
// ballistic transmission of each column.  FisherInfo_IO/src/dist.cu:66-101 (product of per-layer
// attenuations) and, for kind 2, CPU package/src/Dist.c:1077-1128 (attenuation from the absolute
// depth of the voxel, normalised by the number of columns).
__global__ void k_source(SrcArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= a.ncols) return;
  const int p = a.cols[q];
  const int plane = a.nx * a.ny;
  const int axis = a.face / 2;  // 0: along z, 1: along y, 2: along x
  const bool up = (a.face & 1) == 0;
  int n, base, stride, row, col;
  if (axis == 0) {
    n = a.nz;
    base = p;
    stride = plane;
  } else if (axis == 1) {
    n = a.ny;
    row = p / a.nx;  // i
    col = p % a.nx;  // k
    base = row * plane + col;
    stride = a.nx;
  } else {
    n = a.nx;
    row = p / a.ny;  // i
    col = p % a.ny;  // j
    base = row * plane + col * a.nx;
    stride = 1;
  }
  // attenuation with mu_t + i kappa (kappa = 0: the steady state); complex values as (re, im)
  const double kap = a.kappa;
  auto cexpm = [kap](double m, double x, double& re, double& im) {  // exp(-(m + i kap) x)
    const double e = exp(-m * x);
    double sn = 0.0, cs = 1.0;
    if (kap != 0.0) sincos(kap * x, &sn, &cs);
    re = e * cs;
    im = -e * sn;
  };
  double attr = 1.0, atti = 0.0, mt = 0.0;
  for (int t = 0; t < n; ++t) {
    const size_t r = (size_t)base + (size_t)(up ? t : n - 1 - t) * stride;
    mt = a.mut[r];
    const double ms = a.mus[r];
    double vr, vi, er, ei;
    cexpm(mt, a.dlen, er, ei);
    if (a.kind == 2) {  // absolute depth of the voxel top (z- entry only)
      const double tz = (double)t * a.dz + a.z_min + a.dz / 2.0 - a.dz / 2.0;
      double e1r, e1i, e2r, e2i;
      cexpm(mt, tz, e1r, e1i);
      cexpm(mt, tz + a.dz, e2r, e2i);
      vr = e1r - e2r;
      vi = e1i - e2i;
    } else {  // att * (1 - exp(-mu dlen))
      vr = attr * (1.0 - er) + atti * ei;
      vi = atti * (1.0 - er) - attr * ei;
    }
    const double nr = attr * er - atti * ei, ni = attr * ei + atti * er;
    attr = nr;
    atti = ni;
    // amp = ms / (mt + i kap) * v / dV
    double ar, ai = 0.0;
    if (kap == 0.0) {
      ar = ms / mt * vr / a.dV;
    } else {
      const double den = mt * mt + kap * kap;
      ar = ms * (mt * vr + kap * vi) / den / a.dV;
      ai = ms * (mt * vi - kap * vr) / den / a.dV;
    }
    for (int c = 0; c < a.Cfull; ++c)
      if (a.coef[c] != 0.0) {
        a.W[r * a.vstride + c] += ar * a.coef[c];
        if (kap != 0.0) a.W[r * a.vstride + a.Cfull + c] += ai * a.coef[c];
      }
  }
  // exit face = the opposite face, same in-face pixel
  const int ef = a.face ^ 1;
  const size_t a0 = (size_t)a.nx * a.ny, a1 = (size_t)a.nz * a.nx, a2 = (size_t)a.nz * a.ny;
  const size_t off[6] = {0, a0, 2 * a0, 2 * a0 + a1, 2 * a0 + 2 * a1, 2 * a0 + 2 * a1 + a2};
  double br, bi;
  if (a.kind == 2) {
    const double zs = (double)(a.nz - 1) * a.dz + a.z_min + a.dz / 2.0;
    cexpm(mt, zs + a.dz / 2.0, br, bi);
    br *= a.scale;
    bi *= a.scale;
  } else {
    br = a.mag * attr;
    bi = a.mag * atti;
  }
  a.fball[off[ef] + p] = br;
  if (a.fball_im) a.fball_im[off[ef] + p] = bi;
}

// mu_t = mu_a + mu_s (FP64 and FP32 copies), mu_s copy, and max(mu_t) into red_max (>= 0 values,
// so the bit pattern orders like the value).
__global__ void k_medium(const double* mua, const double* mus, double* mut, double* mus_out, float* mutf, int N,
                         double* red_max) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.0;
  if (r < N) {
    m = mua[r] + mus[r];
    mut[r] = m;
    mutf[r] = (float)m;
    if (mus_out != mus) mus_out[r] = mus[r];
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax((unsigned long long*)red_max, (unsigned long long)__double_as_longlong(m));
}

// FMA throughput probe (roofline denominator for the CUDA-core-bound kernels): 8 independent FMA
// chains per thread; the result is written so the work cannot be removed.  k_fma2_peak does the
// same with packed f32x2 FMAs (two FP32 FMAs per instruction).
__global__ void k_fma2_peak(int iters, float* sink) {
  f2_t a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = f2_pack((float)(threadIdx.x + q) * 1e-3f, (float)(threadIdx.x + 2 * q) * 1e-3f);
  const f2_t b = f2_pack(0.999999f, 0.999998f), c = f2_pack(1e-7f, 2e-7f);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = f2_fma(a[q], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    float lo, hi;
    f2_unpack(a[q], lo, hi);
    s += lo + hi;
  }
  if (s == -1.2345f) sink[blockIdx.x] = s;
}

// k_fma2_fresh_peak: packed FMAs whose three operands are all distinct registers (none shared with the
// neighbouring instructions), the operand pattern of the pair kernels' source-row dot products.
__global__ void k_fma2_fresh_peak(int iters, float* sink) {
  f2_t a[12], x[12], y[12];
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    a[q] = f2_pack((float)(threadIdx.x + q) * 1e-3f, (float)(threadIdx.x + 2 * q) * 1e-3f);
    x[q] = f2_pack(0.9999f + (float)q * 1e-7f, 0.9998f + (float)q * 1e-7f);
    y[q] = f2_pack(1e-7f * (float)(q + 1) + (float)threadIdx.x * 1e-9f, 2e-7f * (float)(q + 1));
  }
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 12; ++q) a[q] = f2_fma(x[q], a[q], y[q]);
  }
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    float lo, hi;
    f2_unpack(a[q], lo, hi);
    s += lo + hi;
  }
  if (s == -1.2345f) sink[blockIdx.x] = s;
}

template <typename T>
__global__ void k_fma_peak(int iters, float* sink) {
  T a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = (T)(threadIdx.x + q) * (T)1e-3;
  const T b = (T)0.999999, c = (T)1e-7;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = fma(a[q], b, c);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += a[q];
  if (s == (T)-1.2345) sink[blockIdx.x] = (float)s;
}

// ---------------------------------------------------------------------------------------------
// Detectors and the adjoint gradient.
// Face pixels: z-(ny*nx) z+(ny*nx) y-(nz*nx) y+(nz*nx) x-(nz*ny) x+(nz*ny), row-major.
__device__ __forceinline__ void face_pixel(int q, int nx, int ny, int nz, int& f, int& p, int& r) {
  const int a0 = nx * ny, a1 = nz * nx, a2 = nz * ny;
  const int off[6] = {0, a0, 2 * a0, 2 * a0 + a1, 2 * a0 + 2 * a1, 2 * a0 + 2 * a1 + a2};
  f = 5;
  for (int t = 1; t < 6; ++t)
    if (q < off[t]) {
      f = t - 1;
      break;
    }
  p = q - off[f];
  if (f < 2) {  // p = j*nx + k
    const int i = f == 0 ? 0 : nz - 1;
    r = i * nx * ny + p;
  } else if (f < 4) {  // p = i*nx + k
    const int i = p / nx, k = p % nx, j = f == 2 ? 0 : ny - 1;
    r = (i * ny + j) * nx + k;
  } else {  // p = i*ny + j
    const int i = p / ny, j = p % ny, k = f == 4 ? 0 : nx - 1;
    r = (i * ny + j) * nx + k;
  }
}

__global__ void k_face_flux(FaceArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = 2 * (a.nx * a.ny + a.nz * a.nx + a.nz * a.ny);
  if (q >= total) return;
  int f, p, r;
  face_pixel(q, a.nx, a.ny, a.nz, f, p, r);
  const double* h = a.h + f * a.Cfull;
  const double* o = a.out + (size_t)r * a.vstride;
  double J = 0.0;
  for (int c = 0; c < a.Cfull; ++c) J = fma(h[c], o[c], J);
  if (a.fball) J += a.fball[q];
  a.J[q] = J;
}

// e[r][c] += rho(pixel) h_f[c] for every face pixel (edge voxels belong to several faces)
__global__ void k_adjoint_seed(FaceArgs a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int total = 2 * (a.nx * a.ny + a.nz * a.nx + a.nz * a.ny);
  if (q >= total) return;
  const double rho = a.rho[q];
  if (rho == 0.0) return;
  int f, p, r;
  face_pixel(q, a.nx, a.ny, a.nz, f, p, r);
  for (int c = 0; c < a.Cfull; ++c) atomicAdd(a.e + (size_t)r * a.Cfull + c, rho * a.h[f * a.Cfull + c]);
}

// x *= (-1)^l: the parity of the real SH, R(-w) = (-1)^l R(w); the transpose of the pair operator
// is P A P.
__global__ void k_parity(double* x, int N, int L, int vstride) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int C = (L + 1) * (L + 1);
  if (t >= (long long)N * C) return;
  const int r = (int)(t / C), c = (int)(t % C);
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  if (l & 1) x[(size_t)r * vstride + c] = -x[(size_t)r * vstride + c];
}

// out[r][c] = mask[r] ? fac[l(c)] * in[r][c] : 0 -- the region-restricted tangent sources of the
// reference's inverse and Fisher mains (compute_grad_rte.cu:288-363, rte_fim.cu:253-273).
__global__ void k_masked_scale(const double* in, double* out, const uint8_t* mask, ScatTab fac, int N, int L) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int C = (L + 1) * (L + 1);
  if (t >= (long long)N * C) return;
  const int r = (int)(t / C), c = (int)(t % C);
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  out[t] = mask[r] ? fac.v[l] * in[t] : 0.0;
}

// Per voxel: ga[r] = sum_c fa[l(c)] lam[r][c] out[r][c], gs likewise with fs -- the reference's tangent
// sources (-C out for mu_a, (-C + g^l) out for mu_s, compute_grad_rte.cu:296-299, 343-350) paired with
// an adjoint field.
__global__ void k_tangent_pair_dots(const double* lam, const double* out, ScatTab fa, ScatTab fs, int N, int L,
                                    double* ga, double* gs) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int C = (L + 1) * (L + 1);
  const size_t b = (size_t)r * C;
  double a = 0.0, s = 0.0;
  for (int l = 0; l <= L; ++l)
    for (int c = l * l; c < (l + 1) * (l + 1); ++c) {
      const double p = lam[b + c] * out[b + c];
      a = fma(fa.v[l], p, a);
      s = fma(fs.v[l], p, s);
    }
  ga[r] = a;
  gs[r] = s;
}

__global__ void k_axpy(double* y, const double* x, double alpha, size_t n) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] = fma(alpha, x[t], y[t]);
}

// y = e + D lambda, D = scat_l mu_s(r)
__global__ void k_y_field(double* y, const double* e, const double* lam, const double* mus, ScatTab sc, int N, int L,
                          int Cfull) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * Cfull) return;
  const int r = (int)(t / Cfull), c = (int)(t % Cfull);
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  y[t] = e[t] + (l <= L ? sc.v[l] : 0.0) * mus[r] * lam[t];
}

// Segments of the centre-to-centre path of path_sum, each length handed to `add(v, len * Q / dist)`.
template <typename F>
__device__ __forceinline__ void path_walk(int i, int j, int k, int ip, int jp, int kp, int nx, int plane, int& Q,
                                          F add) {
  const int Dz = abs(ip - i), Dy = abs(jp - j), Dx = abs(kp - k);
  const int mz = max(Dz, 1), my = max(Dy, 1), mx = max(Dx, 1);
  Q = 2 * mx * my * mz;
  const int BIG = 0x3fffffff;
  const int incz = 2 * mx * my, incy = 2 * mx * mz, incx = 2 * my * mz;
  int Az = Dz ? mx * my : BIG, Ay = Dy ? mx * mz : BIG, Ax = Dx ? my * mz : BIG;
  const int stz = ip > i ? plane : -plane, sty = jp > j ? nx : -nx, stx = kp > k ? 1 : -1;
  int v = i * plane + j * nx + k;
  int prev = 0;
  const int steps = Dx + Dy + Dz;
  for (int s = 0; s < steps; ++s) {
    const int m = min(Az, min(Ay, Ax));
    if (m > prev) add(v, m - prev);
    prev = m;
    const bool bz = Az == m;
    const bool by = !bz && (Ay == m);
    const bool bx = !bz && !by;
    v += bz ? stz : (by ? sty : stx);
    Az += bz ? incz : 0;
    Ay += by ? incy : 0;
    Ax += bx ? incx : 0;
  }
  add(v, Q - prev);
}

// ---------------------------------------------------------------------------------------------
// Symmetric back-projection.  The path between voxels r and r' is the same set of segments in
// both directions, so each unordered pair is walked once with the weight of both ordered pairs:
//   w(r, r') = k [ (y_r . R(w)) (R(w) . S_r') + (y_r' . P R(w)) (P R(w) . S_r) ],
// w = (r - r') / |r - r'|, P R(w) = R(-w) = (-1)^l R(w).  Pass 1 (k_bp_weights, once per source,
// summed into Q) evaluates the weights on 64 x 64 tiles of the upper triangle in slot order; pass 2
// (k_bp_walk, once per gradient) walks every pair with w != 0 and adds -w * length to each voxel on
// the path, into a shared-memory copy of the whole gradient per CTA when it fits.
__host__ __device__ constexpr int l_of_c(int c) {
  int l = 0;
  while ((l + 1) * (l + 1) <= c) ++l;
  return l;
}

__device__ __forceinline__ void tri_tile(long long t, int& bd, int& bs) {
  bd = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) / 2.0);
  while ((long long)(bd + 1) * (bd + 2) / 2 <= t) ++bd;
  while ((long long)bd * (bd + 1) / 2 > t) --bd;
  bs = (int)(t - (long long)bd * (bd + 1) / 2);
}

template <int LA, typename T>
__global__ void __launch_bounds__(RTE_KT) k_bp_weights(BpArgs a) {
  constexpr int C = (LA + 1) * (LA + 1);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ys = reinterpret_cast<T*>(smem_raw);             // [64][C] y of the tile's sources
  T* Ss = ys + RTE_KT * C;                             // [64][C] S of the tile's sources
  int* sx = reinterpret_cast<int*>(Ss + RTE_KT * C);   // [64][3] source coordinates
  // FP32 sums at L >= 6: the destination's own y and S rows live in shared memory ([2][C][64], one
  // column per thread) instead of 2C registers, which leaves room for the FP64 SH recurrence at L >= 7
  // (the FP64 kernel keeps them in registers: in shared memory they would halve its CTAs per SM)
  constexpr bool DST_SMEM = C >= 49 && sizeof(T) == 4;
  T* sD = reinterpret_cast<T*>(sx + RTE_KT * 3);
  const int ntile = (a.N + RTE_KT - 1) / RTE_KT;
  int bd, bs;
  tri_tile(blockIdx.x, bd, bs);
  if (bd >= ntile) return;
  const int tid = threadIdx.x;
  const int plane = a.nx * a.ny;
  const int s0 = bs * RTE_KT, d0 = bd * RTE_KT;
  {
    const int sl = s0 + tid;
    const int v = sl < a.N ? a.perm[sl] : 0;
    sx[tid * 3 + 0] = v % a.nx;
    sx[tid * 3 + 1] = (v / a.nx) % a.ny;
    sx[tid * 3 + 2] = v / plane;
  }
  for (int e = tid; e < RTE_KT * C; e += RTE_KT) {  // row by row: neighbouring threads, neighbouring c
    const int q = e / C, c = e % C;
    const int sl = s0 + q;
    const size_t off = sl < a.N ? (size_t)a.perm[sl] * a.Cfull + c : 0;
    ys[e] = sl < a.N ? (T)a.y[off] : T(0);
    Ss[e] = sl < a.N ? (T)a.S[off] : T(0);
  }
  __syncthreads();
  const int d = d0 + tid;
  if (d >= a.N) return;
  const int r = a.perm[d];
  const int k = r % a.nx, j = (r / a.nx) % a.ny, i = r / plane;
  T yd[DST_SMEM ? 1 : C], Sd[DST_SMEM ? 1 : C];
#pragma unroll
  for (int c = 0; c < C; ++c) {
    const T yv = (T)a.y[(size_t)r * a.Cfull + c], Sv = (T)a.S[(size_t)r * a.Cfull + c];
    if constexpr (DST_SMEM) {
      sD[c * RTE_KT + tid] = yv;
      sD[(C + c) * RTE_KT + tid] = Sv;
    } else {
      yd[c] = yv;
      Sd[c] = Sv;
    }
  }
  const T dxf = (T)a.dx, dyf = (T)a.dy, dzf = (T)a.dz, thr = (T)a.prop_thresh, ks = (T)a.kscale;
  T* Qp = reinterpret_cast<T*>(a.Q);
  const int qend = bs == bd ? tid : RTE_KT;  // diagonal tile: each unordered pair once (source slot < destination slot)
  for (int q = 0; q < qend; ++q) {
    const int sl = s0 + q;
    if (sl >= a.N) break;
    const int kp = sx[q * 3 + 0], jp = sx[q * 3 + 1], ip = sx[q * 3 + 2];
    const T ddx = (T)(k - kp) * dxf, ddy = (T)(j - jp) * dyf, ddz = (T)(i - ip) * dzf;
    const T d2 = ddx * ddx + ddy * ddy + ddz * ddz;
    const T dist = sqrt(d2);
    T w = T(0);
    if (d2 > T(0) && dist < thr) {
      T kk;
      if (a.Kmat64) {
        kk = (T)__ldg(a.Kmat64 + (size_t)sl * a.Kld + d);
      } else if (a.Kmat) {
        kk = (T)__ldg(a.Kmat + kmat_index(sl, d, a.Kld));
      } else {
        int Q0;
        const T ps = path_sum<T, double>(i, j, k, ip, jp, kp, a.mut, a.nx, plane, Q0);
        kk = exp(-ps * dist / (T)Q0) * ks / d2;
      }
      const T inv = T(1) / dist;
      T R[C];
      sh_eval_prec<LA, T>(ddx * inv, ddy * inv, ddz * inv, R);
      const T* yq = ys + q * C;
      const T* Sq = Ss + q * C;
      T a1 = T(0), b1 = T(0), a2 = T(0), b2 = T(0);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const T Rp = (l_of_c(c) & 1) ? -R[c] : R[c];
        const T ydc = DST_SMEM ? sD[c * RTE_KT + tid] : yd[DST_SMEM ? 0 : c];
        const T Sdc = DST_SMEM ? sD[(C + c) * RTE_KT + tid] : Sd[DST_SMEM ? 0 : c];
        a1 = fma(ydc, R[c], a1);
        b1 = fma(R[c], Sq[c], b1);
        a2 = fma(yq[c], Rp, a2);
        b2 = fma(Rp, Sdc, b2);
      }
      w = kk * (a1 * b1 + a2 * b2);
    }
    const size_t idx = (size_t)sl * a.Kld + d;
    Qp[idx] = a.accumulate ? Qp[idx] + w : w;
  }
}

__device__ __forceinline__ void group_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

#define RTE_BPW_THREADS 512
template <typename T>
__global__ void __launch_bounds__(RTE_BPW_THREADS) k_bp_walk(BpArgs a) {
  constexpr int G = RTE_BPW_THREADS / RTE_KT;  // independent 64-thread groups, one tile each
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int* sx = reinterpret_cast<int*>(smem_raw);                          // [G][64][3]
  T* acc = reinterpret_cast<T*>(smem_raw + G * RTE_KT * 3 * sizeof(int));  // [N] when use_smem
  const int tid = threadIdx.x, grp = tid / RTE_KT, lane = tid % RTE_KT;
  if (a.use_smem)
    for (int v = tid; v < a.N; v += RTE_BPW_THREADS) acc[v] = T(0);
  __syncthreads();
  const int plane = a.nx * a.ny;
  const int ntile = (a.N + RTE_KT - 1) / RTE_KT;
  const long long ntri = (long long)ntile * (ntile + 1) / 2;
  const T* Qp = reinterpret_cast<const T*>(a.Q);
  int* gx = sx + grp * RTE_KT * 3;
  for (long long t = (long long)blockIdx.x * G + grp; t < ntri; t += (long long)gridDim.x * G) {
    int bd, bs;
    tri_tile(t, bd, bs);
    const int s0 = bs * RTE_KT, d0 = bd * RTE_KT;
    {
      const int sl = s0 + lane;
      const int v = sl < a.N ? a.perm[sl] : 0;
      gx[lane * 3 + 0] = v % a.nx;
      gx[lane * 3 + 1] = (v / a.nx) % a.ny;
      gx[lane * 3 + 2] = v / plane;
    }
    group_sync(grp + 1, RTE_KT);
    const int d = d0 + lane;
    if (d < a.N) {
      const int r = a.perm[d];
      const int k = r % a.nx, j = (r / a.nx) % a.ny, i = r / plane;
      const int qend = bs == bd ? lane : RTE_KT;
      for (int q = 0; q < qend; ++q) {
        const int sl = s0 + q;
        if (sl >= a.N) break;
        const T w = Qp[(size_t)sl * a.Kld + d];
        if (w == T(0)) continue;
        const int kp = gx[q * 3 + 0], jp = gx[q * 3 + 1], ip = gx[q * 3 + 2];
        const T ddx = (T)(k - kp) * (T)a.dx, ddy = (T)(j - jp) * (T)a.dy, ddz = (T)(i - ip) * (T)a.dz;
        const T dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
        const int Dz = abs(ip - i), Dy = abs(jp - j), Dx = abs(kp - k);
        // lengths arrive scaled by Q / dist, Q = 2 max(Dx,1) max(Dy,1) max(Dz,1)
        const T coef = -w * dist / (T)(2 * max(Dx, 1) * max(Dy, 1) * max(Dz, 1));
        int Qw = 1;
        if (a.use_smem)
          path_walk(i, j, k, ip, jp, kp, a.nx, plane, Qw, [&](int v, int len) { atomicAdd(acc + v, coef * (T)len); });
        else
          path_walk(i, j, k, ip, jp, kp, a.nx, plane, Qw,
                    [&](int v, int len) { atomicAdd(a.g + v, (double)(coef * (T)len)); });
      }
    }
    group_sync(grp + 1, RTE_KT);  // the group's coordinates are overwritten by its next tile
  }
  if (a.use_smem) {
    __syncthreads();
    for (int v = tid; v < a.N; v += RTE_BPW_THREADS) {
      const T x = acc[v];
      if (x != T(0)) atomicAdd(a.g + v, (double)x);
    }
  }
}

// Per-voxel parts of the gradient: the scatter D (d/dmu_s: lambda . scat_l . (A S)) and the
// self-voxel term (d/dmu_t: (dV/cm) y . dDself/dmu S).
__global__ void k_grad_local(GradLocalArgs a) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.N) return;
  const size_t b = (size_t)r * a.Cfull;
  double gs = 0.0;
  for (int c = 0; c < a.Cact; ++c) {
    int l = 0;
    while ((l + 1) * (l + 1) <= c) ++l;
    gs = fma(a.lam[b + c] * a.scat[l], a.out[b + c], gs);
  }
  a.gs[r] += gs;
  const double mu = a.mut[r];
  if (a.air_no_self && mu == 0.0) return;
  double gt = 0.0;
  for (int c = 0; c < a.Cact; ++c) {
    double u = 0.0;
    if (a.idx) {
      const double* D = a.dlut + ((size_t)a.idx[r] * a.Cfull + c) * a.Cfull;
      for (int cp = 0; cp < a.Cact; ++cp) u = fma(D[cp], a.S[b + cp], u);
    } else {
      // d/dmu sum_k mu^k M_k = sum_{k>=1} k mu^(k-1) M_k
      for (int kk = a.K - 1; kk >= 1; --kk) {
        const double* M = a.mom + ((size_t)kk * a.Cfull + c) * a.Cfull;
        double t = 0.0;
        for (int cp = 0; cp < a.Cact; ++cp) t = fma(M[cp], a.S[b + cp], t);
        u = fma(mu, u, (double)kk * t);
      }
    }
    gt = fma(a.y[b + c], u, gt);
  }
  a.gt[r] += a.scale * gt;
}

// Complex reference basis <-> real basis.  w = w1 + i w2 with w1, w2 the coefficient sets of
// real functions (w_{l,-m} = (-1)^m conj(w_{l,m})).  u_l0 = Re(w_l0), u_l,m = sqrt2 Re(w_lm),
// u_l,-m = -sqrt2 Im(w_lm) (m > 0).  red[0] accumulates ||u2||^2.
__global__ void k_to_real(const double* __restrict__ w, double* u1, double* u2, int N, int L, double* red,
                          int ostride) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  double n2 = 0.0;
  if (r < N) {
    const int C = (L + 1) * (L + 1);
    // u1/u2 rows are ostride apart (a complex right-hand side's real and imaginary rows interleaved)
    u1 += (size_t)r * ostride - (size_t)r * C;
    if (u2) u2 += (size_t)r * ostride - (size_t)r * C;
    const double s2 = 1.4142135623730951;
    for (int l = 0; l <= L; ++l) {
      const int c0 = l * l + l;
      const double re0 = w[2 * ((size_t)r * C + c0)], im0 = w[2 * ((size_t)r * C + c0) + 1];
      u1[(size_t)r * C + c0] = re0;
      if (u2) u2[(size_t)r * C + c0] = im0;
      n2 += im0 * im0;
      for (int m = 1; m <= l; ++m) {
        const double sg = (m & 1) ? -1.0 : 1.0;
        const size_t ip = (size_t)r * C + c0 + m, in = (size_t)r * C + c0 - m;
        const double rp = w[2 * ip], mp = w[2 * ip + 1], rn = w[2 * in], mn = w[2 * in + 1];
        // w1 = (w + P w)/2, P w_lm = (-1)^m conj(w_l,-m)
        const double r1 = 0.5 * (rp + sg * rn), i1 = 0.5 * (mp - sg * mn);
        // w2 = (w - P w)/(2i)
        const double dr = rp - sg * rn, di = mp + sg * mn;
        const double r2 = 0.5 * di, i2 = -0.5 * dr;
        u1[ip] = s2 * r1;
        u1[in] = -s2 * i1;
        if (u2) {
          u2[ip] = s2 * r2;
          u2[in] = -s2 * i2;
        }
        n2 += r2 * r2 + i2 * i2;
      }
    }
  }
  if (red) {
    for (int o = 16; o > 0; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    if ((threadIdx.x & 31) == 0 && n2 != 0.0) atomicAdd(red, n2);
  }
}

__global__ void k_to_cplx(const double* __restrict__ u1, const double* __restrict__ u2, double* w, int N, int L,
                          int ustride) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= N) return;
  const int C = (L + 1) * (L + 1);
  // u1/u2 rows are ustride apart (several right-hand sides interleaved); w rows are C apart
  u1 += (size_t)r * ustride - (size_t)r * C;
  if (u2) u2 += (size_t)r * ustride - (size_t)r * C;
  const double is2 = 0.70710678118654752;
  for (int l = 0; l <= L; ++l) {
    const int c0 = l * l + l;
    const size_t i0 = (size_t)r * C + c0;
    // w = w1 + i w2
    w[2 * i0] = u1[i0];
    w[2 * i0 + 1] = u2 ? u2[i0] : 0.0;
    for (int m = 1; m <= l; ++m) {
      const double sg = (m & 1) ? -1.0 : 1.0;
      const size_t ip = i0 + m, in = i0 - m;
      // w1_lm = (a - i b)/sqrt2, w1_l,-m = (-1)^m (a + i b)/sqrt2 with a = u_l,m, b = u_l,-m
      const double a1 = u1[ip], b1 = u1[in];
      double wr_p = a1 * is2, wi_p = -b1 * is2, wr_n = sg * a1 * is2, wi_n = sg * b1 * is2;
      if (u2) {
        const double a2 = u2[ip], b2 = u2[in];
        // + i * w2: i(a2 - i b2)/sqrt2 = (b2 + i a2)/sqrt2 ; i * (-1)^m (a2 + i b2)/sqrt2 = (-1)^m(-b2 + i a2)/sqrt2
        wr_p += b2 * is2;
        wi_p += a2 * is2;
        wr_n += -sg * b2 * is2;
        wi_n += sg * a2 * is2;
      }
      w[2 * ip] = wr_p;
      w[2 * ip + 1] = wi_p;
      w[2 * in] = wr_n;
      w[2 * in + 1] = wi_n;
    }
  }
}

// Stop-rule sums of the layer z = nZ-1 (FisherInfo_IO/src/dist.cu:1143-1152) in the real basis;
// cplx: (real, imaginary) row pairs per voxel.
__global__ void k_layer_sums(const double* W, const double* S, int N, int nx, int ny, int nz, int Cfull,
                             double* red, int cplx) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  double lw = 0.0, ls = 0.0;
  const int np = cplx ? 2 : 1;
  if (p < nx * ny) {
    const size_t r = (size_t)(nz - 1) * nx * ny + p;
    for (int q = 0; q < np; ++q)
      for (int c = 0; c < Cfull; ++c) {
        const double wgt = stop_weight(c, q == 1);
        const size_t e = (r * np + q) * Cfull + c;
        lw += wgt * W[e];
        ls += wgt * S[e];
      }
  }
  for (int o = 16; o > 0; o >>= 1) {
    lw += __shfl_xor_sync(0xffffffffu, lw, o);
    ls += __shfl_xor_sync(0xffffffffu, ls, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(red + 2, lw);
    atomicAdd(red + 3, ls);
  }
}

__global__ void k_to_f32_slots(const double* a, float* b, const int* islot, int N, int vstride, int cpad,
                               int Cfull, int cstride) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)N * vstride) return;
  const int r = (int)(t / vstride), e = (int)(t % vstride);
  const int rhs = e / Cfull, c = e - rhs * Cfull;
  b[(size_t)islot[r] * cpad + (size_t)rhs * cstride + c] = (float)(a[t] * kMonic.N[c]);  // N_c W_c, see sh_eval_monic
}

__global__ void k_f64_to_f32(const double* a, float* b, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// ---------------------------------------------------------------------------------------------
// launchers

// Dynamic shared memory above 48 KB for a kernel: the attribute is set to the device's opt-in maximum,
// the same value from every host thread, not to one launch's size.  The size a launch needs can depend
// on the context (the lower-order passes of a pair kernel size their source rows by the context's own
// order), and the server launches the same instantiation from several worker threads; per-launch values
// let one thread lower the limit between another thread's set and launch, which fails that launch with
// an invalid-argument error.  Each launch still asks for its own size.
static cudaError_t allow_smem(const void* kern, size_t smem) {
  int dev = 0, cap = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (smem > (size_t)cap) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

template <int LA, bool TABLE, bool STORED, int NB, bool CPLX = false>
static cudaError_t launch_mixed(const PairArgs& a, cudaStream_t st, int* occ) {
  if constexpr (!STORED && !TABLE && !CPLX && NB == 4 && LA >= 6) {  // shared walks, two groups of two
    const size_t smem = GrpLayout(a.cpad, RTE_GRP_TS).bytes;
    void (*kern)(PairArgs) = k_pair_mixed_grp<LA>;
    cudaError_t e = allow_smem((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, RTE_GRP_THREADS, smem);
    dim3 grid((a.N + RTE_KBLK - 1) / RTE_KBLK, a.nsplit);
    kern<<<grid, RTE_GRP_THREADS, smem, st>>>(a);
    return cudaGetLastError();
  }
  if constexpr (STORED && !TABLE && !CPLX) {  // K tiles staged with the source rows, 32 or 64 sources a tile
    const int ts = a.tile ? 64 : 32;
    const size_t smem = TkLayout(a.cpad, ts).bytes;
    void (*kern)(PairArgs) = a.tile ? k_pair_mixed_tk<LA, NB, 64> : k_pair_mixed_tk<LA, NB, 32>;
    cudaError_t e = allow_smem((const void*)kern, smem);
    if (e != cudaSuccess) return e;
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, RTE_PAIR_THREADS, smem);
    dim3 grid((a.N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS, a.nsplit);
    kern<<<grid, RTE_PAIR_THREADS, smem, st>>>(a);
    return cudaGetLastError();
  }
  const size_t smem = MixedLayout(a.cpad, NB * (LA + 1) * (LA + 1), NB * (LA + 1) * (LA + 1) >= 128 ? 32 : RTE_PAIR_TS).bytes;
  void (*kern)(PairArgs);
  if constexpr (LA == 7 && NB == 1)
    kern = k_pair_mixed_3<LA, TABLE, STORED, NB, CPLX>;
  else
    kern = k_pair_mixed<LA, TABLE, STORED, NB, CPLX>;
  cudaError_t e = allow_smem((const void*)kern, smem);
  if (e != cudaSuccess) return e;
  if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, RTE_PAIR_THREADS, smem);
  dim3 grid((a.N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS, a.nsplit);
  kern<<<grid, RTE_PAIR_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

template <int LA, int NB>
static cudaError_t launch_mixed_nb(const PairArgs& a, int table, int stored, cudaStream_t st, int* occ) {
  if (table)
    return stored ? launch_mixed<LA, true, true, NB>(a, st, occ) : launch_mixed<LA, true, false, NB>(a, st, occ);
  return stored ? launch_mixed<LA, false, true, NB>(a, st, occ) : launch_mixed<LA, false, false, NB>(a, st, occ);
}

template <int LA>
static cudaError_t launch_pair_LA(const PairArgs& a, int precision, int table, int stored, int nb, cudaStream_t st,
                                  int* occ) {
  if (a.kappa != 0.0) {  // one complex right-hand side (exact SH only)
    if (table || nb != 2) return cudaErrorInvalidValue;
    if (precision == 0) {
      void (*kern)(PairArgs) = stored ? k_pair_fp64<LA, false, true, true> : k_pair_fp64<LA, false, true>;
      if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, RTE_PAIR_THREADS, 0);
      dim3 grid((a.N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS, a.nsplit);
      kern<<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
      return cudaGetLastError();
    }
    return stored ? launch_mixed<LA, false, true, 2, true>(a, st, occ) : launch_mixed<LA, false, false, 2, true>(a, st, occ);
  }
  if (precision == 0) {
    void (*kern)(PairArgs) = stored ? (table ? k_pair_fp64<LA, true, false, true> : k_pair_fp64<LA, false, false, true>)
                                    : (table ? k_pair_fp64<LA, true, false> : k_pair_fp64<LA, false, false>);
    if (occ) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, RTE_PAIR_THREADS, 0);
    dim3 grid((a.N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS, a.nsplit);
    kern<<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
    return cudaGetLastError();
  }
  switch (nb) {
    case 1: return launch_mixed_nb<LA, 1>(a, table, stored, st, occ);
    case 2: return launch_mixed_nb<LA, 2>(a, table, stored, st, occ);
    case 4: return launch_mixed_nb<LA, 4>(a, table, stored, st, occ);
  }
  return cudaErrorInvalidValue;
}

static cudaError_t pair_dispatch(const PairArgs& a, int LA, int precision, int table, int stored, int nb,
                                 cudaStream_t st, int* occ) {
  switch (LA) {
    case 0: return launch_pair_LA<0>(a, precision, table, stored, nb, st, occ);
    case 1: return launch_pair_LA<1>(a, precision, table, stored, nb, st, occ);
    case 2: return launch_pair_LA<2>(a, precision, table, stored, nb, st, occ);
    case 3: return launch_pair_LA<3>(a, precision, table, stored, nb, st, occ);
    case 4: return launch_pair_LA<4>(a, precision, table, stored, nb, st, occ);
    case 5: return launch_pair_LA<5>(a, precision, table, stored, nb, st, occ);
    case 6: return launch_pair_LA<6>(a, precision, table, stored, nb, st, occ);
    case 7: return launch_pair_LA<7>(a, precision, table, stored, nb, st, occ);
  }
  return cudaErrorInvalidValue;
}

cudaError_t rte_launch_pair(const PairArgs& a, int LA, int precision, int table, int stored, cudaStream_t st) {
  return pair_dispatch(a, LA, precision, table, stored, a.nb > 0 ? a.nb : 1, st, nullptr);
}

cudaError_t rte_pair_occupancy(int LA, int precision, int table, int stored, int nb, int cpad, int* blocks_per_sm,
                               int cplx, int tile) {
  PairArgs dummy;
  memset(&dummy, 0, sizeof dummy);
  dummy.cpad = cpad;
  dummy.kappa = cplx ? 1.0 : 0.0;
  dummy.tile = tile;
  return pair_dispatch(dummy, LA, precision, table, stored, nb, nullptr, blocks_per_sm);
}

cudaError_t rte_launch_store_kernel(const PairArgs& a, cudaStream_t st, int fp64) {
  const long long nt = (a.N + RTE_KT - 1) / RTE_KT;
  if (fp64)
    k_store_kernel<double><<<(unsigned)(nt * (nt + 1) / 2), RTE_KT, 0, st>>>(a);
  else
    k_store_kernel<float><<<(unsigned)(nt * (nt + 1) / 2), RTE_KT, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_epilogue(const EpiArgs& a, int LA, cudaStream_t st) {
  if (LA < 0 || LA > RTE_MAX_L) return cudaErrorInvalidValue;
  const size_t total = (size_t)a.N * (a.nb > 0 ? a.nb : 1) * a.Cfull;
  const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
  k_epilogue<<<blocks, 256, 0, st>>>(a, (LA + 1) * (LA + 1));
  return cudaGetLastError();
}

cudaError_t rte_launch_self(const SelfArgs& a, cudaStream_t st) {
  if (a.kappa != 0.0) {
    if (a.nb % 2 || a.dmut) return cudaErrorInvalidValue;
    const long long total = (long long)a.N * (a.nb / 2) * a.Cact;
    k_self_cplx<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a);
    return cudaGetLastError();
  }
  const long long total = (long long)a.N * a.nb * a.Cact;
  k_self<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_images(const ImgArgs& a, cudaStream_t st) {
  const int n = a.nx * a.ny;
  k_images<<<(n + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_to_real(const double* cplx, double* u1, double* u2, int N, int L, double* red,
                               cudaStream_t st, int ostride) {
  const int C = (L + 1) * (L + 1);
  k_to_real<<<(N + 127) / 128, 128, 0, st>>>(cplx, u1, u2, N, L, red, ostride > 0 ? ostride : C);
  return cudaGetLastError();
}

cudaError_t rte_launch_to_cplx(const double* u1, const double* u2, double* cplx, int N, int L, cudaStream_t st,
                               int ustride) {
  const int C = (L + 1) * (L + 1);
  k_to_cplx<<<(N + 127) / 128, 128, 0, st>>>(u1, u2, cplx, N, L, ustride > 0 ? ustride : C);
  return cudaGetLastError();
}

cudaError_t rte_launch_layer_sums(const double* W, const double* S, int N, int nx, int ny, int nz, int Cfull,
                                  double* red, cudaStream_t st, int cplx) {
  const int n = nx * ny;
  k_layer_sums<<<(n + 127) / 128, 128, 0, st>>>(W, S, N, nx, ny, nz, Cfull, red, cplx);
  return cudaGetLastError();
}

cudaError_t rte_launch_source(const SrcArgs& a, cudaStream_t st) {
  k_source<<<(a.ncols + 31) / 32, 32, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_medium(const double* mua, const double* mus, double* mut, double* mus_out, float* mutf,
                              int N, double* red_max, cudaStream_t st) {
  k_medium<<<(N + 127) / 128, 128, 0, st>>>(mua, mus, mut, mus_out, mutf, N, red_max);
  return cudaGetLastError();
}

cudaError_t rte_launch_fma_peak(int fp64, int iters, float* sink, cudaStream_t st, int blocks) {
  if (fp64 == 3)
    k_fma2_fresh_peak<<<blocks, 256, 0, st>>>(iters, sink);
  else if (fp64 == 2)
    k_fma2_peak<<<blocks, 256, 0, st>>>(iters, sink);
  else if (fp64)
    k_fma_peak<double><<<blocks, 256, 0, st>>>(iters, sink);
  else
    k_fma_peak<float><<<blocks, 256, 0, st>>>(iters, sink);
  return cudaGetLastError();
}

cudaError_t rte_launch_to_f32_slots(const double* a, float* b, const int* islot, int N, int vstride, int cpad,
                                    int Cfull, int cstride, cudaStream_t st) {
  const long long n = (long long)N * vstride;
  k_to_f32_slots<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, islot, N, vstride, cpad, Cfull, cstride);
  return cudaGetLastError();
}

cudaError_t rte_launch_f64_to_f32(const double* a, float* b, size_t n, cudaStream_t st) {
  k_f64_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a, b, n);
  return cudaGetLastError();
}

cudaError_t rte_launch_face_flux(const FaceArgs& a, cudaStream_t st) {
  const int total = 2 * (a.nx * a.ny + a.nz * a.nx + a.nz * a.ny);
  k_face_flux<<<(total + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_adjoint_seed(const FaceArgs& a, cudaStream_t st) {
  const int total = 2 * (a.nx * a.ny + a.nz * a.nx + a.nz * a.ny);
  k_adjoint_seed<<<(total + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

template <int LA>
static cudaError_t launch_tangent_LA(const PairArgs& a, int fp64, int table, cudaStream_t st) {
  dim3 grid((a.N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS, a.nsplit);
  if (fp64) {
    if (table)
      k_pair_tangent<LA, true, double><<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
    else
      k_pair_tangent<LA, false, double><<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
  } else {
    if (table)
      k_pair_tangent<LA, true, float><<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
    else
      k_pair_tangent<LA, false, float><<<grid, RTE_PAIR_THREADS, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t rte_launch_pair_tangent(const PairArgs& a, int LA, int fp64, int table, cudaStream_t st) {
  switch (LA) {
    case 0: return launch_tangent_LA<0>(a, fp64, table, st);
    case 1: return launch_tangent_LA<1>(a, fp64, table, st);
    case 2: return launch_tangent_LA<2>(a, fp64, table, st);
    case 3: return launch_tangent_LA<3>(a, fp64, table, st);
    case 4: return launch_tangent_LA<4>(a, fp64, table, st);
    case 5: return launch_tangent_LA<5>(a, fp64, table, st);
    case 6: return launch_tangent_LA<6>(a, fp64, table, st);
    case 7: return launch_tangent_LA<7>(a, fp64, table, st);
  }
  return cudaErrorInvalidValue;
}

cudaError_t rte_launch_tangent_rhs(double* q, int qstride, const double* T, const double* out, const double* mus,
                                   const double* dmus, const double* scat, int N, int L, cudaStream_t st) {
  ScatTab sc;
  for (int l = 0; l <= RTE_MAX_L; ++l) sc.v[l] = l <= L ? scat[l] : 0.0;
  const long long n = (long long)N * (L + 1) * (L + 1);
  k_tangent_rhs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(q, qstride, T, out, mus, dmus, sc, N, L);
  return cudaGetLastError();
}

cudaError_t rte_launch_scatter_add(double* dst, int dstride, const int* idx, const double* vals, int n, int C,
                                   cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_scatter_add<<<(n * C + 255) / 256, 256, 0, st>>>(dst, dstride, idx, vals, n, C);
  return cudaGetLastError();
}

cudaError_t rte_launch_strided_add(double* dst, const double* a, int astride, const double* b, int N, int C,
                                   cudaStream_t st) {
  const long long n = (long long)N * C;
  k_strided_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, a, astride, b, N, C);
  return cudaGetLastError();
}

cudaError_t rte_launch_masked_scale(const double* in, double* out, const uint8_t* mask, const double* fac, int N,
                                    int L, cudaStream_t st) {
  ScatTab f;
  for (int l = 0; l <= RTE_MAX_L; ++l) f.v[l] = l <= L ? fac[l] : 0.0;
  const long long n = (long long)N * (L + 1) * (L + 1);
  k_masked_scale<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(in, out, mask, f, N, L);
  return cudaGetLastError();
}

cudaError_t rte_launch_parity(double* x, int N, int L, int vstride, cudaStream_t st) {
  const long long n = (long long)N * (L + 1) * (L + 1);
  k_parity<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, N, L, vstride);
  return cudaGetLastError();
}

cudaError_t rte_launch_tangent_pair_dots(const double* lam, const double* out, const double* fa, const double* fs, int N,
                                         int L, double* ga, double* gs, cudaStream_t st) {
  ScatTab a, b;
  for (int l = 0; l <= RTE_MAX_L; ++l) {
    a.v[l] = l <= L ? fa[l] : 0.0;
    b.v[l] = l <= L ? fs[l] : 0.0;
  }
  k_tangent_pair_dots<<<(N + 127) / 128, 128, 0, st>>>(lam, out, a, b, N, L, ga, gs);
  return cudaGetLastError();
}

cudaError_t rte_launch_axpy(double* y, const double* x, double alpha, size_t n, cudaStream_t st) {
  k_axpy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(y, x, alpha, n);
  return cudaGetLastError();
}

cudaError_t rte_launch_y_field(double* y, const double* e, const double* lam, const double* mus, const double* scat,
                               int N, int L, int Cfull, cudaStream_t st) {
  ScatTab sc;
  for (int l = 0; l <= RTE_MAX_L; ++l) sc.v[l] = scat[l];
  const long long n = (long long)N * Cfull;
  k_y_field<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(y, e, lam, mus, sc, N, L, Cfull);
  return cudaGetLastError();
}

template <int LA, typename T>
static cudaError_t launch_bpw(const BpArgs& a, cudaStream_t st) {
  constexpr int C = (LA + 1) * (LA + 1);
  const size_t smem = (size_t)RTE_KT * C * 2 * sizeof(T) * (C >= 49 && sizeof(T) == 4 ? 2 : 1) + RTE_KT * 3 * sizeof(int);
  cudaError_t e = allow_smem((const void*)k_bp_weights<LA, T>, smem);
  if (e != cudaSuccess) return e;
  const long long nt = (a.N + RTE_KT - 1) / RTE_KT;
  k_bp_weights<LA, T><<<(unsigned)(nt * (nt + 1) / 2), RTE_KT, smem, st>>>(a);
  return cudaGetLastError();
}

template <int LA>
static cudaError_t launch_bpw_LA(const BpArgs& a, int fp64, cudaStream_t st) {
  return fp64 ? launch_bpw<LA, double>(a, st) : launch_bpw<LA, float>(a, st);
}

cudaError_t rte_launch_bp_weights(const BpArgs& a, int LA, int fp64, cudaStream_t st) {
  switch (LA) {
    case 0: return launch_bpw_LA<0>(a, fp64, st);
    case 1: return launch_bpw_LA<1>(a, fp64, st);
    case 2: return launch_bpw_LA<2>(a, fp64, st);
    case 3: return launch_bpw_LA<3>(a, fp64, st);
    case 4: return launch_bpw_LA<4>(a, fp64, st);
    case 5: return launch_bpw_LA<5>(a, fp64, st);
    case 6: return launch_bpw_LA<6>(a, fp64, st);
    case 7: return launch_bpw_LA<7>(a, fp64, st);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
static cudaError_t launch_walk(BpArgs a, cudaStream_t st) {
  const size_t base = (size_t)(RTE_BPW_THREADS / RTE_KT) * RTE_KT * 3 * sizeof(int);
  int dev = 0, maxsm = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  a.use_smem = base + (size_t)a.N * sizeof(T) <= (size_t)maxsm ? 1 : 0;
  const size_t smem = base + (a.use_smem ? (size_t)a.N * sizeof(T) : 0);
  cudaError_t e = allow_smem((const void*)k_bp_walk<T>, smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bp_walk<T>, RTE_BPW_THREADS, smem);
  if (e != cudaSuccess) return e;
  k_bp_walk<T><<<(unsigned)(std::max(per_sm, 1) * sms), RTE_BPW_THREADS, smem, st>>>(a);
  return cudaGetLastError();
}

cudaError_t rte_launch_bp_walk(const BpArgs& a, int fp64, cudaStream_t st) {
  return fp64 ? launch_walk<double>(a, st) : launch_walk<float>(a, st);
}

cudaError_t rte_launch_grad_local(const GradLocalArgs& a, cudaStream_t st) {
  k_grad_local<<<(a.N + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------
// Uniform medium: the off-diagonal operator as a convolution over displacements (host side and the
// transforms in rte_fft.cpp).  k_fft_table samples T_cc'(d) = k(d) R_c(d) R_c'(d) on the padded
// grid, k_fft_pad / k_fft_crop move fields in and out of it, k_fft_product forms the spectral
// products.
// T_cc'(d) for c <= c' (pair p in row-major upper-triangle order) on the padded grid; the padded
// index g maps to the displacement g (g < n), g - M (g > n) or none (g == n).
template <int LA, bool TABLE>
__global__ void k_fft_table(FftTabArgs a, double* T, size_t M) {
  constexpr int C = (LA + 1) * (LA + 1);
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const int gx = (int)(t % a.Mx), gy = (int)((t / a.Mx) % a.My), gz = (int)(t / ((size_t)a.Mx * a.My));
  auto disp = [](int g, int n, int Mg, bool& ok) {
    if (g < n) return g;
    if (g > Mg - n) return g - Mg;
    ok = false;
    return 0;
  };
  bool ok = true;
  const int ix = disp(gx, a.nx, a.Mx, ok), iy = disp(gy, a.ny, a.My, ok), iz = disp(gz, a.nz, a.Mz, ok);
  const double ddx = ix * a.dx, ddy = iy * a.dy, ddz = iz * a.dz;
  const double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
  const double dist = sqrt(d2);
  ok = ok && d2 > 0.0 && dist < a.prop_thresh;
  double R[C];
  double k = 0.0;
  if (ok) {
    k = exp(-a.mut * dist) * a.kscale / d2;
    double ux, uy, uz;
    if (TABLE) {
      table_direction(ddx, ddy, ddz, dist, ux, uy, uz);
    } else {
      ux = ddx / dist;
      uy = ddy / dist;
      uz = ddz / dist;
    }
    sh_eval<LA, double>(ux, uy, uz, R);
  }
  int p = 0;
#pragma unroll 1
  for (int c = 0; c < C; ++c)
#pragma unroll 1
    for (int cp = c; cp < C; ++cp, ++p)
      if (p >= a.p0 && p < a.p1) T[(size_t)(p - a.p0) * M + t] = ok ? k * R[c] * R[cp] : 0.0;
}

// W [N][vstride] (coefficient c of right-hand side b at b*Cfull + c) -> padded fields F[b*Cact + c][M]
__global__ void k_fft_pad(const double* W, int vstride, int Cfull, int Cact, int nb, FftTabArgs a, double* F,
                          size_t M) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = (long long)a.nx * a.ny * a.nz;
  if (t >= N * nb * Cact) return;
  const int c = (int)(t % Cact);
  const int b = (int)((t / Cact) % nb);
  const long long r = t / ((long long)Cact * nb);
  const int x = (int)(r % a.nx), y = (int)((r / a.nx) % a.ny), z = (int)(r / ((long long)a.nx * a.ny));
  F[(size_t)(b * Cact + c) * M + ((size_t)z * a.My + y) * a.Mx + x] = W[(size_t)r * vstride + (size_t)b * Cfull + c];
}

// Spectral products O_c(k) = sum_c' That_cc'(k) W_c'(k).  T_cc'(-d) = (-1)^(l+l') T_cc'(d), so each
// table spectrum is real (l + l' even) or imaginary (odd): the table holds one real number tau per
// pair and frequency (That = tau or i tau), c <= c' in row-major upper-triangle order of the full
// order.  The complex products then split into two real systems over the coefficients,
//   set 0: inputs (Re W_even, Im W_odd) -> outputs (Re O_even, Im O_odd),
//   set 1: inputs (Im W_even, Re W_odd) -> outputs (Im O_even, Re O_odd),
// with sign -1 on the even<-odd terms of set 0 and the odd<-even terms of set 1 (i * i = -1).
__device__ __forceinline__ double fft_sign(int set, bool c_even, bool cp_even) {
  if (c_even == cp_even) return 1.0;
  return (set == 0) == c_even ? -1.0 : 1.0;
}

// The two real systems of a frequency run on adjacent lanes (set = lane parity), so the pair's table
// loads are one memory transaction and the table spectrum (larger than L2 at benchmark sizes) streams
// from HBM once per right-hand side instead of once per set.  Three CTAs per SM (168 registers, a small
// spill) keep more table loads in flight than two at 255 registers: 33^3 L=5 uniform solve 23.6 -> 22.5
// ms (four CTAs: 22.4 ms with a 3 KB spill).
template <int LA>
__global__ void __launch_bounds__(128, 3) k_fft_product_reg(const double* tau, const double2* Wh, double2* Oh, int C,
                                                         int nb, size_t Mk) {
  constexpr int CA = (LA + 1) * (LA + 1);
  __shared__ double sv[CA][128];  // this thread's inputs of its set (column tid)
  const int tid = threadIdx.x;
  const size_t g = (size_t)blockIdx.x * blockDim.x + tid;
  const size_t k = g >> 1;
  const int set = (int)(g & 1);
  const bool act = k < Mk;
  double* Ohd = reinterpret_cast<double*>(Oh);
  for (int b = 0; b < nb; ++b) {
    {
      double q[CA];
#pragma unroll
      for (int c = 0; c < CA; ++c) {
        const bool ev = !(l_of_c(c) & 1);
        const double2 w = act ? Wh[(size_t)(b * CA + c) * Mk + k] : make_double2(0.0, 0.0);
        sv[c][tid] = ((set == 0) == ev) ? w.x : w.y;
        q[c] = 0.0;
      }
      if (act) {
#pragma unroll
        for (int c = 0; c < CA; ++c) {
          const size_t row = (size_t)c * C - (size_t)c * (c - 1) / 2;
          const double vc = sv[c][tid];
#pragma unroll
          for (int cp = c; cp < CA; ++cp) {
            const double t = __ldg(tau + (row + (cp - c)) * Mk + k);
            const bool ec = !(l_of_c(c) & 1), ecp = !(l_of_c(cp) & 1);
            q[c] = fma(fft_sign(set, ec, ecp) * t, sv[cp][tid], q[c]);
            if (cp != c) q[cp] = fma(fft_sign(set, ecp, ec) * t, vc, q[cp]);
          }
        }
#pragma unroll
        for (int c = 0; c < CA; ++c) {
          const bool ev = !(l_of_c(c) & 1);
          Ohd[2 * ((size_t)(b * CA + c) * Mk + k) + (((set == 0) == ev) ? 0 : 1)] = q[c];
        }
      }
    }
  }
}

// any order: coefficients indexed at run time, table entries read once per output coefficient
__global__ void k_fft_product(const double* tau, const double2* Wh, double2* Oh, int C, int Cact, int nb,
                              size_t Mk) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Mk) return;
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < Cact; ++c) {
      const bool ec = !(l_of_c(c) & 1);
      double ox = 0.0, oy = 0.0;
      for (int cp = 0; cp < Cact; ++cp) {
        const int lo = min(c, cp), hi = max(c, cp);
        const double t = tau[((size_t)lo * C - (size_t)lo * (lo - 1) / 2 + (hi - lo)) * Mk + k];
        const double2 w = Wh[(size_t)(b * Cact + cp) * Mk + k];
        if (ec == !(l_of_c(cp) & 1)) {  // real spectrum
          ox = fma(t, w.x, ox);
          oy = fma(t, w.y, oy);
        } else {  // i tau
          ox = fma(-t, w.y, ox);
          oy = fma(t, w.x, oy);
        }
      }
      Oh[(size_t)(b * Cact + c) * Mk + k] = make_double2(ox, oy);
    }
}

// The FIM model snaps directions to its SH table, which breaks the parity of T_cc'; its table keeps
// complex spectra and this product reads them directly.
__global__ void k_fft_product_cplx(const double2* That, const double2* Wh, double2* Oh, int C, int Cact, int nb,
                                   size_t Mk) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Mk) return;
  for (int b = 0; b < nb; ++b)
    for (int c = 0; c < Cact; ++c) {
      double ox = 0.0, oy = 0.0;
      for (int cp = 0; cp < Cact; ++cp) {
        const int lo = min(c, cp), hi = max(c, cp);
        const double2 t = That[((size_t)lo * C - (size_t)lo * (lo - 1) / 2 + (hi - lo)) * Mk + k];
        const double2 w = Wh[(size_t)(b * Cact + cp) * Mk + k];
        ox = fma(t.x, w.x, fma(-t.y, w.y, ox));
        oy = fma(t.x, w.y, fma(t.y, w.x, oy));
      }
      Oh[(size_t)(b * Cact + c) * Mk + k] = make_double2(ox, oy);
    }
}

// tau[p][k] = Re or Im of the table spectrum of pair p (by the parity of l + l')
__global__ void k_fft_extract(const double2* spec, double* tau, int p0, int np, int C, size_t Mk) {
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (size_t)np * Mk) return;
  const int q = (int)(t / Mk);
  int p = p0 + q, c = 0;
  while (p >= C - c) {  // row c of the upper triangle holds C - c pairs
    p -= C - c;
    ++c;
  }
  const int cp = c + p;
  const double2 v = spec[t];
  tau[(size_t)p0 * Mk + t] = ((l_of_c(c) + l_of_c(cp)) & 1) ? v.y : v.x;
}

// padded result fields -> split-K partial layout [N][nb][Cfull] (one split), scaled by 1/M
__global__ void k_fft_crop(const double* F, int Cfull, int Cact, int nb, FftTabArgs a, double* part, size_t M) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long N = (long long)a.nx * a.ny * a.nz;
  if (t >= N * nb * Cact) return;
  const int c = (int)(t % Cact);
  const int b = (int)((t / Cact) % nb);
  const long long r = t / ((long long)Cact * nb);
  const int x = (int)(r % a.nx), y = (int)((r / a.nx) % a.ny), z = (int)(r / ((long long)a.nx * a.ny));
  part[(size_t)r * nb * Cfull + (size_t)b * Cfull + c] =
      F[(size_t)(b * Cact + c) * M + ((size_t)z * a.My + y) * a.Mx + x] / (double)M;
}


cudaError_t rte_launch_fft_table(const FftTabArgs& a, int L, int table, double* T, size_t M, cudaStream_t st) {
  const unsigned blocks = (unsigned)((M + 127) / 128);
  switch (L) {
#define RTE_FFT_TAB(LL)                                          \
  case LL:                                                       \
    if (table)                                                   \
      k_fft_table<LL, true><<<blocks, 128, 0, st>>>(a, T, M);    \
    else                                                         \
      k_fft_table<LL, false><<<blocks, 128, 0, st>>>(a, T, M);   \
    break;
    RTE_FFT_TAB(0) RTE_FFT_TAB(1) RTE_FFT_TAB(2) RTE_FFT_TAB(3) RTE_FFT_TAB(4) RTE_FFT_TAB(5) RTE_FFT_TAB(6)
    RTE_FFT_TAB(7)
#undef RTE_FFT_TAB
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t rte_launch_fft_pad(const double* W, int vstride, int Cfull, int Cact, int nb, const FftTabArgs& a, double* F,
                               size_t M, cudaStream_t st) {
  const long long n = (long long)a.nx * a.ny * a.nz * nb * Cact;
  k_fft_pad<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(W, vstride, Cfull, Cact, nb, a, F, M);
  return cudaGetLastError();
}

cudaError_t rte_launch_fft_extract(const void* spec, double* tau, int p0, int np, int C, size_t Mk, cudaStream_t st) {
  const size_t n = (size_t)np * Mk;
  k_fft_extract<<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const double2*)spec, tau, p0, np, C, Mk);
  return cudaGetLastError();
}

cudaError_t rte_launch_fft_product(const void* That, const void* Wh, void* Oh, int C, int Cact, int nb, size_t Mk,
                                   int complex_table, cudaStream_t st) {
  const unsigned blocks = (unsigned)((Mk + 127) / 128);
  if (complex_table) {
    k_fft_product_cplx<<<blocks, 128, 0, st>>>((const double2*)That, (const double2*)Wh, (double2*)Oh, C, Cact, nb, Mk);
    return cudaGetLastError();
  }
  const double* T = (const double*)That;
  const double2* W = (const double2*)Wh;
  double2* O = (double2*)Oh;
  const unsigned blocks2 = (unsigned)((2 * Mk + 127) / 128);  // one thread per frequency and set
  switch (Cact) {
    case 1: k_fft_product_reg<0><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    case 4: k_fft_product_reg<1><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    case 9: k_fft_product_reg<2><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    case 16: k_fft_product_reg<3><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    case 25: k_fft_product_reg<4><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    case 36: k_fft_product_reg<5><<<blocks2, 128, 0, st>>>(T, W, O, C, nb, Mk); break;
    default: k_fft_product<<<blocks, 128, 0, st>>>(T, W, O, C, Cact, nb, Mk);
  }
  return cudaGetLastError();
}

cudaError_t rte_launch_fft_crop(const double* F, int Cfull, int Cact, int nb, const FftTabArgs& a, double* part,
                                size_t M, cudaStream_t st) {
  const long long n = (long long)a.nx * a.ny * a.nz * nb * Cact;
  k_fft_crop<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(F, Cfull, Cact, nb, a, part, M);
  return cudaGetLastError();
}
