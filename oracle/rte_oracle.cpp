// rte_oracle.cpp -- FP64 CPU restatement of the reference Neumann-series RTE path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library in
// doi_b200/: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
// reference arm may load it.  The product never links or calls it.
//
// It works in the reference's COMPLEX spherical-harmonic basis (coefficient
// index cnt = l*l + l + m, distribution layout W[r*C + cnt], voxel index
// r = (z*nY + y)*nX + x), exactly as the reference host/device code does, so it
// is an independent implementation of what the CUDA library computes in a real
// basis.  Three discretisation modes:
//
//   mode 0  EXACT : exact Y_lm at the exact pair direction, FP64 path integral,
//                   200x200 self-voxel quadrature with per-axis half widths,
//                   Henyey-Greenstein scatter cm*g^l*mu_s.
//   mode 1  FIM   : FisherInfo_IO GPU kernels as written: 100x100 SH lookup table
//                   with the un-wrapped phi index, float-alpha Siddon path,
//                   100x100 self term on a cube of half width delX/2 with tissue 0
//                   (mu_t == 0) given no self term, scatter with g truncated to int.
//   mode 2  CPU   : CPU package (uniform medium): exact SH, exact attenuation,
//                   200x200 self quadrature with per-axis half widths.
//
// Intensity modulation (CPU package/src/RTE_uniform.c:125-129: mu_a -> mu_a + i*modulation/(c/n))
// enters as kappa, a uniform imaginary part of mu_t: pair attenuation exp(-(tau + i kappa r)), the
// self-voxel factor (1 - exp(-mu_t beta)) / mu_t with complex mu_t, and complex ballistic terms.
//
// Citations are to files of the reference project (paths inside it).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <complex>
#include <map>
#include <mutex>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

extern "C" {

typedef struct {
  int nx, ny, nz;
  double dx, dy, dz;           // voxel edge lengths
  double x_min, y_min, z_min;  // lower edges of the box
  int L;                       // SH order
  double g;                    // Henyey-Greenstein anisotropy
  double cm;                   // c/n used by the propagator and scatter
  double prop_thresh;          // pairs with |r-r'| < prop_thresh are coupled
  int mode;                    // 0 exact, 1 fim, 2 cpu
  int ssv;                     // self sub-voxels per axis (reference selfsubVox)
  int nthreads;                // OpenMP threads (0 = default)
  double kappa;                // imaginary part of mu_t (intensity modulation; 0 = steady state)
} orc_params;

typedef struct {
  double pos_x, pos_y, pos_z;
  double diam;
  double mag;
  int kind;  // 0: pencil column containing (pos_x,pos_y) (exact); 1: FIM column x==nX/2.0,y==nY/2.0;
             // 2: CPU package circle |xy-pos| <= diam/2 normalised by columns
} orc_source_t;

}  // extern "C"

static inline int ncoef(int L) { return (L + 1) * (L + 1); }

// ---------------------------------------------------------------------------
// Spherical harmonics in the reference convention.
// FisherInfo_IO/src/sph_harm.cu:112-159 (AssocLegendre, upward recurrence with the
// (-1)^m Condon-Shortley factor) and :74-102 (SpherHarmonic: nrm * P_l^|m| e^{i|m|phi},
// m<0 -> conj()/(-1)^|m|).
static double assoc_legendre(double x, int degree, int order) {
  int m = order < 0 ? -order : order;
  int len = degree - m + 2;
  double old = 0.0, cur, tmp, fact = 1.0;
  if (degree == 0) {
    cur = 1.0;
  } else {
    for (int i = 2 * m - 1; i > 0; i -= 2) fact *= (double)i;
    cur = fact * pow(-1.0, (double)m);
    cur = cur * pow(1.0 - pow(x, 2.0), ((double)m / 2.0));
  }
  int l = m + 1;
  for (int i = 2; i < len; i++) {
    tmp = x * (2.0 * (double)l - 1.0) * cur / ((double)(l - m)) -
          (double)(l + m - 1) / ((double)(l - m)) * old;
    old = cur;
    cur = tmp;
    l++;
  }
  return cur;
}

static cd sph_harm(double theta, double phi, int degree, int order) {
  int m = order < 0 ? -order : order;
  double fact = 1.0;
  for (int i = 0; i < 2 * m; i++) fact *= (double)(m + degree - i);
  double nrm = sqrt(((2.0 * (double)degree + 1.0) / (4.0 * M_PI * fact)));
  double P = assoc_legendre(cos(theta), degree, m);
  cd ret(nrm * P * cos((double)m * phi), nrm * P * sin((double)m * phi));
  if (order < 0) {
    ret = std::conj(ret);
    ret = ret / pow(-1.0, (double)m);
  }
  return ret;
}

static void sph_harm_all(int L, double theta, double phi, cd* out) {
  int c = 0;
  for (int l = 0; l <= L; l++)
    for (int m = -l; m <= l; m++) out[c++] = sph_harm(theta, phi, l, m);
}

// 100x100 lookup table, FisherInfo_IO/src/dist.cu:535-562: theta_i = i*pi/99,
// phi_j = 2*pi*j/99, table[cnt*10^4 + i*100 + j].
struct ShTable {
  int L;
  std::vector<cd> t;
};
static std::mutex g_tab_mu;
static std::map<int, ShTable*> g_tabs;
static const ShTable* get_table(int L) {
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto it = g_tabs.find(L);
  if (it != g_tabs.end()) return it->second;
  ShTable* T = new ShTable;
  T->L = L;
  int C = ncoef(L);
  T->t.resize((size_t)C * 10000);
  int cnt = 0;
  for (int l = 0; l <= L; l++)
    for (int m = -l; m <= l; m++) {
      for (int i = 0; i < 100; i++)
        for (int j = 0; j < 100; j++) {
          double th = (i * M_PI) / 99.0;
          double ph = (j * 2.0 * M_PI) / 99.0;
          T->t[(size_t)cnt * 10000 + i * 100 + j] = sph_harm(th, ph, l, m);
        }
      cnt++;
    }
  g_tabs[L] = T;
  return T;
}

// SPH_HARM_IND, FisherInfo_IO/src/defines.h:53-56: index = cnt*10^4 + rintf(99*theta/pi)*100
// + rintf(99*phi/(2pi)); phi is atan2() without wrapping (kernels.cu:331-333), so the phi
// index can be negative and the flat index lands in the previous theta row.  The flat
// in-table offset (without cnt) is returned; offsets < 0 would read before the table
// (only possible for theta index 0, which needs |dz|/dist > cos(pi/198)); such offsets are
// clamped to 0 and counted.
static long g_table_clamps = 0;
static inline int table_offset(double theta, double phi) {
  int ti = (int)rintf((float)((100 - 1) * (theta) / (M_PI)));
  int pj = (int)rintf((float)((100 - 1) * (phi) / (2 * M_PI)));
  int off = ti * 100 + pj;
  if (off < 0) {
    g_table_clamps++;
    off = 0;
  }
  return off;
}

// ---------------------------------------------------------------------------
// Radiological path between voxel centres.
// FisherInfo_IO/src/kernels.cu:50-148 (mu_int): alpha increments 0.5/|delta| for the first
// crossing on each axis, then 1/|delta|; tie order z, then y, then x; the destination
// voxel contributes half of the last increment.  T selects the arithmetic: float
// reproduces the reference (float alpha and float r), double is the exact path.
template <typename T>
static double mu_int(int si, int sj, int sk, int di, int dj, int dk, T r, const double* mut, int nx,
                     int ny) {
  double tot = 0.0;
  T az = 0, ay = 0, ax = 0, zinc, yinc, xinc, aprev = 0;
  const T INF = (T)10000000;
  int ic = si, jc = sj, kc = sk;
  zinc = (di != si) ? (T)fabs(0.5 / (di - si)) : INF;
  yinc = (dj != sj) ? (T)fabs(0.5 / (dj - sj)) : INF;
  xinc = (dk != sk) ? (T)fabs(0.5 / (dk - sk)) : INF;
  auto MU = [&](int i, int j, int k) { return mut[((size_t)i * ny + j) * nx + k]; };
  int guard = 0;
  while (aprev < 1) {
    if (++guard > 100000) break;
    if (az + zinc <= ax + xinc && az + zinc <= ay + yinc) {
      az += zinc;
      if (ic == si) zinc *= 2;
      tot = tot + MU(ic, jc, kc) * r * (az - aprev);
      ic = (si < di) ? ic + 1 : ic - 1;
      aprev = az;
      if (ic == di && jc == dj && kc == dk) return tot + MU(ic, jc, kc) * r * zinc / 2.0;
    } else if (ay + yinc < az + zinc && ay + yinc <= ax + xinc) {
      ay += yinc;
      if (jc == sj) yinc *= 2;
      tot = tot + MU(ic, jc, kc) * r * (ay - aprev);
      jc = (sj < dj) ? jc + 1 : jc - 1;
      aprev = ay;
      if (ic == di && jc == dj && kc == dk) return tot + MU(ic, jc, kc) * r * yinc / 2.0;
    } else if (ax + xinc < ay + yinc && ax + xinc < az + zinc) {
      ax += xinc;
      if (kc == sk) xinc *= 2;
      tot = tot + MU(ic, jc, kc) * r * (ax - aprev);
      kc = (sk < dk) ? kc + 1 : kc - 1;
      aprev = ax;
      if (ic == di && jc == dj && kc == dk) return tot + MU(ic, jc, kc) * r * xinc / 2.0;
    }
  }
  return tot;
}

// ---------------------------------------------------------------------------
// Self-voxel term.  Dself[c][c'] = sum_sub sum_omega conj(Y_c) Y_c' (1 - exp(-mut*beta))
// sin(theta) dtheta dphi / (ssv^3 * mut * dV), beta = distance from the sub-voxel centre to
// the voxel surface along omega.
//   fim (quad 0): FisherInfo_IO/src/dist.cu:362-533, 100x100 angles theta=i*pi/100,
//     phi=2*pi*j/100, cube [-1,1] in float, beta scaled by delX/2 on every axis.
//   cpu (quad 1): CPU package/src/Kernels_selfsub.c:738-959, 200x200 angles, sph_x/y/z and
//     face coordinates stored as float, beta with per-axis half widths.
// Returned matrix excludes the 1/cm factor (applied by the caller as the reference does,
// FisherInfo_IO/src/kernels.cu:175).
struct SelfKey {
  int quad, L, ssv;
  double mut, kappa, dx, dy, dz;
  bool operator<(const SelfKey& o) const {
    if (quad != o.quad) return quad < o.quad;
    if (L != o.L) return L < o.L;
    if (ssv != o.ssv) return ssv < o.ssv;
    if (mut != o.mut) return mut < o.mut;
    if (kappa != o.kappa) return kappa < o.kappa;
    if (dx != o.dx) return dx < o.dx;
    if (dy != o.dy) return dy < o.dy;
    return dz < o.dz;
  }
};
static std::mutex g_self_mu;
static std::map<SelfKey, std::vector<cd>*> g_self;

// distance (in units of the [-1,1] cube, per axis) from point (ii,jj,kk) to the cube face
// along (sx,sy,sz); the three face tests are made in the reference's order and the last
// matching face wins.  FT is the storage type of the direction cosines.
template <typename FT>
static void cube_exit(FT sx, FT sy, FT sz, float ii, float jj, float kk, int ssv, float* cx, float* cy,
                      float* cz) {
  const int face = 1;
  FT fx, fy, fz;
  if (sx != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fx = fc == 0 ? face : -face;
      fy = (fx - ii * 2.0 / ssv) * sy / sx + jj * 2.0 / ssv;
      fz = (fx - ii * 2.0 / ssv) * sz / sx + kk * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sx * fx >= 0) {
        *cx = fx; *cy = fy; *cz = fz;
      }
    }
  }
  if (sy != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fy = fc == 0 ? face : -face;
      fz = (fy - jj * 2.0 / ssv) * sz / sy + kk * 2.0 / ssv;
      fx = (fy - jj * 2.0 / ssv) * sx / sy + ii * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sy * fy >= 0) {
        *cx = fx; *cy = fy; *cz = fz;
      }
    }
  }
  if (sz != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fz = fc == 0 ? face : -face;
      fx = (fz - kk * 2.0 / ssv) * sx / sz + ii * 2.0 / ssv;
      fy = (fz - kk * 2.0 / ssv) * sy / sz + jj * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sz * fz >= 0) {
        *cx = fx; *cy = fy; *cz = fz;
      }
    }
  }
}

static const std::vector<cd>* self_matrix(int quad, int L, int ssv, double mut, double dx, double dy,
                                          double dz, double kappa = 0.0) {
  SelfKey key{quad, L, ssv, mut, kappa, dx, dy, dz};
  const cd muc(mut, kappa);
  {
    std::lock_guard<std::mutex> lk(g_self_mu);
    auto it = g_self.find(key);
    if (it != g_self.end()) return it->second;
  }
  int C = ncoef(L);
  int ang = quad == 0 ? 100 : 200;
  int nomega = ang * ang;
  std::vector<double> th(nomega), ph(nomega);
  for (int t = 0; t < ang; t++)
    for (int p = 0; p < ang; p++) {
      th[t * ang + p] = t * M_PI / ang;
      ph[t * ang + p] = p * 2.0 * M_PI / ang;
    }
  double dth = th[ang] - th[0], dph = ph[1] - ph[0];
  // weights per omega summed over sub-voxels: f(omega) = sum_sub (1-exp(-mut*beta)) sin(theta)
  std::vector<cd> f(nomega, 0.0);
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  for (float ii = -ssv / 2.0 + 0.5; ii <= ssv / 2.0 - 0.5; ii++)
    for (float jj = -ssv / 2.0 + 0.5; jj <= ssv / 2.0 - 0.5; jj++)
      for (float kk = -ssv / 2.0 + 0.5; kk <= ssv / 2.0 - 0.5; kk++)
        for (int w = 0; w < nomega; w++) {
          double dist;
          if (quad == 0) {
            double sx = cos(ph[w]) * sin(th[w]), sy = sin(ph[w]) * sin(th[w]), sz = cos(th[w]);
            cube_exit<double>(sx, sy, sz, ii, jj, kk, ssv, &cx, &cy, &cz);
            dist = sqrt(pow(ii * 2.0 / ssv - cx, 2.0) + pow(jj * 2.0 / ssv - cy, 2.0) +
                        pow(kk * 2.0 / ssv - cz, 2.0)) * dx / 2.0;
          } else {
            float sx = cos(ph[w]) * sin(th[w]), sy = sin(ph[w]) * sin(th[w]), sz = cos(th[w]);
            cube_exit<float>(sx, sy, sz, ii, jj, kk, ssv, &cx, &cy, &cz);
            dist = sqrt(pow(ii * 2.0 / ssv - cx, 2.0) * pow(dx / 2.0, 2.0) +
                        pow(jj * 2.0 / ssv - cy, 2.0) * pow(dy / 2.0, 2.0) +
                        pow(kk * 2.0 / ssv - cz, 2.0) * pow(dz / 2.0, 2.0));
          }
          f[w] += (1.0 - std::exp(-muc * dist)) * sin(th[w]);
        }
  std::vector<cd> Y((size_t)nomega * C);
  for (int w = 0; w < nomega; w++) sph_harm_all(L, th[w], ph[w], &Y[(size_t)w * C]);
  std::vector<cd>* D = new std::vector<cd>((size_t)C * C, cd(0, 0));
  double dV = dx * dy * dz;
  const cd denom = pow((double)ssv, 3) * muc * dV;
  for (int c = 0; c < C; c++)
    for (int cp = 0; cp < C; cp++) {
      cd s(0, 0);
      for (int w = 0; w < nomega; w++) s += std::conj(Y[(size_t)w * C + c]) * Y[(size_t)w * C + cp] * f[w];
      (*D)[(size_t)c * C + cp] = s * dth * dph / denom;
    }
  std::lock_guard<std::mutex> lk(g_self_mu);
  auto it = g_self.find(key);
  if (it != g_self.end()) {
    delete D;
    return it->second;
  }
  g_self[key] = D;
  return D;
}

// ---------------------------------------------------------------------------
// One application of the attenuation operator A (and optionally the scatter D).
// FisherInfo_IO/src/kernels.cu: compute_diagonal_abs :151-178, compute_propabs :289-366,
// scale_dist_dev :368-383, prop_scat_dev :385-418; host sequence prop_abs :704-808.
// mut_self (nullable): mu_t of each voxel for the self-voxel term when it differs from the mu_t of the
// path integrals (the FisherInfo_IO mains that change tissue values rebuild the self-term table from
// the new values but never refresh the device table the kernels read, e.g. rte_snr.cu:239,
// compute_grad_rte.cu:431: `populate_info_dev();` with its result dropped).
static void apply_op(const orc_params* p, const double* mua, const double* mus, const cd* in, cd* out, int flag,
                     int flag_scat, const int* dests = nullptr, long ndest = -1, const double* mut_self = nullptr) {
  const int nx = p->nx, ny = p->ny, nz = p->nz;
  const size_t N = (size_t)nx * ny * nz;
  const int Cfull = ncoef(p->L);
  const int Lact = flag ? p->L : 0;
  const int C = ncoef(Lact);
  std::vector<double> mut(N);
  for (size_t r = 0; r < N; r++) mut[r] = mua[r] + mus[r];
  const double* mts = mut_self ? mut_self : mut.data();
  const ShTable* tab = p->mode == 1 ? get_table(p->L) : nullptr;
  const int quad = p->mode == 1 ? 0 : 1;
  // self matrices for every distinct mu_t (the reference keeps one per tissue type)
  std::map<double, const std::vector<cd>*> selfm;
  for (size_t r = 0; r < N; r++)
    if (!selfm.count(mts[r])) {
      if (p->mode == 1 && mts[r] == 0.0)
        selfm[mts[r]] = nullptr;  // tissue 0 gets no self term (dist.cu:430 loop starts at 1)
      else
        selfm[mts[r]] = self_matrix(quad, p->L, p->ssv, mts[r], p->dx, p->dy, p->dz, p->mode == 1 ? 0.0 : p->kappa);
    }
  const double cm = p->cm;
  const double dV = p->dx * p->dy * p->dz;
  const long nloop = dests ? ndest : (long)N;
#ifdef _OPENMP
  int nth = p->nthreads > 0 ? p->nthreads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nth)
#endif
  for (long q = 0; q < nloop; q++) {
    const long r = dests ? dests[q] : q;
    int i = (int)(r / ((size_t)nx * ny)), j = (int)((r / nx) % ny), k = (int)(r % nx);
    std::vector<cd> acc(Cfull, cd(0, 0)), Y(Cfull);
    // self voxel
    const std::vector<cd>* D = selfm[mts[r]];
    if (D) {
      for (int c = 0; c < C; c++) {
        cd s(0, 0);
        for (int cp = 0; cp < C; cp++) s = s + (1.0 / cm) * (*D)[(size_t)c * Cfull + cp] * in[r * Cfull + cp];
        acc[c] = s;
      }
    }
    // all pairs
    for (int ip = 0; ip < nz; ip++) {
      double ddz = -(ip - i) * p->dz;
      for (int jp = 0; jp < ny; jp++) {
        double ddy = -(jp - j) * p->dy;
        for (int kp = 0; kp < nx; kp++) {
          double ddx = -(kp - k) * p->dx;
          double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
          if (!((ip != i || jp != j || kp != k) && dist < p->prop_thresh)) continue;
          double theta = acos(ddz / dist);
          double phi = atan2(ddy, ddx);
          size_t rp = ((size_t)ip * ny + jp) * nx + kp;
          double tau;
          if (p->mode == 1) {
            int off = table_offset(theta, phi);
            for (int c = 0; c < C; c++) Y[c] = tab->t[(size_t)c * 10000 + off];
            tau = mu_int<float>(i, j, k, ip, jp, kp, (float)dist, mut.data(), nx, ny);
          } else {
            for (int l = 0, c = 0; l <= Lact; l++)
              for (int m = -l; m <= l; m++) Y[c++] = sph_harm(theta, phi, l, m);
            tau = mu_int<double>(i, j, k, ip, jp, kp, dist, mut.data(), nx, ny);
          }
          cd S(0, 0);
          for (int cp = 0; cp < C; cp++) S = S + in[rp * Cfull + cp] * Y[cp];
          const double kappa = p->mode == 1 ? 0.0 : p->kappa;
          const cd kern = std::exp(-cd(tau, kappa * dist)) * (1.0 / (cm * dist * dist));
          for (int c = 0; c < C; c++) acc[c] = acc[c] + S * std::conj(Y[c]) * kern;
        }
      }
    }
    // x dV, then scatter
    int c = 0;
    for (int l = 0; l <= p->L; l++)
      for (int m = -l; m <= l; m++, c++) {
        cd v = acc[c] * dV;
        if (flag_scat) {
          if (p->mode == 1) {
            if (flag) {  // prop_scat_dev receives the same flag as the other kernels
              float cmf = (float)cm;
              double gi = (double)(int)p->g;  // __int2double_rn(int) truncation, kernels.cu:409
              v = (double)cmf * pow(gi, (double)l) * v * mus[r];
            } else {
              v = v * mus[r];  // kernels.cu:412 (Neumann passes flag = 0 when g == 0, neumann.cu:74-79)
            }
          } else {
            v = cm * pow(p->g, (double)l) * mus[r] * v;
          }
        }
        out[r * Cfull + c] = v;
      }
  }
}

// ---------------------------------------------------------------------------
// Stop rule, FisherInfo_IO/src/dist.cu:1132-1172 and CPU package/src/Kernels_selfsub.c:1184-1233.
static int stop_iteration(const orc_params* p, double* fi, int n, const cd* W, const cd* out) {
  const int C = ncoef(p->L);
  double sumW = 0, sumOut = 0, hi = 0;
  int i = p->nz - 1;
  for (int j = 0; j < p->ny; j++)
    for (int k = 0; k < p->nx; k++) {
      size_t r = ((size_t)i * p->ny + j) * p->nx + k;
      for (int c = 0; c < C; c++) {
        sumW += W[r * C + c].real();
        sumOut += out[r * C + c].real();
      }
    }
  if (n > 1) {
    if (sumOut == 0.0) return 1;
    hi = 1.0 - (sumW / sumOut) * (1.0 / (1.0 - (sumW / sumOut) / *fi));
    *fi = sumW / sumOut;
    if (hi > 1.0 || hi < 0.0) hi = 0.0;
  }
  return hi > 0.9999 ? 1 : 0;
}

extern "C" {

long orc_table_clamps(void) { return g_table_clamps; }

void orc_sh_complex(int L, double theta, double phi, double* out) {
  std::vector<cd> Y(ncoef(L));
  sph_harm_all(L, theta, phi, Y.data());
  memcpy(out, Y.data(), sizeof(cd) * Y.size());
}

double orc_assoc_legendre(double x, int l, int m) { return assoc_legendre(x, l, m); }

double orc_path_integral(const orc_params* p, const double* mut, int si, int sj, int sk, int di, int dj, int dk,
                         int fp32ref) {
  double ddz = -(di - si) * p->dz, ddy = -(dj - sj) * p->dy, ddx = -(dk - sk) * p->dx;
  double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
  if (fp32ref) return mu_int<float>(si, sj, sk, di, dj, dk, (float)dist, mut, p->nx, p->ny);
  return mu_int<double>(si, sj, sk, di, dj, dk, dist, mut, p->nx, p->ny);
}

// self matrix (complex, C*C, without 1/cm); quad 0 = FIM 100x100, 1 = CPU 200x200
void orc_self_matrix(int quad, int L, int ssv, double mut, double dx, double dy, double dz, double* out) {
  const std::vector<cd>* D = self_matrix(quad, L, ssv, mut, dx, dy, dz);
  memcpy(out, D->data(), sizeof(cd) * D->size());
}

// out = [D] A in for the listed destination voxels only (CPU-baseline samples)
int orc_apply_subset(const orc_params* p, const double* mua, const double* mus, const double* in, double* out,
                     int flag, int flag_scat, const int* dests, long ndest) {
  apply_op(p, mua, mus, (const cd*)in, (cd*)out, flag, flag_scat, dests, ndest);
  return 0;
}

// out = [D] A in  (complex interleaved, N*C*2 doubles)
int orc_apply(const orc_params* p, const double* mua, const double* mus, const double* in, double* out, int flag,
              int flag_scat) {
  apply_op(p, mua, mus, (const cd*)in, (cd*)out, flag, flag_scat);
  return 0;
}

// Collimated source term xi_d = D A xi (paper Eq. 23).
// kind 1: FisherInfo_IO/src/dist.cu:66-101 (column x == nX/2.0 && y == nY/2.0, product of
//   per-layer attenuations, no magnitude factor).
// kind 2: CPU package/src/Dist.c:1077-1128 (columns with |xy - pos| <= diam/2, attenuation
//   from the absolute z coordinate, normalised by mag / number of columns; uniform medium).
// kind 0: the column that contains (pos_x, pos_y), product form as kind 1, times mag.
// With kappa != 0 the attenuation factors take the complex mu_t (the CPU package itself builds its
// source before it modulates mu_a, RTE_uniform.c:127-129: pass kappa = 0 to reproduce that).
int orc_source(const orc_params* p, const double* mua, const double* mus, const orc_source_t* s, double* Wd) {
  const int nx = p->nx, ny = p->ny, nz = p->nz, C = ncoef(p->L);
  const double kap = p->mode == 1 ? 0.0 : p->kappa;
  cd* W = (cd*)Wd;
  size_t N = (size_t)nx * ny * nz;
  for (size_t q = 0; q < N * C; q++) W[q] = 0;
  double dV = p->dx * p->dy * p->dz;
  if (s->kind == 2) {
    int total = 0;
    for (int i = 0; i < nz; i++)
      for (int k = 0; k < nx; k++)
        for (int j = 0; j < ny; j++) {
          double xs = (double)k * p->dx + p->x_min + p->dx / 2.0;
          double ys = (double)j * p->dy + p->y_min + p->dy / 2.0;
          double zs = (double)i * p->dz + p->z_min + p->dz / 2.0;
          double rad = sqrt((xs - s->pos_x) * (xs - s->pos_x) + (ys - s->pos_y) * (ys - s->pos_y));
          if (rad <= (s->diam + 1.0e-16) / 2.0) {
            total++;
            size_t r = ((size_t)i * ny + j) * nx + k;
            const cd mt(mua[r] + mus[r], kap);
            double tz = zs - p->dz / 2.0;
            for (int l = 0; l <= p->L; l++)
              W[r * C + l * l + l] = pow(p->g, (double)l) * (mus[r] / mt) * sqrt(((2.0 * l) + 1.0) / (4.0 * M_PI)) *
                                     (std::exp(-mt * tz) - std::exp(-mt * (tz + p->dz))) / dV;
          }
        }
    if (total == 0) return 0;
    double fact = s->mag / ((double)total / (double)nz);
    for (size_t q = 0; q < N * C; q++) W[q] *= fact;
    return 0;
  }
  int cx, cy;
  if (s->kind == 1) {
    if (nx % 2 || ny % 2) return 0;  // k == nX/2.0 never holds for odd grids (dist.cu:76)
    cx = nx / 2;
    cy = ny / 2;
  } else {
    cx = (int)floor((s->pos_x - p->x_min) / p->dx);
    cy = (int)floor((s->pos_y - p->y_min) / p->dy);
    if (cx < 0) cx = 0;
    if (cx >= nx) cx = nx - 1;
    if (cy < 0) cy = 0;
    if (cy >= ny) cy = ny - 1;
  }
  double scale = s->kind == 1 ? 1.0 : s->mag;
  for (int i = 0; i < nz; i++) {
    size_t r = ((size_t)i * ny + cy) * nx + cx;
    cd tmp = 1.0;
    for (int ip = 0; ip < i; ip++) {
      size_t rp = ((size_t)ip * ny + cy) * nx + cx;
      tmp = tmp * std::exp(-cd(mus[rp] + mua[rp], kap) * p->dz);
    }
    const cd mt(mus[r] + mua[r], kap);
    for (int l = 0; l <= p->L; l++)
      W[r * C + l * l + l] = scale * pow(p->g, l) * mus[r] / mt * sqrt(((2.0 * (double)l) + 1.0) / (4.0 * M_PI)) *
                             tmp * (1.0 - std::exp(-mt * p->dz)) / dV;
  }
  return 0;
}

// Neumann series, FisherInfo_IO/src/neumann.cu:23-120.  W (current term) and out (running
// sum) are inputs, as in the reference; on return out = A * sum.  stop_rule 0: reference
// lambda rule (n starts at n0); 1: exactly max_terms terms; 2: ||W_k||_2 < tol*||sum||_2 or
// max_terms.  W is left holding the last term.
int orc_neumann_split(const orc_params* p, const double* mua, const double* mus, const double* mut_self, double* Wd,
                      double* outd, int flag, int stop_rule, int max_terms, double tol, int n0, int* nterms);

int orc_neumann(const orc_params* p, const double* mua, const double* mus, double* Wd, double* outd, int flag,
                int stop_rule, int max_terms, double tol, int n0, int* nterms) {
  return orc_neumann_split(p, mua, mus, nullptr, Wd, outd, flag, stop_rule, max_terms, tol, n0, nterms);
}

// Neumann (neumann.cu:23-120) whose self-voxel term takes mut_self (nullable) instead of mua + mus.
int orc_neumann_split(const orc_params* p, const double* mua, const double* mus, const double* mut_self, double* Wd,
                      double* outd, int flag, int stop_rule, int max_terms, double tol, int n0, int* nterms) {
  const size_t N = (size_t)p->nx * p->ny * p->nz;
  const int C = ncoef(p->L);
  cd* W = (cd*)Wd;
  cd* out = (cd*)outd;
  std::vector<cd> Wn(N * C), tmp(N * C);
  int terms = 0;
  if (flag == 1) {
    int n = n0;
    double fi = 1.0;
    int flag_l = p->g != 0.0 ? 1 : 0;  // neumann.cu:74-79
    for (;;) {
      if (stop_rule == 0) {
        if (stop_iteration(p, &fi, n, W, out)) break;
        if (terms >= 100000) break;
      } else if (terms >= max_terms) {
        break;
      }
      n++;
      apply_op(p, mua, mus, W, Wn.data(), flag_l, 1, nullptr, -1, mut_self);
      double nw = 0, ns = 0;
      for (size_t q = 0; q < N * C; q++) {
        out[q] = Wn[q] + out[q];
        W[q] = Wn[q];
        nw += std::norm(Wn[q]);
        ns += std::norm(out[q]);
      }
      terms++;
      if (stop_rule == 2 && sqrt(nw) < tol * sqrt(ns)) break;
    }
  }
  apply_op(p, mua, mus, out, tmp.data(), 1, 0, nullptr, -1, mut_self);
  memcpy(out, tmp.data(), sizeof(cd) * N * C);
  if (nterms) *nterms = terms;
  return 0;
}

// Exitance images of the z = nZ-1 (transmission) and z = 0 (reflection) faces.
// img_mode 1: FisherInfo_IO/src/dist.cu:103-161 and :229-268 (u_s = s/99, weight 1/99, factor
//   C = 1, ballistic on the FIM source column, reflection +int and x mag).
// img_mode 2: CPU package/src/Dist.c:134-229 (u = s/100 weight 1/100, factor c/n, reflection
//   over u in [-1, 0) with a minus sign, ballistic mag*exp(-mut*(zs[nZ-1]+dz/2)) in the circle).
// img_mode 0: exact hemispherical integrals int_0^1 P_l(u) u du (Gauss-Legendre), factor cm,
//   ballistic mag*prod exp(-mut dz) on the source column, reflection outward (as img_mode 2).
// trans/ref: nx*ny complex (interleaved), x fastest.
int orc_images(const orc_params* p, const double* mua, const double* mus, const orc_source_t* s, int img_mode,
               int with_ballistic, const double* outd, double* transd, double* refd) {
  const int nx = p->nx, ny = p->ny, nz = p->nz, C = ncoef(p->L);
  const double kap = img_mode == 1 ? 0.0 : p->kappa;  // ballistic with the complex mu_t
  const cd* out = (const cd*)outd;
  cd* trans = (cd*)transd;
  cd* ref = (cd*)refd;
  std::vector<double> wt(p->L + 1, 0.0), wr(p->L + 1, 0.0);
  double fac;
  if (img_mode == 1) {
    fac = 2.0 * M_PI * 1.0 * p->dx * p->dy / sqrt(4.0 * M_PI);
    for (int l = 0; l <= p->L; l++)
      for (int q = 0; q < 100; q++) {
        double u = (double)q / (100 - 1.0);
        double P = assoc_legendre(u, l, 0);
        wt[l] += sqrt(2.0 * l + 1.0) * P * u / (100 - 1.0);
      }
    for (int l = 0; l <= p->L; l++) wr[l] = wt[l];
  } else if (img_mode == 2) {
    fac = 2.0 * M_PI * p->dx * p->dy * p->cm / sqrt(4.0 * M_PI);
    for (int l = 0; l <= p->L; l++)
      for (int q = 0; q < 100; q++) {
        double u = (double)q / 100.0;
        wt[l] += sqrt(2.0 * l + 1.0) * assoc_legendre(u, l, 0) * u / 100.0;
        double v = (double)q / 100.0 - 1.0;
        wr[l] -= sqrt(2.0 * l + 1.0) * assoc_legendre(v, l, 0) * v / 100.0;
      }
  } else {
    fac = 2.0 * M_PI * p->dx * p->dy * p->cm / sqrt(4.0 * M_PI);
    // 32-point Gauss-Legendre on [0,1] (exact for the polynomial P_l(u) u, l <= 62)
    const int NG = 32;
    std::vector<double> xg(NG), wg(NG);
    for (int q = 0; q < NG; q++) {
      double x = cos(M_PI * (q + 0.75) / (NG + 0.5));
      for (int it = 0; it < 100; it++) {
        double p0 = 1, p1 = x;
        for (int l = 2; l <= NG; l++) {
          double p2 = ((2 * l - 1) * x * p1 - (l - 1) * p0) / l;
          p0 = p1;
          p1 = p2;
        }
        double dp = NG * (x * p1 - p0) / (x * x - 1);
        double dx = p1 / dp;
        x -= dx;
        if (fabs(dx) < 1e-16) break;
      }
      double p0 = 1, p1 = x;
      for (int l = 2; l <= NG; l++) {
        double p2 = ((2 * l - 1) * x * p1 - (l - 1) * p0) / l;
        p0 = p1;
        p1 = p2;
      }
      double dp = NG * (x * p1 - p0) / (x * x - 1);
      xg[q] = 0.5 * (x + 1);
      wg[q] = 1.0 / ((1 - x * x) * dp * dp);  // 2/((1-x^2)P'^2) scaled by 1/2
    }
    for (int l = 0; l <= p->L; l++)
      for (int q = 0; q < NG; q++) {
        double u = xg[q];
        wt[l] += sqrt(2.0 * l + 1.0) * assoc_legendre(u, l, 0) * u * wg[q];
        wr[l] += sqrt(2.0 * l + 1.0) * assoc_legendre(-u, l, 0) * u * wg[q];
      }
  }
  for (int j = 0; j < ny; j++)
    for (int k = 0; k < nx; k++) {
      size_t rt = ((size_t)(nz - 1) * ny + j) * nx + k;
      size_t rr = ((size_t)0 * ny + j) * nx + k;
      cd vt(0, 0), vr(0, 0);
      if (with_ballistic) {
        if (img_mode == 1) {
          if (nx % 2 == 0 && ny % 2 == 0 && k == nx / 2 && j == ny / 2) {
            double tmp = s->mag;
            for (int i = 0; i < nz; i++) {
              size_t r = ((size_t)i * ny + j) * nx + k;
              tmp *= exp(-(mus[r] + mua[r]) * p->dz);
            }
            vt += tmp;
          }
        } else if (img_mode == 2) {
          double xs = (double)k * p->dx + p->x_min + p->dx / 2.0;
          double ys = (double)j * p->dy + p->y_min + p->dy / 2.0;
          double rad = sqrt((xs - s->pos_x) * (xs - s->pos_x) + (ys - s->pos_y) * (ys - s->pos_y));
          if (rad <= (s->diam + 1.0e-16) / 2.0) {
            // CPU package normalises mag by the number of source columns (Dist.c:1113-1114)
            int cols = 0;
            for (int jj = 0; jj < ny; jj++)
              for (int kk = 0; kk < nx; kk++) {
                double x2 = (double)kk * p->dx + p->x_min + p->dx / 2.0;
                double y2 = (double)jj * p->dy + p->y_min + p->dy / 2.0;
                if (sqrt((x2 - s->pos_x) * (x2 - s->pos_x) + (y2 - s->pos_y) * (y2 - s->pos_y)) <=
                    (s->diam + 1.0e-16) / 2.0)
                  cols++;
              }
            double zs = (double)(nz - 1) * p->dz + p->z_min + p->dz / 2.0;
            const cd mt(mua[rt] + mus[rt], kap);
            vt += (s->mag / cols) * std::exp(-mt * (zs + p->dz / 2.0));
          }
        } else {
          int cx = (int)floor((s->pos_x - p->x_min) / p->dx), cy = (int)floor((s->pos_y - p->y_min) / p->dy);
          cx = cx < 0 ? 0 : (cx >= nx ? nx - 1 : cx);
          cy = cy < 0 ? 0 : (cy >= ny ? ny - 1 : cy);
          if (k == cx && j == cy) {
            cd tmp = s->mag;
            for (int i = 0; i < nz; i++) {
              size_t r = ((size_t)i * ny + j) * nx + k;
              tmp *= std::exp(-cd(mus[r] + mua[r], kap) * p->dz);
            }
            vt += tmp;
          }
        }
      }
      for (int l = 0; l <= p->L; l++) {
        vt += fac * wt[l] * out[rt * C + l * l + l];
        vr += fac * wr[l] * out[rr * C + l * l + l];
      }
      trans[(size_t)j * nx + k] = vt;
      ref[(size_t)j * nx + k] = img_mode == 1 ? vr * s->mag : vr;
    }
  return 0;
}

}  // extern "C"
