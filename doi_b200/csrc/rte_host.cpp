// rte_host.cpp -- host side of the B200 RTE solver: context, discretisation set-up and the
// Neumann driver behind the C ABI of include/rte_b200.h.
//
// Reference entry points mirrored (paths inside the reference project):
//   Neumann()              FisherInfo_IO/src/neumann.cu:23-120
//   prop_abs()             FisherInfo_IO/src/kernels.cu:704-808
//   generate_source_beam   FisherInfo_IO/src/dist.cu:66-101 (and CPU package/src/Dist.c:1077-1128)
//   generate_trans_image   FisherInfo_IO/src/dist.cu:103-161
//   generate_ref_image     FisherInfo_IO/src/dist.cu:229-268
//   generate_diag_terms_host FisherInfo_IO/src/dist.cu:362-533 (self-voxel term)
//   StopIteration          FisherInfo_IO/src/dist.cu:1132-1172
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <complex>
#include <array>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rte_b200.h"
#include "rte_internal.h"

namespace {

inline int ncoef(int L) { return (L + 1) * (L + 1); }

}  // namespace

// ---------------------------------------------------------------------------------------
// Real spherical harmonics (host copy of the device recurrence in rte_kernels.cu).
// Normalisation K_lm = sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!) (times sqrt2 for m > 0) of the
// reference's complex basis (FisherInfo_IO/src/sph_harm.cu:19-64), Condon-Shortley phase from
// P_m^m = (-1)^m (2m-1)!! (1-z^2)^{m/2} (sph_harm.cu:133-137).
ShTables make_sh_tables() {
  ShTables t;
  memset(&t, 0, sizeof t);
  auto K = [](int l, int m) {
    double f = 1.0;  // (l+m)!/(l-m)!
    for (int i = l - m + 1; i <= l + m; i++) f *= (double)i;
    double k = sqrt((2.0 * l + 1.0) / (4.0 * M_PI) / f);
    return m > 0 ? k * sqrt(2.0) : k;
  };
  for (int m = 0; m <= RTE_MAX_L; m++) {
    double dfact = 1.0;
    for (int i = 2 * m - 1; i > 0; i -= 2) dfact *= (double)i;
    t.Q0[m] = K(m, m) * ((m & 1) ? -1.0 : 1.0) * dfact;
    for (int l = m + 1; l <= RTE_MAX_L; l++) {
      int id = l * (l + 1) / 2 + m;
      t.A[id] = K(l, m) * (2.0 * l - 1.0) / ((double)(l - m) * K(l - 1, m));
      t.B[id] = (l - 2 >= m) ? K(l, m) * (double)(l + m - 1) / ((double)(l - m) * K(l - 2, m)) : 0.0;
    }
  }
  return t;
}

void sh_real_host(const ShTables& t, int L, double x, double y, double z, double* R) {
  double cmv = 1.0, smv = 0.0;
  for (int m = 0; m <= L; m++) {
    if (m > 0) {
      double c2 = cmv * x - smv * y, s2 = cmv * y + smv * x;
      cmv = c2;
      smv = s2;
    }
    double q2 = 0.0, q1 = t.Q0[m];
    if (m == 0)
      R[0] = q1;
    else {
      R[m * m + 2 * m] = q1 * cmv;
      R[m * m] = q1 * smv;
    }
    for (int l = m + 1; l <= L; l++) {
      int id = l * (l + 1) / 2 + m;
      double q = t.A[id] * z * q1 - t.B[id] * q2;
      q2 = q1;
      q1 = q;
      if (m == 0)
        R[l * l + l] = q;
      else {
        R[l * l + l + m] = q * cmv;
        R[l * l + l - m] = q * smv;
      }
    }
  }
}

namespace {

// Legendre polynomial P_l(u) (m = 0 associated Legendre of sph_harm.cu:172-237).
double legendre(int l, double u) {
  double p0 = 1.0, p1 = u;
  if (l == 0) return 1.0;
  for (int k = 2; k <= l; k++) {
    double p2 = ((2.0 * k - 1.0) * u * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  return p1;
}

// Gauss-Legendre nodes/weights on [0,1].
void gauss01(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; i++) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 200; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-17) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; k++) {
      double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[i] = 0.5 * (z + 1.0);
    w[i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

// ---------------------------------------------------------------------------------------
// Self-voxel quadrature.  For each sub-voxel and direction, beta = distance from the
// sub-voxel centre to the voxel surface.  quad 0 follows FisherInfo_IO/src/dist.cu:404-480
// (100x100 directions, direction cosines in double, face point in float, cube scaled by delX/2
// on every axis); quad 1 follows CPU package/src/Kernels_selfsub.c:838-927 (200x200 directions,
// direction cosines and face point in float, per-axis half widths).  The face tests are made
// in the reference order and the last hit wins.
template <typename FT>
void exit_point(FT sx, FT sy, FT sz, float ii, float jj, float kk, int ssv, float& cx, float& cy, float& cz) {
  const int face = 1;
  FT fx, fy, fz;
  if (sx != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fx = fc == 0 ? face : -face;
      fy = (fx - ii * 2.0 / ssv) * sy / sx + jj * 2.0 / ssv;
      fz = (fx - ii * 2.0 / ssv) * sz / sx + kk * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sx * fx >= 0) {
        cx = fx;
        cy = fy;
        cz = fz;
      }
    }
  }
  if (sy != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fy = fc == 0 ? face : -face;
      fz = (fy - jj * 2.0 / ssv) * sz / sy + kk * 2.0 / ssv;
      fx = (fy - jj * 2.0 / ssv) * sx / sy + ii * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sy * fy >= 0) {
        cx = fx;
        cy = fy;
        cz = fz;
      }
    }
  }
  if (sz != 0.0) {
    for (int fc = 0; fc < 2; fc++) {
      fz = fc == 0 ? face : -face;
      fx = (fz - kk * 2.0 / ssv) * sx / sz + ii * 2.0 / ssv;
      fy = (fz - kk * 2.0 / ssv) * sy / sz + jj * 2.0 / ssv;
      if (fx <= face && fx >= -face && fy <= face && fy >= -face && fz <= face && fz >= -face && sz * fz >= 0) {
        cx = fx;
        cy = fy;
        cz = fz;
      }
    }
  }
}

// Self-term moments.  Dself(mu) W = sum_k mu^k M_k W with
//   M_k[c][c'] = dth dph / (ssv^3 dV) * (-1)^k/(k+1)! * sum_sub sum_w sin(th) R_c R_c' beta^(k+1),
// the power series of (1 - exp(-mu beta))/mu (dist.cu:479-500 divides by mu_t).
struct SelfQuad {
  int L = -1, quad = -1, ssv = 0;
  double dx = 0, dy = 0, dz = 0;
  int nw = 0, nsub = 0;
  std::vector<double> R;      // [nw][C]
  std::vector<double> wgt;    // [nw]  sin(theta) dth dph
  std::vector<double> beta;   // [nsub][nw]
  double beta_max = 0;
};

void build_quad(SelfQuad& q, int L, int quad, int ssv, double dx, double dy, double dz, const ShTables& sh) {
  q.L = L;
  q.quad = quad;
  q.ssv = ssv;
  q.dx = dx;
  q.dy = dy;
  q.dz = dz;
  const int ang = quad == 0 ? 100 : 200;
  const int C = ncoef(L);
  q.nw = ang * ang;
  std::vector<double> th(q.nw), ph(q.nw);
  for (int t = 0; t < ang; t++)
    for (int p = 0; p < ang; p++) {
      th[t * ang + p] = t * M_PI / ang;
      ph[t * ang + p] = p * 2.0 * M_PI / ang;
    }
  const double dth = th[ang] - th[0], dph = ph[1] - ph[0];
  q.R.assign((size_t)q.nw * C, 0.0);
  q.wgt.assign(q.nw, 0.0);
  for (int w = 0; w < q.nw; w++) {
    double st = sin(th[w]);
    sh_real_host(sh, L, cos(ph[w]) * st, sin(ph[w]) * st, cos(th[w]), &q.R[(size_t)w * C]);
    q.wgt[w] = st * dth * dph;
  }
  q.nsub = ssv * ssv * ssv;
  q.beta.assign((size_t)q.nsub * q.nw, 0.0);
  q.beta_max = 0;
  int sub = 0;
  float cx = 0.0f, cy = 0.0f, cz = 0.0f;
  for (float ii = -ssv / 2.0 + 0.5; ii <= ssv / 2.0 - 0.5; ii++)
    for (float jj = -ssv / 2.0 + 0.5; jj <= ssv / 2.0 - 0.5; jj++)
      for (float kk = -ssv / 2.0 + 0.5; kk <= ssv / 2.0 - 0.5; kk++, sub++)
        for (int w = 0; w < q.nw; w++) {
          double b;
          if (quad == 0) {
            double sx = cos(ph[w]) * sin(th[w]), sy = sin(ph[w]) * sin(th[w]), sz = cos(th[w]);
            exit_point<double>(sx, sy, sz, ii, jj, kk, ssv, cx, cy, cz);
            b = sqrt(pow(ii * 2.0 / ssv - cx, 2.0) + pow(jj * 2.0 / ssv - cy, 2.0) + pow(kk * 2.0 / ssv - cz, 2.0)) *
                dx / 2.0;
          } else {
            float sx = cos(ph[w]) * sin(th[w]), sy = sin(ph[w]) * sin(th[w]), sz = cos(th[w]);
            exit_point<float>(sx, sy, sz, ii, jj, kk, ssv, cx, cy, cz);
            b = sqrt(pow(ii * 2.0 / ssv - cx, 2.0) * pow(dx / 2.0, 2.0) +
                     pow(jj * 2.0 / ssv - cy, 2.0) * pow(dy / 2.0, 2.0) +
                     pow(kk * 2.0 / ssv - cz, 2.0) * pow(dz / 2.0, 2.0));
          }
          q.beta[(size_t)sub * q.nw + w] = b;
          q.beta_max = std::max(q.beta_max, b);
        }
}

void build_moments(const SelfQuad& q, int K, double dV, std::vector<double>& mom) {
  const int C = ncoef(q.L);
  mom.assign((size_t)K * C * C, 0.0);
  const int nth = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::vector<double>> part(nth, std::vector<double>((size_t)K * C * C, 0.0));
  auto work = [&](int t) {
    std::vector<double> g(K);
    std::vector<double>& M = part[t];
    for (int w = t; w < q.nw; w += nth) {
      for (int k = 0; k < K; k++) g[k] = 0.0;
      for (int s = 0; s < q.nsub; s++) {
        double b = q.beta[(size_t)s * q.nw + w], bp = b;
        for (int k = 0; k < K; k++) {
          g[k] += bp;
          bp *= b;
        }
      }
      const double* R = &q.R[(size_t)w * C];
      for (int k = 0; k < K; k++) {
        const double gk = g[k] * q.wgt[w];
        if (gk == 0.0) continue;
        double* Mk = &M[(size_t)k * C * C];
        for (int c = 0; c < C; c++) {
          const double a = gk * R[c];
          for (int cp = c; cp < C; cp++) Mk[c * C + cp] += a * R[cp];
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (int t = 0; t < nth; t++) th.emplace_back(work, t);
  for (auto& x : th) x.join();
  double fact = 1.0;
  for (int k = 0; k < K; k++) {
    fact *= (double)(k + 1);  // (k+1)!
    const double sc = ((k & 1) ? -1.0 : 1.0) / fact / ((double)q.nsub * dV);
    for (int c = 0; c < C; c++)
      for (int cp = c; cp < C; cp++) {
        double v = 0.0;
        for (int t = 0; t < nth; t++) v += part[t][(size_t)k * C * C + c * C + cp];
        mom[(size_t)k * C * C + c * C + cp] = v * sc;
        mom[(size_t)k * C * C + cp * C + c] = v * sc;
      }
  }
}

}  // namespace

// ---------------------------------------------------------------------------------------
struct rte_ctx {
  rte_config cfg;
  int nx, ny, nz, N, L, C;
  double dx, dy, dz, dV, cm, prop_thresh;
  int model, precision, kernel_mode;
  std::string err;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ShTables sh;
  SelfQuad quad;
  int K = 0;  // moments in use
  int* d_perm = nullptr;
  double *d_mut = nullptr, *d_mus = nullptr;
  float* d_mutf = nullptr;
  double *d_W = nullptr, *d_Wn = nullptr, *d_sum = nullptr, *d_part = nullptr, *d_mom = nullptr;
  double *d_aux1 = nullptr, *d_aux2 = nullptr, *d_aux3 = nullptr, *d_aux4 = nullptr;  // real-basis staging
  float* d_Wf = nullptr;
  float* d_K = nullptr;
  double* d_K64 = nullptr;      // FP64 pair kernel (FP64 contexts in RTE_KERNEL_STORE mode)
  bool K_valid = false;
  double* d_cplx = nullptr;
  double* d_red = nullptr;
  double* d_img = nullptr;  // trans, ref (complex)
  bool medium_set = false;
  int max_split = 8;
  std::vector<std::array<int, 4>> splits;  // (kernel key, S, chunk, tile) of each planned launch shape
  size_t Kld = 0;
  double* d_selfp = nullptr;    // self-voxel term [N][nb][C]
  int* d_self_idx = nullptr;    // voxel -> distinct mu_t
  double* d_self_lut = nullptr; // [ndistinct][C][C]
  bool self_lut_ok = false;
  size_t lut_cap = 0;
  std::vector<double> h_mom;    // host copy of the moments [K][C][C]
  int* d_islot = nullptr;       // voxel -> slot
  float4* d_slot_xyz = nullptr; // slot -> (x, y, z, voxel)
  int* d_err = nullptr;         // bounded-wait failure flag of the pair kernels
  int cpad = 0;                 // FP32 source row length (nb = 1)
  int cstride = 0;              // FP32 stride of one right-hand side within a row (multiple of 4: 16-byte loads)
  // batched solves (several sources on one medium): buffers for up to bcap right-hand sides
  int bcap = 0;
  double *d_bW = nullptr, *d_bWn = nullptr, *d_bsum = nullptr, *d_bres = nullptr, *d_bball = nullptr;
  float* d_bWf = nullptr;
  size_t part_cap = 0, selfp_cap = 0;
  // detectors and gradient
  double* d_h = nullptr;        // [6][C] face flux weights
  double *d_S = nullptr, *d_out = nullptr, *d_e = nullptr, *d_lam = nullptr, *d_y = nullptr;
  double *d_gt = nullptr, *d_gs = nullptr, *d_J = nullptr, *d_rho = nullptr, *d_dlut = nullptr;
  std::vector<double> h_h;      // host copy of the face weights
  size_t dlut_cap = 0;
  double* d_fball = nullptr;    // ballistic flux per face pixel of the current single source
  double* d_q = nullptr;        // point-source emission of the current single source [N][C]
  bool has_point = false;
  bool capturing = false;       // recording a CUDA graph: no host synchronisation allowed
  bool capture_store = false;   // record the pair-kernel precompute into the graph being captured
  // captured Neumann series per right-hand-side count (1, 2, 4) and terms
  cudaGraphExec_t graph[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int graph_terms[5] = {0, 0, 0, 0, 0};
  double* graph_w0[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // buffers the graph reads W0 / S0 from
  double* graph_s0[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double* d_bq = nullptr;       // batched point emissions [N][nb][C]
  cudaEvent_t ev_graph[2] = {nullptr, nullptr};  // device time of one graph request
  // every device pointer and scalar a recorded graph baked into its kernel parameters; a graph whose
  // signature differs from the context's current one (a buffer was reallocated, the self-term path
  // or its series length changed with the medium) is recorded again before it is replayed
  std::vector<uintptr_t> graph_sig[5];
  void* d_Qbp = nullptr;        // gradient: weight of every unordered voxel pair (N x round32(N))
  uint8_t* d_mask = nullptr;    // region mask of the reference-compatible tangent solves [N]
  bool transpose = false;       // pair kernels apply A^T (table model: reverse-displacement snapping)
  // split medium (rte_set_medium_tissue_split): the self-voxel term, the source and its ballistic beam
  // take d_mut_self / d_mus_src, while the pair kernels and the scatter keep d_mut / d_mus
  bool split = false;
  double* d_mut_self = nullptr;
  double* d_mus_src = nullptr;
  bool uniform = false;         // the medium has one mu_t: the operator is a convolution
  double uniform_mut = 0.0;
  FftState* fft = nullptr;      // its table spectra, buffers and plans
  bool fft_capture_ready = false;  // a graph recording may capture the transforms
  bool fft_graph_failed = false;   // recording the transforms failed once: graphs use the pair kernels
  bool fft_in_graph[5] = {false, false, false, false, false};
  double* d_dmut = nullptr;     // Fisher: parameter direction of mu_t and mu_s [N], tangent dA S [N][C]
  double* d_dmus = nullptr;
  double* d_T = nullptr;
  int* d_cidx = nullptr;        // source-column voxels and their source derivative
  double* d_cval = nullptr;
  // intensity modulation (CPU package/src/RTE_uniform.c:120-176): mu_a -> mu_a + i modulation/(c/n),
  // so mu_t has the uniform imaginary part kappa; radiance is complex, (real, imaginary) row pairs
  double modulation = 0.0, kappa = 0.0;
  double mumax = 0.0;             // max real mu_t of the medium
  double* d_self_lut_im = nullptr;  // imaginary part of the self-term table
  size_t lut_im_cap = 0;
  double* d_fball_im = nullptr;   // imaginary part of the single source's ballistic flux
  size_t qbp_bytes = 0;
  size_t bytes = 0;
  double last_setup_ms = 0.0;
  // measurement: launch count and per-class event pairs (0 pair, 1 store, 2 epilogue)
  long long launches = 0;
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[3];
  std::vector<cudaEvent_t> ev_pool;
  double ms_acc[3] = {0, 0, 0};
  long long n_acc[3] = {0, 0, 0};
};

static cudaEvent_t pool_event(rte_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// brackets one launch of class k with events when profiling
struct ProfScope {
  rte_ctx* c;
  int k;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(rte_ctx* c_, int k_) : c(c_), k(k_) {
    c->launches++;
    if (c->profiling) {
      a = pool_event(c);
      b = pool_event(c);
      cudaEventRecord(a, c->st);
    }
  }
  ~ProfScope() {
    if (a) {
      cudaEventRecord(b, c->st);
      c->ev[k].push_back({a, b});
    }
  }
};

static thread_local std::string g_create_err;

void rte_set_global_error(const char* msg) { g_create_err = msg ? msg : ""; }

static int fail(rte_ctx* c, int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c)
    c->err = buf;
  else
    g_create_err = buf;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                       \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? RTE_ERR_NOMEM : RTE_ERR_DEVICE,          \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);           \
  } while (0)

template <class T>
static cudaError_t dalloc(rte_ctx* c, T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e == cudaSuccess) c->bytes += n * sizeof(T);
  return e;
}

static void free_all(rte_ctx* c) {
  rte_fft_destroy(c->fft);
  c->fft = nullptr;
  for (int k = 0; k < 5; k++)
    if (c->graph[k]) cudaGraphExecDestroy(c->graph[k]);
  for (int k = 0; k < 2; k++)
    if (c->ev_graph[k]) cudaEventDestroy(c->ev_graph[k]);
  for (int k = 0; k < 3; k++)
    for (auto& p : c->ev[k]) {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
  for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
  void* ps[] = {c->d_perm, c->d_mut, c->d_mus, c->d_mutf, c->d_W, c->d_Wn, c->d_sum, c->d_part, c->d_mom,
                c->d_aux1, c->d_aux2, c->d_aux3, c->d_aux4, c->d_Wf, c->d_K, c->d_K64, c->d_cplx, c->d_red, c->d_img,
                c->d_selfp, c->d_self_idx, c->d_self_lut, c->d_islot, c->d_slot_xyz, c->d_err,
                c->d_bW, c->d_bWn, c->d_bsum, c->d_bres, c->d_bball, c->d_bWf, c->d_h, c->d_S, c->d_out,
                c->d_e, c->d_lam, c->d_y, c->d_gt, c->d_gs, c->d_J, c->d_rho, c->d_dlut, c->d_fball, c->d_q, c->d_bq,
                c->d_Qbp, c->d_mask, c->d_dmut, c->d_dmus, c->d_mut_self, c->d_mus_src, c->d_T, c->d_cidx, c->d_cval, c->d_self_lut_im,
                c->d_fball_im};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->st) cudaStreamDestroy(c->st);
}

// destination order: Morton (z-order) over (x, y, z) so that a warp's 32 destinations form a
// compact brick (coherent path walks, shared cache lines of mu_t).
static std::vector<int> morton_perm(int nx, int ny, int nz) {
  auto spread = [](uint64_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 21; b++) r |= ((v >> b) & 1ull) << (3 * b);
    return r;
  };
  std::vector<std::pair<uint64_t, int>> keys;
  keys.reserve((size_t)nx * ny * nz);
  for (int i = 0; i < nz; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nx; k++)
        keys.push_back({spread(k) | (spread(j) << 1) | (spread(i) << 2), (i * ny + j) * nx + k});
  std::sort(keys.begin(), keys.end());
  std::vector<int> p(keys.size());
  for (size_t q = 0; q < keys.size(); q++) p[q] = keys[q].second;
  return p;
}

extern "C" {

int rte_create(const rte_config* cfg, rte_ctx** out) {
  g_create_err.clear();
  if (!cfg || !out) return fail(nullptr, RTE_ERR_ARG, "null argument");
  *out = nullptr;
  if (cfg->nx <= 0 || cfg->ny <= 0 || cfg->nz <= 0 || cfg->nx > 1024 || cfg->ny > 1024 || cfg->nz > 1024)
    return fail(nullptr, RTE_ERR_ARG, "grid %dx%dx%d out of range", cfg->nx, cfg->ny, cfg->nz);
  if ((long long)cfg->nx * cfg->ny * cfg->nz > (1ll << 26))
    return fail(nullptr, RTE_ERR_UNSUPPORTED, "more than 2^26 voxels");
  if (cfg->nL < 0 || cfg->nL > RTE_MAX_L) return fail(nullptr, RTE_ERR_UNSUPPORTED, "nL=%d outside 0..%d", cfg->nL, RTE_MAX_L);
  if (cfg->model < RTE_MODEL_EXACT || cfg->model > RTE_MODEL_CPU) return fail(nullptr, RTE_ERR_ARG, "bad model");
  if (cfg->precision != RTE_PREC_FP64 && cfg->precision != RTE_PREC_MIXED)
    return fail(nullptr, RTE_ERR_ARG, "bad precision");
  if (cfg->n <= 0 || cfg->c <= 0) return fail(nullptr, RTE_ERR_ARG, "refractive index and speed must be > 0");
  if (cfg->self_sub_vox < 1 || cfg->self_sub_vox > 16) return fail(nullptr, RTE_ERR_ARG, "selfsubVox out of range");
  rte_ctx* c = new rte_ctx;
  c->cfg = *cfg;
  c->nx = cfg->nx;
  c->ny = cfg->ny;
  c->nz = cfg->nz;
  c->N = cfg->nx * cfg->ny * cfg->nz;
  c->L = cfg->nL;
  c->C = ncoef(cfg->nL);
  c->model = cfg->model;
  c->precision = cfg->precision;
  c->kernel_mode = cfg->kernel_mode;
  if (c->model == RTE_MODEL_FIM) {
    // Geometry extents and propThresh are float fields in the reference (rte.h:58-73) and
    // cm = C/n with C = 1 is a float (rte.h:108, rte.cu:63).
    c->dx = (double)((float)cfg->x_max - (float)cfg->x_min) / (double)cfg->nx;
    c->dy = (double)((float)cfg->y_max - (float)cfg->y_min) / (double)cfg->ny;
    c->dz = (double)((float)cfg->z_max - (float)cfg->z_min) / (double)cfg->nz;
    c->prop_thresh = (double)(float)cfg->prop_thresh;
    c->cm = (double)(float)(1.0 / cfg->n);
  } else {
    c->dx = (cfg->x_max - cfg->x_min) / cfg->nx;
    c->dy = (cfg->y_max - cfg->y_min) / cfg->ny;
    c->dz = (cfg->z_max - cfg->z_min) / cfg->nz;
    c->prop_thresh = cfg->prop_thresh;
    c->cm = cfg->c / cfg->n;
  }
  if (!(c->dx > 0 && c->dy > 0 && c->dz > 0)) {
    delete c;
    return fail(nullptr, RTE_ERR_ARG, "voxel size must be positive");
  }
  c->dV = c->dx * c->dy * c->dz;
  c->sh = make_sh_tables();
  int rc = RTE_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == RTE_OK)
      rc = fail(nullptr, e == cudaErrorMemoryAllocation ? RTE_ERR_NOMEM : RTE_ERR_DEVICE, "%s: %s", what,
                cudaGetErrorString(e));
  };
  cu(cudaSetDevice(cfg->device), "cudaSetDevice");
  if (rc == RTE_OK) cu(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking), "stream");
  if (rc == RTE_OK) cu(cudaEventCreate(&c->ev0), "event");
  if (rc == RTE_OK) cu(cudaEventCreate(&c->ev1), "event");
  if (rc == RTE_OK) {  // the tables do not depend on the order: one upload per device and process
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), cfg->device) == done.end()) {
      cu(rte_upload_sh_tables(c->sh), "SH tables");
      if (rc == RTE_OK) done.push_back(cfg->device);
    }
  }
  const size_t NC = (size_t)c->N * c->C;
  if (const char* e = getenv("RTE_MAX_SPLIT")) c->max_split = std::max(1, std::min(32, atoi(e)));
  if (rc == RTE_OK) cu(dalloc(c, &c->d_perm, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_mut, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_mus, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_mutf, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_W, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_Wn, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_sum, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_aux1, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_aux2, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_aux3, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_aux4, NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_part, NC * c->max_split), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_selfp, NC), "alloc");
  c->part_cap = NC * c->max_split;
  c->selfp_cap = NC;
  if (rc == RTE_OK) cu(dalloc(c, &c->d_self_idx, c->N), "alloc");
  c->cstride = (c->C + 3) / 4 * 4;
  c->cpad = (c->cstride + 3) / 4 * 4;
  if (rc == RTE_OK) cu(dalloc(c, &c->d_Wf, (size_t)c->N * c->cpad), "alloc");
  if (rc == RTE_OK) cu(cudaMemset(c->d_Wf, 0, sizeof(float) * (size_t)c->N * c->cpad), "memset");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_islot, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_slot_xyz, c->N), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_err, 1), "alloc");
  if (rc == RTE_OK) cu(cudaMemset(c->d_err, 0, sizeof(int)), "memset");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_cplx, 2 * NC), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_red, 8), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_img, 4 * (size_t)c->nx * c->ny), "alloc");  // trans, ref (complex)
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  if (rc == RTE_OK) cu(dalloc(c, &c->d_fball, npix), "alloc");
  if (rc == RTE_OK) cu(dalloc(c, &c->d_q, NC), "alloc");
  if (rc == RTE_OK) {
    std::vector<int> p = morton_perm(c->nx, c->ny, c->nz);
    std::vector<int> inv(c->N);
    std::vector<float4> xyz(c->N);
    for (int q = 0; q < c->N; q++) {
      const int v = p[q];
      inv[v] = q;
      int bits;
      memcpy(&bits, &v, sizeof bits);
      float w;
      memcpy(&w, &bits, sizeof w);
      xyz[q] = make_float4((float)(v % c->nx), (float)((v / c->nx) % c->ny), (float)(v / (c->nx * c->ny)), w);
    }
    cu(cudaMemcpy(c->d_perm, p.data(), sizeof(int) * c->N, cudaMemcpyHostToDevice), "perm upload");
    if (rc == RTE_OK) cu(cudaMemcpy(c->d_islot, inv.data(), sizeof(int) * c->N, cudaMemcpyHostToDevice), "upload");
    if (rc == RTE_OK)
      cu(cudaMemcpy(c->d_slot_xyz, xyz.data(), sizeof(float4) * c->N, cudaMemcpyHostToDevice), "upload");
  }
  if (rc != RTE_OK) {
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return RTE_OK;
}

void rte_destroy(rte_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->cfg.device);
  cudaStreamSynchronize(c->st);
  free_all(c);
  delete c;
}

const char* rte_last_error(const rte_ctx* c) { return c ? c->err.c_str() : g_create_err.c_str(); }

size_t rte_device_bytes(const rte_ctx* c) { return c ? c->bytes : 0; }

}  // extern "C"

// ---------------------------------------------------------------------------------------
static int ensure_moments(rte_ctx* c, double mumax) {
  const int quad = c->model == RTE_MODEL_FIM ? 0 : 1;
  const int ssv = c->cfg.self_sub_vox;
  if (c->quad.L != c->L || c->quad.quad != quad || c->quad.ssv != ssv)
    build_quad(c->quad, c->L, quad, ssv, c->dx, c->dy, c->dz, c->sh);
  const double x = mumax * c->quad.beta_max;
  // terms until x^(k+1)/(k+1)! is below 1e-18 of the leading term
  int K = 1;
  double term = x;
  while (K < RTE_MAX_MOM && term > 1e-18) {
    term *= x / (K + 1);
    K++;
  }
  if (x > 12.0 || term > 1e-18)
    return fail(c, RTE_ERR_UNSUPPORTED, "self-voxel series: mu_t*voxel = %.3g too large", x);
  K = std::max(K, 4);
  if (K <= c->K && c->d_mom) return RTE_OK;
  std::vector<double>& mom = c->h_mom;
  build_moments(c->quad, K, c->dV, mom);
  if (!c->d_mom)  // room for the longest series, so the table never moves (recorded graphs keep it)
    CUDA_TRY(c, dalloc(c, &c->d_mom, (size_t)RTE_MAX_MOM * c->C * c->C));
  CUDA_TRY(c, cudaMemcpy(c->d_mom, mom.data(), sizeof(double) * mom.size(), cudaMemcpyHostToDevice));
  c->K = K;
  return RTE_OK;
}

// mu_t of the self-voxel term and (mu_t, mu_s) of the source: the medium's, or the split table's
static const double* self_mut(const rte_ctx* c) { return c->split ? c->d_mut_self : c->d_mut; }
static const double* source_mus(const rte_ctx* c) { return c->split ? c->d_mus_src : c->d_mus; }

// Self-voxel matrices D(mu) = sum_k mu^k M_k for each distinct mu_t of the medium (a handful for
// tissue maps and sphere phantoms), and the voxel -> matrix index.  Media with more than 4096
// distinct values use the power series on the device instead.
static int build_self_lut(rte_ctx* c) {
  std::vector<double> mut(c->N);
  CUDA_TRY(c, cudaMemcpyAsync(mut.data(), self_mut(c), sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  std::unordered_map<double, int> id;
  std::vector<int> idx(c->N);
  std::vector<double> vals;
  for (int r = 0; r < c->N; r++) {
    auto it = id.find(mut[r]);
    if (it == id.end()) {
      if (vals.size() >= 4096) {
        c->self_lut_ok = false;
        c->uniform = false;
        return RTE_OK;
      }
      it = id.emplace(mut[r], (int)vals.size()).first;
      vals.push_back(mut[r]);
    }
    idx[r] = it->second;
  }
  const int C = c->C, K = c->K;
  std::vector<double> lut(vals.size() * C * C, 0.0), dlut(vals.size() * C * C, 0.0), lut_im;
  for (size_t q = 0; q < vals.size(); q++) {
    double* D = &lut[q * C * C];
    double* dD = &dlut[q * C * C];
    for (int k = K - 1; k >= 0; k--)  // Horner in mu
      for (int e = 0; e < C * C; e++) D[e] = D[e] * vals[q] + c->h_mom[(size_t)k * C * C + e];
    for (int k = K - 1; k >= 1; k--)  // d/dmu
      for (int e = 0; e < C * C; e++) dD[e] = dD[e] * vals[q] + (double)k * c->h_mom[(size_t)k * C * C + e];
  }
  if (c->kappa != 0.0) {  // D(mu_t + i kappa): Horner in the complex mu
    lut_im.assign(vals.size() * C * C, 0.0);
    for (size_t q = 0; q < vals.size(); q++) {
      double* Dr = &lut[q * C * C];
      double* Di = &lut_im[q * C * C];
      for (int e = 0; e < C * C; e++) Dr[e] = 0.0;
      for (int k = K - 1; k >= 0; k--)
        for (int e = 0; e < C * C; e++) {
          const double nr = Dr[e] * vals[q] - Di[e] * c->kappa + c->h_mom[(size_t)k * C * C + e];
          Di[e] = Dr[e] * c->kappa + Di[e] * vals[q];
          Dr[e] = nr;
        }
    }
    if (lut_im.size() > c->lut_im_cap) {
      if (c->d_self_lut_im) {
        cudaFree(c->d_self_lut_im);
        c->bytes -= c->lut_im_cap * sizeof(double);
        c->d_self_lut_im = nullptr;
      }
      const size_t cap = std::max(lut_im.size(), (size_t)16 * C * C);
      CUDA_TRY(c, dalloc(c, &c->d_self_lut_im, cap));
      c->lut_im_cap = cap;
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->d_self_lut_im, lut_im.data(), sizeof(double) * lut_im.size(),
                                cudaMemcpyHostToDevice, c->st));
  }
  {
    int rc = 0;
    if (dlut.size() > c->dlut_cap) {
      if (c->d_dlut) {
        cudaFree(c->d_dlut);
        c->bytes -= c->dlut_cap * sizeof(double);
        c->d_dlut = nullptr;
      }
      const size_t cap = std::max(dlut.size(), (size_t)16 * C * C);  // headroom: fewer reallocations
      CUDA_TRY(c, dalloc(c, &c->d_dlut, cap));
      c->dlut_cap = cap;
    }
    (void)rc;
    CUDA_TRY(c, cudaMemcpyAsync(c->d_dlut, dlut.data(), sizeof(double) * dlut.size(), cudaMemcpyHostToDevice, c->st));
  }
  if (lut.size() > c->lut_cap) {
    if (c->d_self_lut) {
      cudaFree(c->d_self_lut);
      c->bytes -= c->lut_cap * sizeof(double);
      c->d_self_lut = nullptr;
    }
    const size_t cap = std::max(lut.size(), (size_t)16 * C * C);
    CUDA_TRY(c, dalloc(c, &c->d_self_lut, cap));
    c->lut_cap = cap;
  }
  CUDA_TRY(c, cudaMemcpyAsync(c->d_self_lut, lut.data(), sizeof(double) * lut.size(), cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_self_idx, idx.data(), sizeof(int) * c->N, cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  c->self_lut_ok = true;
  c->uniform = vals.size() == 1 && !c->split;  // a split medium keeps the pair kernels
  c->uniform_mut = vals[0];
  return RTE_OK;
}

// mu_t, mu_s (and the FP32 mu_t) from device arrays; the pair kernel becomes stale.
static int medium_from_device(rte_ctx* c, const double* d_mua, const double* d_mus) {
  CUDA_TRY(c, cudaMemsetAsync(c->d_red + 6, 0, sizeof(double), c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_medium(d_mua, d_mus, c->d_mut, c->d_mus, c->d_mutf, c->N, c->d_red + 6, c->st)));
  double mumax = 0.0;
  CUDA_TRY(c, cudaMemcpyAsync(&mumax, c->d_red + 6, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  c->K_valid = false;
  c->medium_set = true;
  c->split = false;
  c->mumax = mumax;
  int rc = ensure_moments(c, std::hypot(mumax, c->kappa));
  if (rc) return rc;
  return build_self_lut(c);
}

extern "C" int rte_set_medium_voxel(rte_ctx* c, const double* mua, const double* mus) {
  if (!c || !mua || !mus) return fail(c, RTE_ERR_ARG, "null argument");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  for (int r = 0; r < c->N; r++)
    if (!(mua[r] >= 0.0) || !(mus[r] >= 0.0)) return fail(c, RTE_ERR_ARG, "negative or NaN coefficient at voxel %d", r);
  CUDA_TRY(c, cudaMemcpyAsync(c->d_aux1, mua, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_aux2, mus, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
  return medium_from_device(c, c->d_aux1, c->d_aux2);
}

extern "C" int rte_set_medium_device(rte_ctx* c, const double* d_mua, const double* d_mus) {
  if (!c || !d_mua || !d_mus) return fail(c, RTE_ERR_ARG, "null argument");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  return medium_from_device(c, d_mua, d_mus);
}

extern "C" int rte_set_medium_tissue(rte_ctx* c, const uint8_t* tiss, int ntypes, const double* mua,
                                     const double* mus) {
  if (!c || !tiss || !mua || !mus || ntypes <= 0 || ntypes > 256) return fail(c, RTE_ERR_ARG, "bad tissue arguments");
  std::vector<double> a(c->N), s(c->N);
  for (int r = 0; r < c->N; r++) {
    if (tiss[r] >= ntypes) return fail(c, RTE_ERR_ARG, "tissue type %d at voxel %d >= %d", tiss[r], r, ntypes);
    a[r] = mua[tiss[r]];
    s[r] = mus[tiss[r]];
  }
  return rte_set_medium_voxel(c, a.data(), s.data());
}

static int unsupported_modulated(rte_ctx* c, const char* what);

// Two tissue tables on one tissue map, as the FisherInfo_IO SNR and region-gradient mains leave them:
// they change tissue values on the host (self-voxel table, source and images follow) but drop the
// result of populate_info_dev() (rte_snr.cu:239, compute_grad_rte.cu:431), so the device kernels'
// path integrals (compute_propabs) and scatter (prop_scat_dev) keep the .par values.
extern "C" int rte_set_medium_tissue_split(rte_ctx* c, const uint8_t* tiss, int ntypes, const double* mua,
                                           const double* mus, const double* mua_kernel, const double* mus_kernel) {
  if (!c || !tiss || !mua || !mus || !mua_kernel || !mus_kernel || ntypes <= 0 || ntypes > 256)
    return fail(c, RTE_ERR_ARG, "bad tissue arguments");
  if (c->kappa != 0.0) return unsupported_modulated(c, "a split tissue table");
  int rc = rte_set_medium_tissue(c, tiss, ntypes, mua_kernel, mus_kernel);
  if (rc) return rc;
  std::vector<double> t(c->N), sc(c->N);
  double mumax = c->mumax;
  for (int r = 0; r < c->N; r++) {
    if (!(mua[tiss[r]] >= 0.0) || !(mus[tiss[r]] >= 0.0)) return fail(c, RTE_ERR_ARG, "negative or NaN coefficient");
    t[r] = mua[tiss[r]] + mus[tiss[r]];
    sc[r] = mus[tiss[r]];
    mumax = std::max(mumax, t[r]);
  }
  if (!c->d_mut_self) CUDA_TRY(c, dalloc(c, &c->d_mut_self, (size_t)c->N));
  if (!c->d_mus_src) CUDA_TRY(c, dalloc(c, &c->d_mus_src, (size_t)c->N));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_mut_self, t.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_mus_src, sc.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
  c->split = true;
  c->mumax = mumax;
  rc = ensure_moments(c, mumax);
  if (!rc) rc = build_self_lut(c);
  if (rc) c->medium_set = false;
  return rc;
}

// scatter factor per l (prop_scat_dev, FisherInfo_IO/src/kernels.cu:385-418)
static void scatter_factors(const rte_ctx* c, int flag, double* s) {
  for (int l = 0; l <= RTE_MAX_L; l++) {
    if (c->model == RTE_MODEL_FIM) {
      if (flag) {
        // pow(__int2double_rn(g), l): the int parameter truncates g (0.8 -> 0)
        s[l] = (double)(float)c->cm * pow((double)(int)c->cfg.g, (double)l);
      } else {
        s[l] = 1.0;  // flag == 0 (g == 0): out *= mu_s only
      }
    } else {
      s[l] = c->cm * pow(c->cfg.g, (double)l);
    }
  }
}

// The stored pair kernel: FP32 for the mixed method (store or automatic mode), FP64 for the FP64
// method when RTE_KERNEL_STORE asks for it (automatic FP64 contexts keep recomputing: the plain method).
static int ensure_pair_kernel(rte_ctx* c, bool* stored) {
  *stored = false;
  const bool f64 = c->precision == RTE_PREC_FP64;
  if (c->kernel_mode == RTE_KERNEL_RECOMPUTE || (f64 && c->kernel_mode != RTE_KERNEL_STORE)) return RTE_OK;
  const size_t ld = ((size_t)c->N + 31) / 32 * 32;  // 128-byte rows
  const size_t need = f64 ? (size_t)c->N * ld * sizeof(double)
                          : ((size_t)c->N + RTE_KBLK - 1) / RTE_KBLK * RTE_KBLK * ld * sizeof(float);
  if (f64 ? !c->d_K64 : !c->d_K) {
    size_t fr = 0, tot = 0;
    CUDA_TRY(c, cudaMemGetInfo(&fr, &tot));
    if (need + (1ull << 30) > fr) {
      if (c->kernel_mode == RTE_KERNEL_STORE)
        return fail(c, RTE_ERR_NOMEM, "pair kernel needs %.1f GB, %.1f GB free", need / 1e9, fr / 1e9);
      return RTE_OK;  // auto: recompute
    }
    if (f64)
      CUDA_TRY(c, dalloc(c, &c->d_K64, (size_t)c->N * ld));
    else  // whole 128-destination blocks of ld source rows (kmat_index)
      CUDA_TRY(c, dalloc(c, &c->d_K, ((size_t)c->N + RTE_KBLK - 1) / RTE_KBLK * RTE_KBLK * ld));
    c->Kld = ld;
  }
  if (!c->K_valid || c->capture_store) {
    PairArgs a;
    memset(&a, 0, sizeof a);
    a.N = c->N;
    a.nx = c->nx;
    a.ny = c->ny;
    a.nz = c->nz;
    a.Cfull = c->C;
    a.dx = c->dx;
    a.dy = c->dy;
    a.dz = c->dz;
    a.prop_thresh = c->prop_thresh;
    a.kscale = c->dV / c->cm;
    a.perm = c->d_perm;
    a.mut = c->d_mut;
    a.mutf = c->d_mutf;
    a.Kmat = c->d_K;
    a.Kmat64 = c->d_K64;
    a.Kld = c->Kld;
    if (c->capturing) {
      CUDA_TRY(c, rte_launch_store_kernel(a, c->st, f64 ? 1 : 0));
    } else {
      CUDA_TRY(c, cudaEventRecord(c->ev0, c->st));
      {
        ProfScope ps(c, 1);
        CUDA_TRY(c, rte_launch_store_kernel(a, c->st, f64 ? 1 : 0));
      }
      CUDA_TRY(c, cudaEventRecord(c->ev1, c->st));
      CUDA_TRY(c, cudaEventSynchronize(c->ev1));
      float ms = 0;
      cudaEventElapsedTime(&ms, c->ev0, c->ev1);
      c->last_setup_ms = ms;
    }
    c->K_valid = true;
  }
  *stored = true;
  return RTE_OK;
}

// Split-K plan: the number of source chunks S so that tiles x S CTAs fill whole waves of the
// kernel's resident CTAs (a partial last wave idles SMs).
static int check_kernel_err(rte_ctx* c);

// Pair-kernel arguments for nb right-hand sides split S ways (chunk sources per split).
static PairArgs pair_args(const rte_ctx* c, const double* in64, const float* in32, int nb, int S, int chunk) {
  PairArgs a;
  memset(&a, 0, sizeof a);
  a.N = c->N;
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.Cfull = c->C;
  a.dx = c->dx;
  a.dy = c->dy;
  a.dz = c->dz;
  a.prop_thresh = c->prop_thresh;
  a.kscale = c->dV / c->cm;
  a.perm = c->d_perm;
  a.mut = c->d_mut;
  a.mutf = c->d_mutf;
  a.Win = in64;
  a.Winf = in32;
  a.Kmat = c->d_K;
  a.Kmat64 = c->d_K64;
  a.Kld = c->Kld;
  a.part = c->d_part;
  a.partf = reinterpret_cast<float*>(c->d_part);
  a.chunk = chunk;
  a.nsplit = S;
  a.nb = nb;
  a.slot_xyz = c->d_slot_xyz;
  a.cstride = (c->C + 3) / 4 * 4;
  a.cpad = (nb * a.cstride + 3) / 4 * 4;
  a.err = c->d_err;
  a.kappa = c->kappa;
  a.transpose = c->transpose ? 1 : 0;
  return a;
}

static inline int split_chunk(int N, int S) {
  return ((N + S - 1) / S + RTE_PAIR_TS - 1) / RTE_PAIR_TS * RTE_PAIR_TS;
}

// Split-K autotuner.  The pair kernel's grid is (destination tiles) x S source chunks; the best S
// balances wave quantisation on the 148 SMs against the partial-sum traffic of the epilogue and
// depends on N, the order, the right-hand-side count and the kernel variant.  Candidates are the
// splits whose occupancy-model wave fill is within 25% of the best; each is launched on the
// context's own buffers and timed with CUDA events (best of two), and the winner is kept for the
// process (every context of that shape on that device reuses it).  RTE_AUTOTUNE=0 keeps the
// occupancy model's choice; RTE_NSPLIT forces a split.
namespace {
using TuneKey = std::tuple<int, int, int, int, int, int, int>;  // device, N, LA, stored, nb, precision, table
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tuned;  // (S, tile)
struct Plan {
  double fill;  // wave fill of the occupancy model
  int S, tile;
};
}  // namespace

// Launch-plan autotuner: each candidate (split S, source tile) is launched on the context's own buffers
// and timed with CUDA events (best of two); the fastest is kept for the process.
static int tune_split(rte_ctx* c, int LA, int stored, int nb, const std::vector<Plan>& cands, int* S_best,
                      int* tile_best) {
  const int table = c->model == RTE_MODEL_FIM ? 1 : 0;
  const double* in64 = nb == 1 ? c->d_W : c->d_bW;
  const float* in32 = nb == 1 ? c->d_Wf : c->d_bWf;
  if (!in64 || (c->precision == RTE_PREC_MIXED && !in32)) return RTE_OK;
  cudaEvent_t e0, e1;
  CUDA_TRY(c, cudaEventCreate(&e0));
  CUDA_TRY(c, cudaEventCreate(&e1));
  double best = 1e30;
  cudaError_t err = cudaSuccess;
  // each launch is checked with cudaGetLastError: clear what an earlier call of this thread left there
  // (a failure handled where it happened, or one inside a library), so it is not read as a launch's
  (void)cudaGetLastError();
  for (const auto& cand : cands) {
    PairArgs a = pair_args(c, in64, in32, nb, cand.S, split_chunk(c->N, cand.S));
    a.tile = cand.tile;
    float t = 1e30f;
    for (int rep = 0; rep < 2 && err == cudaSuccess; rep++) {
      cudaEventRecord(e0, c->st);
      err = rte_launch_pair(a, LA, c->precision, table, stored, c->st);
      cudaEventRecord(e1, c->st);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0;
      if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
      if (rep == 1 || cands.size() == 1) t = std::min(t, ms);
    }
    c->launches += 2;
    if (err != cudaSuccess) break;
    if (t < best) {
      best = t;
      *S_best = cand.S;
      *tile_best = cand.tile;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return fail(c, RTE_ERR_DEVICE, "launch autotuner: %s", cudaGetErrorString(err));
  return check_kernel_err(c);
}

// The tile-staged stored-kernel launch (mixed precision, exact directions, real right-hand sides: see
// k_pair_mixed_tk) keeps each CTA's FP32 sums in registers over its whole source chunk; chunks of at most
// kTkChunk sources keep those sums short (the epilogue adds the chunks in FP64): 33^3 L=5 error against
// FP64 3.9e-6 with chunks of ~4,500 sources, see the bench line's fp64_rel_err for the capped chunks.
static const int kTkChunk = 1024;
static bool tk_kernel(const rte_ctx* c, int stored, int cplx) {
  return c->precision == RTE_PREC_MIXED && stored && c->model != RTE_MODEL_FIM && !cplx;
}
// The recomputed four-right-hand-side kernel at L >= 6 (k_pair_mixed_grp: two thread groups sharing the
// path walks) leaves FP32 chunk sums as well.
static bool grp_kernel(const rte_ctx* c, int stored, int cplx, int nb, int LA) {
  return c->precision == RTE_PREC_MIXED && !stored && c->model != RTE_MODEL_FIM && !cplx && nb == 4 && LA >= 6;
}

template <class T>
static int grow(rte_ctx* c, T** p, size_t& cap, size_t n);

static int plan_split(rte_ctx* c, int LA, int stored, int nb, int* S_out, int* chunk_out, int* tile_out = nullptr) {
  const int cplx = c->kappa != 0.0 ? 1 : 0;
  const int key = (((LA * 2 + stored) * 8 + nb) * 2 + (c->precision == RTE_PREC_MIXED ? 1 : 0)) * 2 + cplx;
  for (auto& e : c->splits)
    if (e[0] == key) {
      *S_out = e[1];
      *chunk_out = e[2];
      if (tile_out) *tile_out = e[3];
      return RTE_OK;
    }
  const int table = c->model == RTE_MODEL_FIM ? 1 : 0;
  const int cpad = (nb * ((c->C + 3) / 4 * 4) + 3) / 4 * 4;
  int sms = 0;
  CUDA_TRY(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
  const int tiles = (c->N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS;
  const bool tk = tk_kernel(c, stored, cplx);
  const bool chunked = tk || grp_kernel(c, stored, cplx, nb, LA);  // FP32 chunk sums, chunks capped
  const int Smin = chunked ? (c->N + kTkChunk - 1) / kTkChunk : 1;
  const int Smax = chunked ? Smin + c->max_split : c->max_split;
  if (chunked) {  // partial sums of Smax chunks (before any capture: plan_split runs ahead of graph recording)
    int rc = grow(c, &c->d_part, c->part_cap, (size_t)c->N * c->C * nb * Smax);
    if (rc) return rc;
  }
  // occupancy-model candidates: (wave fill, S, tile) for each source tile the kernel offers
  std::vector<Plan> fills;
  Plan model{-1.0, Smin, 0};
  for (int tile = 0; tile < (tk ? 2 : 1); tile++) {
    int occ = 0;
    CUDA_TRY(c, rte_pair_occupancy(LA, c->precision, table, stored, nb, cpad, &occ, cplx, tile));
    const long long slots = (long long)std::max(occ, 1) * sms;
    double best = -1.0;
    int bestS = Smin;
    for (int S = Smin; S <= Smax; S++) {
      const int Sreal = (c->N + split_chunk(c->N, S) - 1) / split_chunk(c->N, S);
      if (Sreal != S) continue;
      const double waves = (double)tiles * S / (double)slots;
      const double eff = waves / ceil(waves);
      fills.push_back({eff, S, tile});
      // prefer the smallest S within 3% of the best fill, and at least one full wave when possible
      if (eff > best + 0.03 || (best < 0.97 && eff > best)) {
        best = eff;
        bestS = S;
      }
    }
    if (tile == 0) model = {best, bestS, 0};
  }
  int bestS = model.S, bestTile = 0;
  const char* forced = getenv("RTE_NSPLIT");
  const char* at = getenv("RTE_AUTOTUNE");
  const bool tune = !forced && !(at && at[0] == '0') && !c->capturing && c->precision == RTE_PREC_MIXED &&
                    c->N >= 4096;
  if (forced) {
    bestS = std::max(Smin, std::min(Smax, atoi(forced)));
  } else if (tune) {
    const TuneKey tk_key{c->cfg.device, c->N, LA, stored, nb, c->precision, table + 2 * cplx};
    bool have = false;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      auto it = g_tuned.find(tk_key);
      if (it != g_tuned.end() && it->second.first <= Smax && it->second.first >= Smin) {
        bestS = it->second.first;
        bestTile = it->second.second;
        have = true;
      }
    }
    if (!have) {
      // per tile: the splits whose wave fill is within 25% of that tile's best, the four best of them
      std::vector<Plan> cands;
      for (int tile = 0; tile < (tk ? 2 : 1); tile++) {
        double best = 0.0;
        for (auto& f : fills)
          if (f.tile == tile) best = std::max(best, f.fill);
        std::vector<Plan> mine;
        for (auto& f : fills)
          if (f.tile == tile && f.fill >= 0.75 * best) mine.push_back(f);
        std::sort(mine.begin(), mine.end(), [](const Plan& x, const Plan& y) {
          return x.fill > y.fill || (x.fill == y.fill && x.S < y.S);
        });
        if (mine.size() > 4) mine.resize(4);
        cands.insert(cands.end(), mine.begin(), mine.end());
      }
      int rc = tune_split(c, LA, stored, nb, cands, &bestS, &bestTile);
      if (rc) return rc;
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tuned[tk_key] = {bestS, bestTile};
    }
  }
  const int chunk = split_chunk(c->N, bestS);
  const int S = (c->N + chunk - 1) / chunk;
  c->splits.push_back({key, S, chunk, bestTile});
  *S_out = S;
  *chunk_out = chunk;
  if (tile_out) *tile_out = bestTile;
  return RTE_OK;
}

// One term on the real basis for nb right-hand sides (layout [N][nb][C]): out = [D] A in.
// in64 is FP64 (and in32 its FP32 copy for the mixed kernels).  sum != null accumulates the result;
// d_red receives the norms.
static const int kMaxBatch = 4;  // right-hand sides of one batched solve

// Uniform media in automatic kernel mode take the convolution path (rte_fft.cpp), outside graph
// capture (the transforms plan and synchronise); RTE_NO_FFT=1 keeps the pair kernels.
static bool fft_eligible(const rte_ctx* c) {
  static const bool off = getenv("RTE_NO_FFT") && getenv("RTE_NO_FFT")[0] == '1';
  return c->uniform && c->kernel_mode == RTE_KERNEL_AUTO && !off && c->kappa == 0.0;
}

// inside a graph capture only when the recording prepared the transforms beforehand
static bool fft_active(const rte_ctx* c) {
  return fft_eligible(c) && !c->transpose && (!c->capturing || c->fft_capture_ready);
}

static int ensure_fft(rte_ctx* c) {
  FftTabArgs a;
  memset(&a, 0, sizeof a);
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.dx = c->dx;
  a.dy = c->dy;
  a.dz = c->dz;
  a.prop_thresh = c->prop_thresh;
  a.kscale = c->dV / c->cm;
  a.mut = c->uniform_mut;
  const bool first = c->fft == nullptr;
  CUDA_TRY(c, rte_fft_prepare(&c->fft, a, c->L, c->model == RTE_MODEL_FIM ? 1 : 0, kMaxBatch, c->st));
  if (first) c->bytes += rte_fft_bytes(c->nx, c->ny, c->nz, c->L, kMaxBatch);
  return RTE_OK;
}

static int apply_term(rte_ctx* c, const double* in64, const float* in32, double* out, float* out32, double* sum,
                      int flag, int flag_scat, int nb = 1) {
  const int LA = flag ? c->L : 0;
  int S = 1, chunk = c->N;
  bool f32part = false;  // the tile-staged kernel leaves FP32 chunk sums
  int rc;
  if (fft_active(c)) {
    rc = ensure_fft(c);
    if (rc) return rc;
    ProfScope ps(c, 0);
    CUDA_TRY(c, (c->launches += 5, rte_fft_apply(c->fft, in64, nb * c->C, c->C, LA, nb, c->d_part, c->st)));
  } else {
    bool stored = false;
    rc = ensure_pair_kernel(c, &stored);
    if (rc) return rc;
    int tile = 0;
    rc = plan_split(c, LA, stored ? 1 : 0, nb, &S, &chunk, &tile);
    if (rc) return rc;
    PairArgs a = pair_args(c, in64, in32, nb, S, chunk);
    a.tile = tile;
    f32part = tk_kernel(c, stored ? 1 : 0, c->kappa != 0.0 ? 1 : 0) ||
              grp_kernel(c, stored ? 1 : 0, c->kappa != 0.0 ? 1 : 0, nb, LA);
    ProfScope ps(c, 0);
    CUDA_TRY(c, rte_launch_pair(a, LA, c->precision, c->model == RTE_MODEL_FIM ? 1 : 0, stored ? 1 : 0, c->st));
  }
  SelfArgs sa;
  memset(&sa, 0, sizeof sa);
  sa.N = c->N;
  sa.nb = nb;
  sa.Cfull = c->C;
  sa.Cact = (LA + 1) * (LA + 1);
  sa.K = c->K;
  sa.W = in64;
  sa.mut = self_mut(c);
  sa.idx = c->self_lut_ok ? c->d_self_idx : nullptr;
  sa.lut = c->d_self_lut;
  sa.mom = c->d_mom;
  sa.scale = c->dV / c->cm;
  sa.air_no_self = c->model == RTE_MODEL_FIM ? 1 : 0;
  sa.out = c->d_selfp;
  sa.kappa = c->kappa;
  sa.lut_im = c->d_self_lut_im;
  if (c->kappa != 0.0 && nb % 2) return fail(c, RTE_ERR_STATE, "a modulated term needs (real, imaginary) row pairs");
  if (LA < c->L) CUDA_TRY(c, cudaMemsetAsync(c->d_selfp, 0, (size_t)c->N * nb * c->C * sizeof(double), c->st));
  {
    ProfScope ps(c, 2);
    CUDA_TRY(c, rte_launch_self(sa, c->st));
  }
  EpiArgs e;
  memset(&e, 0, sizeof e);
  e.N = c->N;
  e.nx = c->nx;
  e.ny = c->ny;
  e.nz = c->nz;
  e.Cfull = c->C;
  e.S = S;
  e.nb = nb;
  e.part = c->d_part;
  e.partf = f32part ? reinterpret_cast<const float*>(c->d_part) : nullptr;
  e.selfp = c->d_selfp;
  e.mus = c->d_mus;
  e.flag_scat = flag_scat;
  scatter_factors(c, flag, e.scat);
  e.Wout = out;
  e.Woutf = out32;
  e.islot = c->d_islot;
  e.cstride = (c->C + 3) / 4 * 4;
  e.cpad = (nb * e.cstride + 3) / 4 * 4;
  e.sum = sum;
  e.red = c->d_red;
  e.cplx = c->kappa != 0.0 ? 1 : 0;
  CUDA_TRY(c, cudaMemsetAsync(c->d_red, 0, 4 * sizeof(double), c->st));
  {
    ProfScope ps(c, 2);
    CUDA_TRY(c, rte_launch_epilogue(e, LA, c->st));
  }
  return RTE_OK;
}

// A pair kernel whose bounded wait ran out leaves its result invalid and raises d_err.
static int check_kernel_err(rte_ctx* c) {
  int h = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  if (h) {
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    return fail(c, RTE_ERR_TIMEOUT, "a pair kernel's wait for its shared-memory tile ran out");
  }
  return RTE_OK;
}

// Neumann series on one real part.  W0 (FP64 real) is the first term, S0 the initial running
// sum; the result A * sum is written to `res`.  rule/max_terms/tol as rte_stop.  When force_terms
// >= 0 exactly that many terms are taken (used for the second real part of complex input).
static int neumann_real(rte_ctx* c, const double* W0, const double* S0, double* res, int flag, const rte_stop* stop,
                        int force_terms, int* nterms, double* last_rel) {
  const size_t NC = (size_t)c->N * c->C;
  const bool mixed = c->precision == RTE_PREC_MIXED;
  CUDA_TRY(c, cudaMemcpyAsync(c->d_sum, S0, NC * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  int terms = 0;
  double rel = 0.0;
  if (flag) {
    CUDA_TRY(c, cudaMemcpyAsync(c->d_W, W0, NC * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    if (mixed) CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_W, c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C, c->cstride, c->st)));
    const int flag_l = c->cfg.g != 0.0 ? 1 : 0;  // neumann.cu:74-79
    const int rule = force_terms >= 0 ? RTE_STOP_FIXED : stop->rule;
    const int maxt = force_terms >= 0 ? force_terms : (rule == RTE_STOP_REFERENCE ? 10000 : stop->max_terms);
    int n = c->model == RTE_MODEL_CPU ? 1 : 2;  // CPU package starts n at 1, FIM at 2
    double fi = 1.0;
    double hred[4] = {0, 0, 0, 0};
    if (rule == RTE_STOP_REFERENCE) {
      CUDA_TRY(c, cudaMemsetAsync(c->d_red, 0, 4 * sizeof(double), c->st));
      CUDA_TRY(c, (c->launches++, rte_launch_layer_sums(c->d_W, c->d_sum, c->N, c->nx, c->ny, c->nz, c->C, c->d_red, c->st)));
      CUDA_TRY(c, cudaMemcpyAsync(hred, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      CUDA_TRY(c, cudaStreamSynchronize(c->st));
    }
    for (;;) {
      if (rule == RTE_STOP_REFERENCE) {
        // StopIteration (dist.cu:1132-1172) on the layer sums of W and the running sum
        const double sumW = hred[2], sumOut = hred[3];
        double hi = 0.0;
        bool stopnow = false;
        if (n > 1) {
          if (sumOut == 0.0) {
            stopnow = true;
          } else {
            hi = 1.0 - (sumW / sumOut) * (1.0 / (1.0 - (sumW / sumOut) / fi));
            fi = sumW / sumOut;
            if (hi > 1.0 || hi < 0.0) hi = 0.0;
          }
        }
        if (stopnow || hi > 0.9999 || terms >= maxt) break;
      } else if (terms >= maxt) {
        break;
      }
      n++;
      int rc = apply_term(c, c->d_W, c->d_Wf, c->d_Wn, mixed ? c->d_Wf : nullptr, c->d_sum, flag_l, 1);
      if (rc) return rc;
      std::swap(c->d_W, c->d_Wn);
      terms++;
      if (rule != RTE_STOP_FIXED) {
        CUDA_TRY(c, cudaMemcpyAsync(hred, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CUDA_TRY(c, cudaStreamSynchronize(c->st));
        rel = hred[1] > 0 ? sqrt(hred[0] / hred[1]) : 0.0;
        if (rule == RTE_STOP_REL_L2 && rel < stop->tol) break;
      }
    }
  }
  // final A on the running sum (no scatter), neumann.cu:95-118
  float* in32 = nullptr;
  if (mixed) {
    CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_sum, c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C, c->cstride, c->st)));
    in32 = c->d_Wf;
  }
  int rc = apply_term(c, c->d_sum, in32, res, nullptr, nullptr, 1, 0);
  if (rc) return rc;
  rc = check_kernel_err(c);
  if (rc) return rc;
  if (nterms) *nterms = terms;
  if (last_rel) *last_rel = rel;
  return RTE_OK;
}

// complex (host) -> real parts on the device; returns whether the second (imaginary-function)
// part is non-zero.
static int upload_cplx(rte_ctx* c, const rte_cplx* h, double* u1, double* u2, bool* has2) {
  const size_t NC = (size_t)c->N * c->C;
  CUDA_TRY(c, cudaMemcpyAsync(c->d_cplx, h, NC * sizeof(rte_cplx), cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_red + 4, 0, sizeof(double), c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_to_real(c->d_cplx, u1, u2, c->N, c->L, c->d_red + 4, c->st)));
  double n2 = 0;
  CUDA_TRY(c, cudaMemcpyAsync(&n2, c->d_red + 4, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  *has2 = n2 > 0.0;
  return RTE_OK;
}

static int download_cplx(rte_ctx* c, const double* u1, const double* u2, rte_cplx* h) {
  const size_t NC = (size_t)c->N * c->C;
  CUDA_TRY(c, (c->launches++, rte_launch_to_cplx(u1, u2, c->d_cplx, c->N, c->L, c->st)));
  CUDA_TRY(c, cudaMemcpyAsync(h, c->d_cplx, NC * sizeof(rte_cplx), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Intensity modulation (CPU package/src/RTE_uniform.c:120-176): mu_a -> mu_a + i modulation/(c/n)
// in every voxel, so mu_t gains the uniform imaginary part kappa and the radiance is complex.  A
// complex distribution w = w1 + i w2 (w1, w2 coefficient sets of real functions) lives on the
// device as (real, imaginary) row pairs per voxel, [N][2][C] in the batch buffers; the pair kernels
// apply k exp(-i kappa r) to the pair, the self term D(mu_t + i kappa), the scatter acts on both rows.
static int ensure_batch(rte_ctx* c, int nb);

static int upload_pair(rte_ctx* c, const rte_cplx* h, double* d_pair) {
  const size_t NC = (size_t)c->N * c->C;
  CUDA_TRY(c, cudaMemcpyAsync(c->d_cplx, h, NC * sizeof(rte_cplx), cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_to_real(c->d_cplx, d_pair, d_pair + c->C, c->N, c->L, nullptr, c->st,
                                                 2 * c->C)));
  return RTE_OK;
}

static int download_pair(rte_ctx* c, const double* d_pair, rte_cplx* h) {
  const size_t NC = (size_t)c->N * c->C;
  CUDA_TRY(c, (c->launches++, rte_launch_to_cplx(d_pair, d_pair + c->C, c->d_cplx, c->N, c->L, c->st, 2 * c->C)));
  CUDA_TRY(c, cudaMemcpyAsync(h, c->d_cplx, NC * sizeof(rte_cplx), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  return RTE_OK;
}

// Neumann series of one complex right-hand side: first term in d_bW, initial running sum in d_bsum
// (row pairs); A * sum to d_bres.  Stop rules as neumann_real (the reference rule on the real parts
// of the complex-basis layer sums, as StopIteration takes creal, Kernels_selfsub.c:1184-1220).
static int neumann_cplx(rte_ctx* c, int flag, const rte_stop* stop, int* nterms, double* last_rel) {
  const int vs = 2 * c->C, cp = (2 * c->cstride + 3) / 4 * 4;
  const bool mixed = c->precision == RTE_PREC_MIXED;
  int terms = 0;
  double rel = 0.0;
  if (flag) {
    if (mixed)
      CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_bW, c->d_bWf, c->d_islot, c->N, vs, cp, c->C,
                                                          c->cstride, c->st)));
    const int flag_l = c->cfg.g != 0.0 ? 1 : 0;
    const int rule = stop->rule;
    const int maxt = rule == RTE_STOP_REFERENCE ? 10000 : stop->max_terms;
    int n = c->model == RTE_MODEL_CPU ? 1 : 2;
    double fi = 1.0;
    double hred[4] = {0, 0, 0, 0};
    if (rule == RTE_STOP_REFERENCE) {
      CUDA_TRY(c, cudaMemsetAsync(c->d_red, 0, 4 * sizeof(double), c->st));
      CUDA_TRY(c, (c->launches++, rte_launch_layer_sums(c->d_bW, c->d_bsum, c->N, c->nx, c->ny, c->nz, c->C, c->d_red,
                                                        c->st, 1)));
      CUDA_TRY(c, cudaMemcpyAsync(hred, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      CUDA_TRY(c, cudaStreamSynchronize(c->st));
    }
    for (;;) {
      if (rule == RTE_STOP_REFERENCE) {
        const double sumW = hred[2], sumOut = hred[3];
        double hi = 0.0;
        bool stopnow = false;
        if (n > 1) {
          if (sumOut == 0.0) {
            stopnow = true;
          } else {
            hi = 1.0 - (sumW / sumOut) * (1.0 / (1.0 - (sumW / sumOut) / fi));
            fi = sumW / sumOut;
            if (hi > 1.0 || hi < 0.0) hi = 0.0;
          }
        }
        if (stopnow || hi > 0.9999 || terms >= maxt) break;
      } else if (terms >= maxt) {
        break;
      }
      n++;
      int rc = apply_term(c, c->d_bW, c->d_bWf, c->d_bWn, mixed ? c->d_bWf : nullptr, c->d_bsum, flag_l, 1, 2);
      if (rc) return rc;
      std::swap(c->d_bW, c->d_bWn);
      terms++;
      if (rule != RTE_STOP_FIXED) {
        CUDA_TRY(c, cudaMemcpyAsync(hred, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CUDA_TRY(c, cudaStreamSynchronize(c->st));
        rel = hred[1] > 0 ? sqrt(hred[0] / hred[1]) : 0.0;
        if (rule == RTE_STOP_REL_L2 && rel < stop->tol) break;
      }
    }
  }
  if (mixed)
    CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_bsum, c->d_bWf, c->d_islot, c->N, vs, cp, c->C,
                                                        c->cstride, c->st)));
  int rc = apply_term(c, c->d_bsum, c->d_bWf, c->d_bres, nullptr, nullptr, 1, 0, 2);
  if (!rc) rc = check_kernel_err(c);
  if (rc) return rc;
  if (nterms) *nterms = terms;
  if (last_rel) *last_rel = rel;
  return RTE_OK;
}

extern "C" int rte_set_modulation(rte_ctx* c, double modulation) {
  if (!c) return fail(c, RTE_ERR_ARG, "null argument");
  if (!std::isfinite(modulation)) return fail(c, RTE_ERR_ARG, "modulation must be finite");
  if (modulation != 0.0 && c->model == RTE_MODEL_FIM)
    return fail(c, RTE_ERR_UNSUPPORTED, "intensity modulation takes the exact or the CPU-package model");
  if (modulation != 0.0 && c->split) return fail(c, RTE_ERR_UNSUPPORTED, "intensity modulation of a split tissue table");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  const double kappa = modulation / c->cm;  // mu_a + i modulation / (c/n), RTE_uniform.c:129
  if (kappa != 0.0 && !c->d_fball_im) {
    const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
    CUDA_TRY(c, dalloc(c, &c->d_fball_im, npix));
  }
  if (kappa == c->kappa) {
    c->modulation = modulation;
    return RTE_OK;
  }
  const double old_mod = c->modulation, old_kappa = c->kappa;
  c->modulation = modulation;
  c->kappa = kappa;
  if (c->medium_set) {
    int rc = ensure_moments(c, std::hypot(c->mumax, c->kappa));
    if (!rc) rc = build_self_lut(c);
    if (rc) {  // keep the context consistent: back to the previous modulation and its self-term table
      const std::string msg = c->err;
      c->modulation = old_mod;
      c->kappa = old_kappa;
      if (build_self_lut(c) != RTE_OK) c->medium_set = false;
      c->err = msg;
      return rc;
    }
  }
  return RTE_OK;
}

static int unsupported_modulated(rte_ctx* c, const char* what) {
  return fail(c, RTE_ERR_UNSUPPORTED, "%s is not available under intensity modulation (rte_set_modulation 0)", what);
}

extern "C" int rte_prop_abs(rte_ctx* c, const rte_cplx* in, rte_cplx* out, int flag, int flag_scat) {
  if (!c || !in || !out) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  if (c->kappa != 0.0) {  // complex operator on the (real, imaginary) pair
    int rc = ensure_batch(c, 2);
    if (!rc) rc = upload_pair(c, in, c->d_bW);
    if (rc) return rc;
    if (c->precision == RTE_PREC_MIXED)
      CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_bW, c->d_bWf, c->d_islot, c->N, 2 * c->C,
                                                          (2 * c->cstride + 3) / 4 * 4, c->C, c->cstride, c->st)));
    rc = apply_term(c, c->d_bW, c->d_bWf, c->d_bres, nullptr, nullptr, flag, flag_scat, 2);
    if (!rc) rc = check_kernel_err(c);
    if (rc) return rc;
    return download_pair(c, c->d_bres, out);
  }
  bool has2 = false;
  int rc = upload_cplx(c, in, c->d_aux1, c->d_aux2, &has2);
  if (rc) return rc;
  const size_t NC = (size_t)c->N * c->C;
  const bool mixed = c->precision == RTE_PREC_MIXED;
  // part 1 -> d_W, part 2 -> d_sum (both scratch here)
  if (mixed) CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_aux1, c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C, c->cstride, c->st)));
  rc = apply_term(c, c->d_aux1, c->d_Wf, c->d_W, nullptr, nullptr, flag, flag_scat);
  if (rc) return rc;
  if (has2) {
    if (mixed) CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_aux2, c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C, c->cstride, c->st)));
    rc = apply_term(c, c->d_aux2, c->d_Wf, c->d_sum, nullptr, nullptr, flag, flag_scat);
    if (rc) return rc;
  }
  rc = check_kernel_err(c);
  if (rc) return rc;
  return download_cplx(c, c->d_W, has2 ? c->d_sum : nullptr, out);
}

// out = A^H in: the adjoint of prop_abs without scatter.  In the real basis A^T = P A P (P = (-1)^l) for
// exact directions; the table model applies its transposed pair kernels (see adjoint_series).
extern "C" int rte_prop_abs_adjoint(rte_ctx* c, const rte_cplx* in, rte_cplx* out, int flag) {
  if (!c || !in || !out) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (c->kappa != 0.0) return unsupported_modulated(c, "the adjoint operator");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  bool has2 = false;
  int rc = upload_cplx(c, in, c->d_aux1, c->d_aux2, &has2);
  if (rc) return rc;
  const bool mixed = c->precision == RTE_PREC_MIXED, table = c->model == RTE_MODEL_FIM;
  double* parts[2] = {c->d_aux1, c->d_aux2};
  double* res[2] = {c->d_W, c->d_sum};
  for (int k = 0; k < (has2 ? 2 : 1) && !rc; k++) {
    if (!table) CUDA_TRY(c, (c->launches++, rte_launch_parity(parts[k], c->N, c->L, c->C, c->st)));
    if (mixed)
      CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(parts[k], c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C,
                                                          c->cstride, c->st)));
    c->transpose = table;
    rc = apply_term(c, parts[k], c->d_Wf, res[k], nullptr, nullptr, flag, 0);
    c->transpose = false;
    if (!rc && !table) CUDA_TRY(c, (c->launches++, rte_launch_parity(res[k], c->N, c->L, c->C, c->st)));
  }
  if (!rc) rc = check_kernel_err(c);
  if (rc) return rc;
  return download_cplx(c, c->d_W, has2 ? c->d_sum : nullptr, out);
}

extern "C" int rte_neumann(rte_ctx* c, const rte_cplx* src, rte_cplx* out, int flag, const rte_stop* stop,
                           int* nterms) {
  if (!c || !out || (flag && (!src || !stop))) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  if (c->kappa != 0.0) {  // one complex series: src -> first term, out -> initial sum
    int rc = ensure_batch(c, 2);
    if (!rc) rc = upload_pair(c, out, c->d_bsum);
    if (!rc && flag) rc = upload_pair(c, src, c->d_bW);
    int terms = 0;
    if (!rc) rc = neumann_cplx(c, flag, stop, &terms, nullptr);
    if (!rc) rc = download_pair(c, c->d_bres, out);
    if (rc) return rc;
    if (nterms) *nterms = terms;
    return RTE_OK;
  }
  // real parts: src -> (aux1, aux2), out -> (aux3, aux4); each Neumann copies its inputs
  // into its own work buffers first, so the result of part k overwrites the input sum of part k.
  bool o_has2 = false, s_has2 = false;
  int rc = upload_cplx(c, out, c->d_aux3, c->d_aux4, &o_has2);
  if (rc) return rc;
  if (flag) {
    rc = upload_cplx(c, src, c->d_aux1, c->d_aux2, &s_has2);
    if (rc) return rc;
  }
  int terms = 0;
  double rel = 0;
  rc = neumann_real(c, c->d_aux1, c->d_aux3, c->d_aux3, flag, stop, -1, &terms, &rel);
  if (rc) return rc;
  const bool has2 = o_has2 || s_has2;
  if (has2) {
    rc = neumann_real(c, c->d_aux2, c->d_aux4, c->d_aux4, flag, stop, terms, nullptr, nullptr);
    if (rc) return rc;
  }
  rc = download_cplx(c, c->d_aux3, has2 ? c->d_aux4 : nullptr, out);
  if (rc) return rc;
  if (nterms) *nterms = terms;
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Sources (real basis: the beam is m = 0 only, where both bases coincide).
// In-face pixel of a face position: z faces (x, y) -> j*nx + k; y faces (x, z) -> i*nx + k;
// x faces (y, z) -> i*ny + j.
static int face_pixel_of(const rte_ctx* c, int face, double px, double py, double pz) {
  auto idx = [](double p, double lo, double d, int n) {
    int v = (int)floor((p - lo) / d);
    return std::min(std::max(v, 0), n - 1);
  };
  const int k = idx(px, c->cfg.x_min, c->dx, c->nx), j = idx(py, c->cfg.y_min, c->dy, c->ny),
            i = idx(pz, c->cfg.z_min, c->dz, c->nz);
  if (face < 2) return j * c->nx + k;
  if (face < 4) return i * c->nx + k;
  return i * c->ny + j;
}

// Beam columns (entry-face pixels) and amplitude scale of a source.
static int source_columns(const rte_ctx* c, const rte_source* s, std::vector<int>& cols, double& scale) {
  cols.clear();
  scale = 1.0;
  if (s->kind == RTE_SRC_FIM) {
    // k == nX/2.0 && j == nY/2.0 (dist.cu:76): no column for odd grids
    if (c->nx % 2 == 0 && c->ny % 2 == 0) cols.push_back((c->ny / 2) * c->nx + c->nx / 2);
    return RTE_OK;
  }
  if (s->kind == RTE_SRC_CPU) {
    for (int j = 0; j < c->ny; j++)
      for (int k = 0; k < c->nx; k++) {
        const double xs = (double)k * c->dx + c->cfg.x_min + c->dx / 2.0;
        const double ys = (double)j * c->dy + c->cfg.y_min + c->dy / 2.0;
        const double rad = sqrt((xs - s->pos_x) * (xs - s->pos_x) + (ys - s->pos_y) * (ys - s->pos_y));
        if (rad <= (s->diam + 1.0e-16) / 2.0) cols.push_back(j * c->nx + k);
      }
    if (!cols.empty()) scale = s->mag / (double)cols.size();
    return RTE_OK;
  }
  if (s->kind == RTE_SRC_COLUMN) {
    cols.push_back(face_pixel_of(c, 0, s->pos_x, s->pos_y, s->pos_z));
    scale = s->mag;
    return RTE_OK;
  }
  if (s->kind == RTE_SRC_BEAM || s->kind == RTE_SRC_POINT) {
    if (s->face < 0 || s->face > 5) return RTE_ERR_ARG;
    cols.push_back(face_pixel_of(c, s->face, s->pos_x, s->pos_y, s->pos_z));
    scale = s->mag;
    return RTE_OK;
  }
  return RTE_ERR_ARG;
}

static inline int source_face(const rte_source* s) {
  return (s->kind == RTE_SRC_BEAM || s->kind == RTE_SRC_POINT) ? s->face : 0;
}

// voxel of face pixel p at depth t behind face f
static int face_voxel(const rte_ctx* c, int f, int p, int t) {
  const int plane = c->nx * c->ny;
  if (f < 2) return (f == 0 ? t : c->nz - 1 - t) * plane + p;
  if (f < 4) {
    const int i = p / c->nx, k = p % c->nx, j = f == 2 ? t : c->ny - 1 - t;
    return i * plane + j * c->nx + k;
  }
  const int i = p / c->ny, j = p % c->ny, k = f == 4 ? t : c->nx - 1 - t;
  return i * plane + j * c->nx + k;
}

// Source terms of one right-hand side, built on the device into d_dst (real basis, rows vstride
// apart): beams put xi = D A xi_beam on their column (dist.cu:66-101; Dist.c:1077-1128 for
// RTE_SRC_CPU) and their ballistic exitant flux in d_fball; a point source puts its isotropic
// emission q into d_q (its uncollided and scattered orders follow from the series).
// HG scatter of a collimated beam entering through `face`: coefficient scale g^l R_lm(d), d the
// face's inward normal (the z = 0 face's m = 0 values written in closed form, dist.cu:86-92)
static void beam_coefs(const rte_ctx* c, int face, double scale, double* coef) {
  const double dirs[6][3] = {{0, 0, 1}, {0, 0, -1}, {0, 1, 0}, {0, -1, 0}, {1, 0, 0}, {-1, 0, 0}};
  std::vector<double> R(c->C);
  sh_real_host(c->sh, c->L, dirs[face][0], dirs[face][1], dirs[face][2], R.data());
  for (int l = 0, q = 0; l <= c->L; l++)
    for (int m = -l; m <= l; m++, q++) {
      double v = scale * pow(c->cfg.g, (double)l) * R[q];
      if (m == 0 && face == 0) v = scale * pow(c->cfg.g, (double)l) * sqrt((2.0 * l + 1.0) / (4.0 * M_PI));
      coef[q] = fabs(v) < 1e-300 ? 0.0 : v;
    }
}

// Under intensity modulation (c->kappa != 0) the attenuation is complex: d_dst holds (real, imaginary)
// row pairs (vstride >= 2 C) and the ballistic flux's imaginary part goes to d_fball_im.
static int launch_source(rte_ctx* c, const rte_source* s, double* d_dst, int vstride = 0, double* d_fball = nullptr,
                         bool zero = true, double* d_q = nullptr, double* d_fball_im = nullptr) {
  if (s->modulation != 0.0 && s->modulation != c->modulation)
    return fail(c, RTE_ERR_STATE, "source modulation %g differs from the context's %g (rte_set_modulation)",
                s->modulation, c->modulation);
  std::vector<int> cols;
  double scale;
  if (source_columns(c, s, cols, scale)) return fail(c, RTE_ERR_ARG, "bad source kind %d / face %d", s->kind, s->face);
  if ((int)cols.size() > RTE_MAX_SRC_COLS) return fail(c, RTE_ERR_UNSUPPORTED, "beam covers more than %d columns", RTE_MAX_SRC_COLS);
  if (vstride <= 0) vstride = c->C;
  const bool cplx = c->kappa != 0.0;
  if (cplx && vstride < 2 * c->C) return fail(c, RTE_ERR_STATE, "a modulated source needs (real, imaginary) row pairs");
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  if (!d_fball) d_fball = c->d_fball;
  if (cplx && !d_fball_im) d_fball_im = c->d_fball_im;
  if (zero) {
    CUDA_TRY(c, cudaMemsetAsync(d_dst, 0, (size_t)c->N * vstride * sizeof(double), c->st));
    CUDA_TRY(c, cudaMemsetAsync(d_fball, 0, npix * sizeof(double), c->st));
    if (cplx) CUDA_TRY(c, cudaMemsetAsync(d_fball_im, 0, npix * sizeof(double), c->st));
  }
  if (cols.empty()) return RTE_OK;
  if (s->kind == RTE_SRC_POINT) {
    if (!d_q) return fail(c, RTE_ERR_UNSUPPORTED, "point sources are not available in this call");
    const int r0 = face_voxel(c, s->face, cols[0], 0);
    const double q = s->mag / (sqrt(4.0 * M_PI) * c->dV);  // isotropic: w_00 = I sqrt(4 pi), I = mag/(4 pi dV)
    CUDA_TRY(c, cudaMemcpyAsync(d_q + (size_t)r0 * vstride, &q, sizeof(double), cudaMemcpyHostToDevice, c->st));
    c->has_point = true;
    return RTE_OK;
  }
  SrcArgs a;
  memset(&a, 0, sizeof a);
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.Cfull = c->C;
  a.L = c->L;
  a.kind = s->kind;
  a.face = source_face(s);
  a.ncols = (int)cols.size();
  for (size_t q = 0; q < cols.size(); q++) a.cols[q] = cols[q];
  beam_coefs(c, a.face, scale, a.coef);
  a.scale = scale;
  a.mag = s->mag;
  a.dlen = a.face < 2 ? c->dz : (a.face < 4 ? c->dy : c->dx);
  a.dV = c->dV;
  a.z_min = c->cfg.z_min;
  a.dz = c->dz;
  a.vstride = vstride;
  a.mut = self_mut(c);
  a.mus = source_mus(c);
  a.W = d_dst;
  a.fball = d_fball;
  a.kappa = c->kappa;
  a.fball_im = cplx ? d_fball_im : nullptr;
  CUDA_TRY(c, (c->launches++, rte_launch_source(a, c->st)));
  return RTE_OK;
}

// per-l image weights and the ballistic pixel (dist.cu:103-161, 229-268; Dist.c:134-229)
static int image_weights(rte_ctx* c, const rte_source* s, ImgArgs& a) {
  memset(a.wt, 0, sizeof a.wt);
  memset(a.wr, 0, sizeof a.wr);
  const double mag = s ? s->mag : 1.0;
  if (c->model == RTE_MODEL_FIM) {
    const double fac = 2.0 * M_PI * 1.0 * c->dx * c->dy / sqrt(4.0 * M_PI);
    for (int l = 0; l <= c->L; l++) {
      double w = 0;
      for (int q = 0; q < 100; q++) {
        const double u = (double)q / (100 - 1.0);
        w += sqrt(2.0 * l + 1.0) * legendre(l, u) * u / (100 - 1.0);
      }
      a.wt[l] = fac * w;
      a.wr[l] = fac * w * mag;
    }
  } else if (c->model == RTE_MODEL_CPU) {
    const double fac = 2.0 * M_PI * c->dx * c->dy * c->cm / sqrt(4.0 * M_PI);
    for (int l = 0; l <= c->L; l++) {
      double w = 0, v = 0;
      for (int q = 0; q < 100; q++) {
        const double u = (double)q / 100.0, u2 = (double)q / 100.0 - 1.0;
        w += sqrt(2.0 * l + 1.0) * legendre(l, u) * u / 100.0;
        v -= sqrt(2.0 * l + 1.0) * legendre(l, u2) * u2 / 100.0;
      }
      a.wt[l] = fac * w;
      a.wr[l] = fac * v;
    }
  } else {
    const double fac = 2.0 * M_PI * c->dx * c->dy * c->cm / sqrt(4.0 * M_PI);
    std::vector<double> x, w;
    gauss01(24, x, w);
    for (int l = 0; l <= c->L; l++) {
      double t = 0, f = 0;
      for (size_t q = 0; q < x.size(); q++) {
        t += sqrt(2.0 * l + 1.0) * legendre(l, x[q]) * x[q] * w[q];
        f += sqrt(2.0 * l + 1.0) * legendre(l, -x[q]) * x[q] * w[q];
      }
      a.wt[l] = fac * t;
      a.wr[l] = fac * f;
    }
  }
  return RTE_OK;
}

// images of a real-basis distribution on the device; with_ball adds the ballistic term left in
// d_ball by the last launch_source.
static int run_images(rte_ctx* c, const double* d_out, const rte_source* s, bool with_ball, rte_cplx* trans,
                      rte_cplx* ref, int vstride = 0, const double* d_fball = nullptr, const double* d_out_im = nullptr,
                      const double* d_fball_im = nullptr) {
  ImgArgs a;
  memset(&a, 0, sizeof a);
  a.nx = c->nx;
  a.ny = c->ny;
  a.nz = c->nz;
  a.Cfull = c->C;
  a.L = c->L;
  a.vstride = vstride > 0 ? vstride : c->C;
  a.out = d_out;
  int rc = image_weights(c, s, a);
  if (rc) return rc;
  const size_t np = (size_t)c->nx * c->ny;
  a.fball = with_ball ? (d_fball ? d_fball : c->d_fball) : nullptr;
  a.fball_im = with_ball ? d_fball_im : nullptr;
  a.out_im = d_out_im;
  a.trans = c->d_img;
  a.ref = c->d_img + 2 * np;
  CUDA_TRY(c, (c->launches++, rte_launch_images(a, c->st)));
  if (trans) CUDA_TRY(c, cudaMemcpyAsync(trans, a.trans, np * sizeof(rte_cplx), cudaMemcpyDeviceToHost, c->st));
  if (ref) CUDA_TRY(c, cudaMemcpyAsync(ref, a.ref, np * sizeof(rte_cplx), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  return RTE_OK;
}

extern "C" int rte_source_beam(rte_ctx* c, const rte_source* s, rte_cplx* xi) {
  if (!c || !s || !xi) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  if (c->kappa != 0.0) {
    int rc = ensure_batch(c, 2);
    if (!rc) rc = launch_source(c, s, c->d_bW, 2 * c->C);
    if (rc) return rc;
    return download_pair(c, c->d_bW, xi);
  }
  int rc = launch_source(c, s, c->d_aux1);
  if (rc) return rc;
  return download_cplx(c, c->d_aux1, nullptr, xi);
}

extern "C" int rte_images(rte_ctx* c, const rte_cplx* out, const rte_source* s, rte_cplx* trans, rte_cplx* ref) {
  if (!c || !out) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  int rc;
  if (c->kappa != 0.0) {  // complex ballistic term and both parts of the distribution in one pass
    rc = ensure_batch(c, 2);
    if (!rc && s) rc = launch_source(c, s, c->d_bW, 2 * c->C, nullptr, true, c->d_bq);
    bool has2 = false;
    if (!rc) rc = upload_cplx(c, out, c->d_aux1, c->d_aux2, &has2);
    if (rc) return rc;
    return run_images(c, c->d_aux1, s, s != nullptr, trans, ref, 0, nullptr, c->d_aux2, c->d_fball_im);
  }
  if (s) {  // ballistic term of this source (the source itself goes to scratch)
    rc = launch_source(c, s, c->d_aux3, 0, nullptr, true, c->d_aux4);
    if (rc) return rc;
  }
  bool has2 = false;
  rc = upload_cplx(c, out, c->d_aux1, c->d_aux2, &has2);
  if (rc) return rc;
  rc = run_images(c, c->d_aux1, s, s != nullptr, trans, ref);
  if (rc || !has2) return rc;
  // imaginary-function part: its images go to the imaginary component
  const size_t np = (size_t)c->nx * c->ny;
  std::vector<rte_cplx> t2(np), r2(np);
  rc = run_images(c, c->d_aux2, s, false, t2.data(), r2.data());
  if (rc) return rc;
  for (size_t q = 0; q < np; q++) {
    if (trans) trans[q].im += t2[q].re;
    if (ref) ref[q].im += r2[q].re;
  }
  return RTE_OK;
}

// First term and initial running sum of the series for beams (xi) and point sources (q):
// W0 = xi + D A q, S0 = xi + q + D A q (the point's uncollided field enters through the final A).
// xi (in d_xi) becomes S0; W0 goes to d_w0.  nb right-hand sides interleaved ([N][nb][C]).
static int series_start(rte_ctx* c, double* d_xi, double* d_q, double* d_w0, int nb, float* d_f32, int cpad) {
  const size_t n = (size_t)c->N * nb * c->C;
  if (!c->has_point) {
    CUDA_TRY(c, cudaMemcpyAsync(d_w0, d_xi, n * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    return RTE_OK;
  }
  if (c->precision == RTE_PREC_MIXED)
    CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(d_q, d_f32, c->d_islot, c->N, nb * c->C, cpad, c->C,
                                                        c->cstride, c->st)));
  int rc = apply_term(c, d_q, d_f32, d_w0, nullptr, nullptr, 1, 1, nb);
  if (rc) return rc;
  CUDA_TRY(c, (c->launches++, rte_launch_axpy(d_w0, d_xi, 1.0, n, c->st)));  // W0 = xi + DAq
  CUDA_TRY(c, cudaMemcpyAsync(d_xi, d_w0, n * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_axpy(d_xi, d_q, 1.0, n, c->st)));   // S0 = W0 + q
  return RTE_OK;
}

// Modulated forward solve: source with complex attenuation, complex series, complex images.
static int forward_cplx(rte_ctx* c, const rte_source* s, const rte_stop* stop, rte_cplx* W_out, rte_cplx* trans,
                        rte_cplx* ref, int* terms, double* rel) {
  int rc = ensure_batch(c, 2);
  if (rc) return rc;
  const size_t NC = (size_t)c->N * c->C;
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  CUDA_TRY(c, cudaMemsetAsync(c->d_bsum, 0, 2 * NC * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_bq, 0, 2 * NC * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_bball, 0, 2 * npix * sizeof(double), c->st));
  c->has_point = false;
  rc = launch_source(c, s, c->d_bsum, 2 * c->C, c->d_bball, false, c->d_bq, c->d_bball + npix);
  // W0 -> d_bW, S0 -> d_bsum
  if (!rc) rc = series_start(c, c->d_bsum, c->d_bq, c->d_bW, 2, c->d_bWf, (2 * c->cstride + 3) / 4 * 4);
  if (!rc) rc = neumann_cplx(c, 1, stop, terms, rel);
  if (!rc && (trans || ref))
    rc = run_images(c, c->d_bres, s, true, trans, ref, 2 * c->C, c->d_bball, c->d_bres + c->C, c->d_bball + npix);
  if (!rc && W_out) rc = download_pair(c, c->d_bres, W_out);
  return rc;
}

extern "C" int rte_forward(rte_ctx* c, const rte_source* s, const rte_stop* stop, rte_cplx* W_out, rte_cplx* trans,
                           rte_cplx* ref, rte_report* rep) {
  if (!c || !s || !stop) return fail(c, RTE_ERR_ARG, "null argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  if (s->modulation != c->modulation) {  // a solve runs at its source's modulation
    int rc = rte_set_modulation(c, s->modulation);
    if (rc) return rc;
  }
  if (c->kappa != 0.0) {
    cudaEvent_t t0, t1;
    CUDA_TRY(c, cudaEventCreate(&t0));
    CUDA_TRY(c, cudaEventCreate(&t1));
    CUDA_TRY(c, cudaEventRecord(t0, c->st));
    int terms = 0;
    double rel = 0.0;
    int rc = forward_cplx(c, s, stop, W_out, trans, ref, &terms, &rel);
    float ms = 0;
    if (!rc) {
      CUDA_TRY(c, cudaEventRecord(t1, c->st));
      CUDA_TRY(c, cudaEventSynchronize(t1));
      cudaEventElapsedTime(&ms, t0, t1);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc) return rc;
    if (rep) {
      rep->terms = terms;
      rep->last_rel = rel;
      rep->ms_device = ms;
      rep->ms_setup = c->last_setup_ms;
    }
    return RTE_OK;
  }
  cudaEvent_t t0, t1;
  CUDA_TRY(c, cudaEventCreate(&t0));
  CUDA_TRY(c, cudaEventCreate(&t1));
  CUDA_TRY(c, cudaEventRecord(t0, c->st));
  int terms = 0;
  double rel = 0;
  c->has_point = false;
  int rc = RTE_OK;
  if (s->kind == RTE_SRC_POINT) CUDA_TRY(c, cudaMemsetAsync(c->d_q, 0, (size_t)c->N * c->C * sizeof(double), c->st));
  rc = launch_source(c, s, c->d_aux1, 0, nullptr, true, c->d_q);
  if (!rc) rc = series_start(c, c->d_aux1, c->d_q, c->d_aux3, 1, c->d_Wf, c->cpad);
  if (!rc) rc = neumann_real(c, c->d_aux3, c->d_aux1, c->d_aux2, 1, stop, -1, &terms, &rel);
  if (!rc && (trans || ref)) rc = run_images(c, c->d_aux2, s, true, trans, ref);
  if (!rc) CUDA_TRY(c, cudaEventRecord(t1, c->st));
  if (!rc && W_out) rc = download_cplx(c, c->d_aux2, nullptr, W_out);
  float ms = 0;
  if (!rc) {
    CUDA_TRY(c, cudaEventSynchronize(t1));
    cudaEventElapsedTime(&ms, t0, t1);
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc) return rc;
  if (rep) {
    rep->terms = terms;
    rep->last_rel = rel;
    rep->ms_device = ms;
    rep->ms_setup = c->last_setup_ms;
  }
  return RTE_OK;
}

extern "C" int rte_measure_fma_peak(int device, int fp64, double* tflops) {
  if (!tflops || fp64 < 0 || fp64 > 4) return RTE_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return RTE_ERR_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  float* sink = nullptr;
  if (cudaMalloc(&sink, 65536 * sizeof(float)) != cudaSuccess) return RTE_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, iters = fp64 == 1 ? 20000 : 40000;
  double best = 0;
  // mode 0: the faster of the scalar and packed (f32x2) FP32 streams; 1: FP64; 2: scalar FP32 only;
  // 3: packed FP32 only; 4: packed FP32 with three distinct operands per instruction
  int variants[2] = {0, 2}, nv = 2;
  if (fp64 == 1) variants[0] = 1, nv = 1;
  if (fp64 == 2) nv = 1;
  if (fp64 == 3) variants[0] = 2, nv = 1;
  if (fp64 == 4) variants[0] = 3, nv = 1;
  for (int v = 0; v < nv; v++)
    for (int rep = 0; rep < 4; rep++) {
      cudaEventRecord(e0, 0);
      rte_launch_fma_peak(variants[v], iters, sink, 0, blocks);
      cudaEventRecord(e1, 0);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      const double per_iter = variants[v] == 3 ? 24.0 : (variants[v] == 2 ? 16.0 : 8.0);  // FMAs per thread
      const double flops = 2.0 * per_iter * (double)iters * blocks * 256.0;
      if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  *tflops = best;
  return e == cudaSuccess ? RTE_OK : RTE_ERR_DEVICE;
}

extern "C" void* rte_get_stream(rte_ctx* c) { return c ? (void*)c->st : nullptr; }

extern "C" int rte_set_profiling(rte_ctx* c, int on) {
  if (!c) return RTE_ERR_ARG;
  c->profiling = on != 0;
  return RTE_OK;
}

extern "C" int rte_get_stats(rte_ctx* c, rte_stats* out) {
  if (!c || !out) return fail(c, RTE_ERR_ARG, "null argument");
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  for (int k = 0; k < 3; k++) {
    for (auto& p : c->ev[k]) {
      float ms = 0;
      cudaEventElapsedTime(&ms, p.first, p.second);
      c->ms_acc[k] += ms;
      c->n_acc[k]++;
      c->ev_pool.push_back(p.first);
      c->ev_pool.push_back(p.second);
    }
    c->ev[k].clear();
  }
  out->launches = c->launches;
  out->ms_pair = c->ms_acc[0];
  out->n_pair = c->n_acc[0];
  out->ms_store = c->ms_acc[1];
  out->n_store = c->n_acc[1];
  out->ms_epi = c->ms_acc[2];
  out->n_epi = c->n_acc[2];
  c->launches = 0;
  for (int k = 0; k < 3; k++) {
    c->ms_acc[k] = 0;
    c->n_acc[k] = 0;
  }
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Batched forward solves: nsrc sources on one medium propagated together (the pair kernels reuse
// each pair's direction, SH and kernel value for every source).

template <class T>
static int grow(rte_ctx* c, T** p, size_t& cap, size_t n) {
  if (n <= cap) return RTE_OK;
  if (*p) {
    cudaFree(*p);
    c->bytes -= cap * sizeof(T);
    *p = nullptr;
  }
  CUDA_TRY(c, dalloc(c, p, n));
  cap = n;
  return RTE_OK;
}

static int ensure_batch(rte_ctx* c, int nb) {
  const size_t NC = (size_t)c->N * c->C;
  int rc = grow(c, &c->d_part, c->part_cap, NC * nb * c->max_split);
  if (!rc) rc = grow(c, &c->d_selfp, c->selfp_cap, NC * nb);
  if (rc || nb <= c->bcap) return rc;
  double** bufs[] = {&c->d_bW, &c->d_bWn, &c->d_bsum, &c->d_bres};
  for (double** b : bufs) {
    if (*b) cudaFree(*b);
    *b = nullptr;
    CUDA_TRY(c, dalloc(c, b, NC * nb));
  }
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  if (c->d_bball) cudaFree(c->d_bball);
  c->d_bball = nullptr;
  CUDA_TRY(c, dalloc(c, &c->d_bball, (size_t)nb * npix));
  if (c->d_bq) cudaFree(c->d_bq);
  c->d_bq = nullptr;
  CUDA_TRY(c, dalloc(c, &c->d_bq, NC * nb));
  if (c->d_bWf) cudaFree(c->d_bWf);
  c->d_bWf = nullptr;
  const int cp = (nb * c->cstride + 3) / 4 * 4;
  CUDA_TRY(c, dalloc(c, &c->d_bWf, (size_t)c->N * cp));
  CUDA_TRY(c, cudaMemset(c->d_bWf, 0, sizeof(float) * (size_t)c->N * cp));
  c->bcap = nb;
  return RTE_OK;
}

// Neumann series of nb right-hand sides together (mixed precision): W_0 in d_bW, the initial running
// sum in d_bsum ([N][nb][C]); result A sum in d_bres.  Stop rule FIXED or REL_L2 (norms over all
// right-hand sides).
static int series_batch(rte_ctx* c, int nb, const rte_stop* stop, int* terms_out, double* rel_out) {
  const int vs = nb * c->C;
  const int cp = (nb * c->cstride + 3) / 4 * 4;
  CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_bW, c->d_bWf, c->d_islot, c->N, vs, cp, c->C, c->cstride, c->st)));
  const int flag_l = c->cfg.g != 0.0 ? 1 : 0;
  int terms = 0;
  double rel = 0.0;
  while (terms < stop->max_terms) {
    int rc = apply_term(c, c->d_bW, c->d_bWf, c->d_bWn, c->d_bWf, c->d_bsum, flag_l, 1, nb);
    if (rc) return rc;
    std::swap(c->d_bW, c->d_bWn);
    terms++;
    if (stop->rule == RTE_STOP_REL_L2) {
      double hred[4];
      CUDA_TRY(c, cudaMemcpyAsync(hred, c->d_red, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
      CUDA_TRY(c, cudaStreamSynchronize(c->st));
      rel = hred[1] > 0 ? sqrt(hred[0] / hred[1]) : 0.0;
      if (rel < stop->tol) break;
    }
  }
  CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_bsum, c->d_bWf, c->d_islot, c->N, vs, cp, c->C, c->cstride, c->st)));
  int rc = apply_term(c, c->d_bsum, c->d_bWf, c->d_bres, nullptr, nullptr, 1, 0, nb);
  if (!rc) rc = check_kernel_err(c);
  if (terms_out) *terms_out = terms;
  if (rel_out) *rel_out = rel;
  return rc;
}

extern "C" int rte_forward_batch(rte_ctx* c, int nsrc, const rte_source* srcs, const rte_stop* stop,
                                 rte_cplx* W_out, rte_cplx* trans, rte_cplx* ref, rte_report* rep) {
  if (!c || !srcs || !stop || nsrc < 1) return fail(c, RTE_ERR_ARG, "bad argument");
  if (nsrc > kMaxBatch) return fail(c, RTE_ERR_UNSUPPORTED, "at most %d sources per batch", kMaxBatch);
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (stop->rule == RTE_STOP_REFERENCE)
    return fail(c, RTE_ERR_UNSUPPORTED, "batched solves take a fixed or relative-L2 stop rule");
  const size_t NC = (size_t)c->N * c->C, np = (size_t)c->nx * c->ny;
  // four right-hand sides of 49-64 coefficients exceed one thread's registers: at L >= 6 the recomputed
  // path integrals take k_pair_mixed_grp (two thread groups of two sharing the walks), the other forms
  // run two batches of two
  const bool grp = c->kernel_mode == RTE_KERNEL_RECOMPUTE && c->model != RTE_MODEL_FIM && c->kappa == 0.0;
  if (c->L >= 6 && nsrc > 2 && c->precision == RTE_PREC_MIXED && !grp) {
    rte_report r1, r2;
    int rc = rte_forward_batch(c, 2, srcs, stop, W_out, trans, ref, &r1);
    if (!rc)
      rc = rte_forward_batch(c, nsrc - 2, srcs + 2, stop, W_out ? W_out + 2 * NC : nullptr, trans ? trans + 2 * np : nullptr,
                             ref ? ref + 2 * np : nullptr, &r2);
    if (rc) return rc;
    if (rep) {
      *rep = r2;
      rep->ms_device = r1.ms_device + r2.ms_device;
    }
    return RTE_OK;
  }
  bool modulated = c->kappa != 0.0;
  for (int b = 0; b < nsrc; b++) modulated = modulated || srcs[b].modulation != 0.0;
  if (c->precision != RTE_PREC_MIXED || nsrc == 1 || modulated) {  // one source at a time
    double ms = 0;
    rte_report r1;
    for (int b = 0; b < nsrc; b++) {
      int rc = rte_forward(c, &srcs[b], stop, W_out ? W_out + b * NC : nullptr, trans ? trans + b * np : nullptr,
                           ref ? ref + b * np : nullptr, &r1);
      if (rc) return rc;
      ms += r1.ms_device;
    }
    if (rep) {
      *rep = r1;
      rep->ms_device = ms;
    }
    return RTE_OK;
  }
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  const int nb = nsrc <= 2 ? 2 : 4;  // kernel instantiations; extra right-hand sides stay zero
  int rc = ensure_batch(c, nb);
  if (rc) return rc;
  const int vs = nb * c->C;
  const int cp = (nb * c->cstride + 3) / 4 * 4;
  cudaEvent_t t0, t1;
  CUDA_TRY(c, cudaEventCreate(&t0));
  CUDA_TRY(c, cudaEventCreate(&t1));
  CUDA_TRY(c, cudaEventRecord(t0, c->st));
  const size_t npix = 2 * (np + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  CUDA_TRY(c, cudaMemsetAsync(c->d_bsum, 0, NC * nb * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_bq, 0, NC * nb * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_bball, 0, npix * nb * sizeof(double), c->st));
  c->has_point = false;
  for (int b = 0; b < nsrc && !rc; b++)
    rc = launch_source(c, &srcs[b], c->d_bsum + b * c->C, vs, c->d_bball + b * npix, false, c->d_bq + b * c->C);
  if (rc) return rc;
  // W0 -> d_bW, S0 -> d_bsum
  rc = series_start(c, c->d_bsum, c->d_bq, c->d_bW, nb, c->d_bWf, cp);
  if (rc) return rc;
  int terms = 0;
  double rel = 0.0;
  rc = series_batch(c, nb, stop, &terms, &rel);
  for (int b = 0; b < nsrc && !rc && (trans || ref); b++)
    rc = run_images(c, c->d_bres + b * c->C, &srcs[b], true, trans ? trans + b * np : nullptr,
                    ref ? ref + b * np : nullptr, vs, c->d_bball + b * npix);
  if (!rc) CUDA_TRY(c, cudaEventRecord(t1, c->st));
  for (int b = 0; b < nsrc && !rc && W_out; b++) {
    CUDA_TRY(c, (c->launches++, rte_launch_to_cplx(c->d_bres + b * c->C, nullptr, c->d_cplx, c->N, c->L, c->st, vs)));
    CUDA_TRY(c, cudaMemcpyAsync(W_out + b * NC, c->d_cplx, NC * sizeof(rte_cplx), cudaMemcpyDeviceToHost, c->st));
  }
  float ms = 0;
  if (!rc) {
    CUDA_TRY(c, cudaStreamSynchronize(c->st));
    cudaEventElapsedTime(&ms, t0, t1);
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (rc) return rc;
  if (rep) {
    rep->terms = terms;
    rep->last_rel = rel;
    rep->ms_device = ms;
    rep->ms_setup = c->last_setup_ms;
  }
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Detectors: exitant flux through the six faces, binned; the adjoint gradient of a binned-flux misfit.
// Face order: z- (z = 0), z+ (z = nZ-1), y-, y+, x-, x+.

// h_f[c] = cm * (pixel area) * int_{w.n > 0} R_c(w) (w.n) dw, by Gauss-Legendre in w.n and a
// uniform rule around n (exact for the polynomial integrand up to the order used).
static void face_weights(rte_ctx* c) {
  const int C = c->C;
  c->h_h.assign(6 * C, 0.0);
  std::vector<double> mu, wmu;
  gauss01(24, mu, wmu);
  const int M = 64;
  const double nrm[6][3] = {{0, 0, -1}, {0, 0, 1}, {0, -1, 0}, {0, 1, 0}, {-1, 0, 0}, {1, 0, 0}};
  const double area[6] = {c->dx * c->dy, c->dx * c->dy, c->dx * c->dz, c->dx * c->dz, c->dy * c->dz, c->dy * c->dz};
  std::vector<double> R(C);
  for (int f = 0; f < 6; f++) {
    const double* n = nrm[f];
    double e1[3], e2[3];
    if (fabs(n[2]) > 0.5) {
      e1[0] = 1; e1[1] = 0; e1[2] = 0;
    } else {
      e1[0] = 0; e1[1] = 0; e1[2] = 1;
    }
    e2[0] = n[1] * e1[2] - n[2] * e1[1];
    e2[1] = n[2] * e1[0] - n[0] * e1[2];
    e2[2] = n[0] * e1[1] - n[1] * e1[0];
    for (size_t a = 0; a < mu.size(); a++) {
      const double m = mu[a], s = sqrt(1.0 - m * m);
      for (int b = 0; b < M; b++) {
        const double ps = 2.0 * M_PI * (b + 0.5) / M;
        const double cp = cos(ps), sp = sin(ps);
        double w[3];
        for (int d = 0; d < 3; d++) w[d] = m * n[d] + s * (cp * e1[d] + sp * e2[d]);
        sh_real_host(c->sh, c->L, w[0], w[1], w[2], R.data());
        const double wt = wmu[a] * (2.0 * M_PI / M) * m;
        for (int q = 0; q < C; q++) c->h_h[f * C + q] += wt * R[q];
      }
    }
    for (int q = 0; q < C; q++) c->h_h[f * C + q] *= c->cm * area[f];
  }
}

static int ensure_detector_buffers(rte_ctx* c) {
  if (c->d_h) return RTE_OK;
  const size_t NC = (size_t)c->N * c->C;
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  face_weights(c);
  CUDA_TRY(c, dalloc(c, &c->d_h, c->h_h.size()));
  CUDA_TRY(c, cudaMemcpy(c->d_h, c->h_h.data(), sizeof(double) * c->h_h.size(), cudaMemcpyHostToDevice));
  double** bufs[] = {&c->d_S, &c->d_out, &c->d_e, &c->d_lam, &c->d_y};
  for (double** b : bufs) CUDA_TRY(c, dalloc(c, b, NC));
  CUDA_TRY(c, dalloc(c, &c->d_gt, c->N));
  CUDA_TRY(c, dalloc(c, &c->d_gs, c->N));
  CUDA_TRY(c, dalloc(c, &c->d_J, npix));
  CUDA_TRY(c, dalloc(c, &c->d_rho, npix));
  return RTE_OK;
}

// face geometry: rows x cols of pixels and offset of each face in the concatenated pixel array
static void face_dims(const rte_ctx* c, int f, int& P, int& Q, size_t& off) {
  const size_t a0 = (size_t)c->nx * c->ny, a1 = (size_t)c->nz * c->nx, a2 = (size_t)c->nz * c->ny;
  const size_t offs[6] = {0, a0, 2 * a0, 2 * a0 + a1, 2 * a0 + 2 * a1, 2 * a0 + 2 * a1 + a2};
  off = offs[f];
  if (f < 2) {
    P = c->ny;
    Q = c->nx;
  } else if (f < 4) {
    P = c->nz;
    Q = c->nx;
  } else {
    P = c->nz;
    Q = c->ny;
  }
}

// fraction of pixel p (of P along an edge) inside bin a (of nb)
static inline double overlap(int p, int P, int a, int nb) {
  const double lo = std::max((double)p / P, (double)a / nb), hi = std::min((double)(p + 1) / P, (double)(a + 1) / nb);
  return hi > lo ? (hi - lo) * P : 0.0;
}

// bins[f][a][b] = sum over the face's pixels of overlap x overlap x J
static void bin_faces(const rte_ctx* c, const rte_detector* d, const std::vector<double>& J, double* bins) {
  const int nb = d->nbins;
  for (int f = 0; f < 6; f++) {
    double* B = bins + (size_t)f * nb * nb;
    for (int q = 0; q < nb * nb; q++) B[q] = 0.0;
    if (!((d->faces >> f) & 1)) continue;
    int P, Q;
    size_t off;
    face_dims(c, f, P, Q, off);
    for (int p = 0; p < P; p++)
      for (int a = 0; a < nb; a++) {
        const double wa = overlap(p, P, a, nb);
        if (wa == 0.0) continue;
        for (int q = 0; q < Q; q++)
          for (int b = 0; b < nb; b++) {
            const double wb = overlap(q, Q, b, nb);
            if (wb != 0.0) B[a * nb + b] += wa * wb * J[off + (size_t)p * Q + q];
          }
      }
  }
}

// rho(pixel) = sum over bins of dL/dbin x (pixel's weight in the bin)
static void unbin_faces(const rte_ctx* c, const rte_detector* d, const double* dbins, std::vector<double>& rho) {
  const int nb = d->nbins;
  std::fill(rho.begin(), rho.end(), 0.0);
  for (int f = 0; f < 6; f++) {
    if (!((d->faces >> f) & 1)) continue;
    const double* B = dbins + (size_t)f * nb * nb;
    int P, Q;
    size_t off;
    face_dims(c, f, P, Q, off);
    for (int p = 0; p < P; p++)
      for (int a = 0; a < nb; a++) {
        const double wa = overlap(p, P, a, nb);
        if (wa == 0.0) continue;
        for (int q = 0; q < Q; q++)
          for (int b = 0; b < nb; b++) {
            const double wb = overlap(q, Q, b, nb);
            if (wb != 0.0) rho[off + (size_t)p * Q + q] += wa * wb * B[a * nb + b];
          }
      }
  }
}

// forward solve of one source leaving S (running sum) in d_S and out = A S in d_out; fluxes of
// all face pixels (ballistic included) in J.
static int forward_with_flux(rte_ctx* c, const rte_source* s, const rte_stop* stop, std::vector<double>& J, int* terms) {
  const size_t NC = (size_t)c->N * c->C;
  c->has_point = false;
  if (s->kind == RTE_SRC_POINT) CUDA_TRY(c, cudaMemsetAsync(c->d_q, 0, NC * sizeof(double), c->st));
  int rc = launch_source(c, s, c->d_aux1, 0, nullptr, true, c->d_q);
  if (!rc) rc = series_start(c, c->d_aux1, c->d_q, c->d_aux3, 1, c->d_Wf, c->cpad);
  if (rc) return rc;
  rc = neumann_real(c, c->d_aux3, c->d_aux1, c->d_out, 1, stop, -1, terms, nullptr);
  if (rc) return rc;
  CUDA_TRY(c, cudaMemcpyAsync(c->d_S, c->d_sum, NC * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  FaceArgs fa;
  memset(&fa, 0, sizeof fa);
  fa.nx = c->nx;
  fa.ny = c->ny;
  fa.nz = c->nz;
  fa.Cfull = c->C;
  fa.vstride = c->C;
  fa.out = c->d_out;
  fa.h = c->d_h;
  fa.fball = c->d_fball;
  fa.J = c->d_J;
  CUDA_TRY(c, (c->launches++, rte_launch_face_flux(fa, c->st)));
  CUDA_TRY(c, cudaMemcpyAsync(J.data(), c->d_J, J.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  return RTE_OK;
}

static int check_detector(rte_ctx* c, int nsrc, const rte_source* srcs, const rte_stop* stop, const rte_detector* d) {
  if (c && c->kappa != 0.0) return unsupported_modulated(c, "binned detectors");
  if (!srcs || !stop || !d || nsrc < 1) return fail(c, RTE_ERR_ARG, "null argument");
  if (d->nbins < 1 || d->nbins > 1024 || d->faces <= 0 || d->faces > 63) return fail(c, RTE_ERR_ARG, "bad detector");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (stop->rule == RTE_STOP_REFERENCE) return fail(c, RTE_ERR_UNSUPPORTED, "detectors take a fixed or relative-L2 stop rule");
  for (int q = 0; q < nsrc; q++) {
    std::vector<int> cols;
    double scale;
    if (source_columns(c, &srcs[q], cols, scale)) return fail(c, RTE_ERR_ARG, "bad source %d", q);
    if (cols.size() > 1) return fail(c, RTE_ERR_UNSUPPORTED, "detectors support single-column sources");
  }
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  return ensure_detector_buffers(c);
}

extern "C" int rte_detector_flux(rte_ctx* c, int nsrc, const rte_source* srcs, const rte_stop* stop,
                                 const rte_detector* d, double* flux) {
  if (!c) return RTE_ERR_ARG;
  int rc = check_detector(c, nsrc, srcs, stop, d);
  if (rc) return rc;
  const size_t npix = 2 * ((size_t)c->nx * c->ny + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  std::vector<double> J(npix);
  for (int q = 0; q < nsrc; q++) {
    int terms = 0;
    rc = forward_with_flux(c, &srcs[q], stop, J, &terms);
    if (rc) return rc;
    bin_faces(c, d, J, flux + (size_t)q * 6 * d->nbins * d->nbins);
  }
  return RTE_OK;
}

// Gradient of L = sum_{sources, bins} (F - target)^2 with respect to per-voxel mu_a and mu_s by the
// adjoint method.  With S = sum_k (DA)^k xi, out = A S and e = dL/dout:
//   lambda = (I - (DA)^T)^-1 A^T e, computed as P A (P e + sum_k (DA)^k D A P e), P = (-1)^l;
//   y = e + D lambda;
//   dL/dmu_t(v) = -sum_{pairs} len(v) k (y.R)(R.S) + (dV/cm) y_v . dDself/dmu S_v;
//   dL/dmu_s(v) += lambda_v . scat_l (A S)_v;   plus the source column and ballistic terms.
// Arguments of the back-projection passes; the pair-weight buffer (N x ld, FP32 for the mixed
// precision path, FP64 otherwise) is allocated on first use and kept with the context.
static BpArgs bp_args(rte_ctx* c, bool accumulate) {
  BpArgs bp;
  memset(&bp, 0, sizeof bp);
  bp.N = c->N;
  bp.nx = c->nx;
  bp.ny = c->ny;
  bp.nz = c->nz;
  bp.Cfull = c->C;
  bp.dx = c->dx;
  bp.dy = c->dy;
  bp.dz = c->dz;
  bp.prop_thresh = c->prop_thresh;
  bp.kscale = c->dV / c->cm;
  bp.perm = c->d_perm;
  bp.islot = c->d_islot;
  bp.mut = c->d_mut;
  bp.mutf = c->d_mutf;
  bp.y = c->d_y;
  bp.S = c->d_S;
  bp.Kmat = c->K_valid && c->d_K ? c->d_K : nullptr;
  bp.Kmat64 = c->K_valid && c->d_K64 ? c->d_K64 : nullptr;
  bp.Kld = ((size_t)c->N + 31) / 32 * 32;
  bp.g = c->d_gt;
  bp.Q = c->d_Qbp;
  bp.accumulate = accumulate ? 1 : 0;
  return bp;
}

static int ensure_bp_buffer(rte_ctx* c) {
  const size_t ld = ((size_t)c->N + 31) / 32 * 32;
  const size_t need = (size_t)c->N * ld * (c->precision == RTE_PREC_MIXED ? sizeof(float) : sizeof(double));
  if (c->d_Qbp && c->qbp_bytes >= need) return RTE_OK;
  if (c->d_Qbp) {
    cudaFree(c->d_Qbp);
    c->bytes -= c->qbp_bytes;
    c->d_Qbp = nullptr;
  }
  size_t fr = 0, tot = 0;
  CUDA_TRY(c, cudaMemGetInfo(&fr, &tot));
  if (need + (1ull << 30) > fr)
    return fail(c, RTE_ERR_NOMEM, "gradient pair weights need %.1f GB, %.1f GB free", need / 1e9, fr / 1e9);
  CUDA_TRY(c, cudaMalloc(&c->d_Qbp, need));
  c->qbp_bytes = need;
  c->bytes += need;
  return RTE_OK;
}

// Adjoint field of one source: lambda = (I - A^T D)^-1 A^T e for the seed e = dL/d(out) in d_e, with
// A^T = P A P (P = (-1)^l in the real basis: A's kernel is symmetric in (r, r') and R(-w) = P R(w)), so
// lambda = P A (I - D A)^-1 P e: the forward machinery on P e, the same number of terms as the forward
// solve it differentiates (`terms`), result in d_lam.
// The table model (RTE_MODEL_FIM) snaps pair directions to its 100 x 100 table, and snapping does not
// commute with negation: there A^T is applied directly (pair kernels in transposed mode; the self term
// and D are symmetric), lambda = (I - A^T D)^-1 A^T e = A^T (I - D A^T)^-1 e.
static int adjoint_series(rte_ctx* c, const rte_stop* stop, int terms) {
  const size_t NC = (size_t)c->N * c->C;
  const bool table = c->model == RTE_MODEL_FIM;
  CUDA_TRY(c, cudaMemcpyAsync(c->d_aux3, c->d_e, NC * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  if (!table) CUDA_TRY(c, (c->launches++, rte_launch_parity(c->d_aux3, c->N, c->L, c->C, c->st)));
  if (c->precision == RTE_PREC_MIXED)
    CUDA_TRY(c, (c->launches++, rte_launch_to_f32_slots(c->d_aux3, c->d_Wf, c->d_islot, c->N, c->C, c->cpad, c->C,
                                                        c->cstride, c->st)));
  c->transpose = table;
  int rc = apply_term(c, c->d_aux3, c->d_Wf, c->d_aux4, nullptr, nullptr, 1, 1);
  if (!rc) {
    CUDA_TRY(c, (c->launches++, rte_launch_axpy(c->d_aux3, c->d_aux4, 1.0, NC, c->st)));
    rc = neumann_real(c, c->d_aux4, c->d_aux3, c->d_lam, 1, stop, std::max(terms - 1, 0), nullptr, nullptr);
  }
  c->transpose = false;
  if (rc) return rc;
  if (!table) CUDA_TRY(c, (c->launches++, rte_launch_parity(c->d_lam, c->N, c->L, c->C, c->st)));
  return RTE_OK;
}

// Exact derivative of the discrete model for one source, after its forward solve (d_S = running sum,
// d_out = A S) and with the seed e = dL/d(out) in d_e: the adjoint series, the pair weights of the
// back-projection (pass 1, summed into the pair-weight buffer; `first` overwrites it), the self-term
// and scatter parts (into d_gt, d_gs), and on the host the source column and the ballistic beam of a
// z = 0 collimated source (rho_ball = dL/d(ballistic flux at the z = nZ-1 exit pixel of the column),
// into ga, gsum).  The walk of pass 2 runs once after all sources (rte_launch_bp_walk).
static int adjoint_source_terms(rte_ctx* c, const rte_source* s, const rte_stop* stop, int terms, double rho_ball,
                                bool first, const std::vector<double>& mut, const std::vector<double>& mus,
                                std::vector<double>& ga, std::vector<double>& gsum) {
  const bool mixed = c->precision == RTE_PREC_MIXED;
  double scat[RTE_MAX_L + 1];
  scatter_factors(c, 1, scat);
  int rc = adjoint_series(c, stop, terms);
  if (rc) return rc;
  CUDA_TRY(c, (c->launches++, rte_launch_y_field(c->d_y, c->d_e, c->d_lam, c->d_mus, scat, c->N, c->L, c->C, c->st)));
  // back-projection through exp(-tau), pass 1: this source's weight of every unordered pair, summed
  // over the sources in the pair-weight buffer
  BpArgs bp = bp_args(c, !first);
  {
    ProfScope ps(c, 0);
    CUDA_TRY(c, (c->launches++, rte_launch_bp_weights(bp, c->L, mixed ? 0 : 1, c->st)));
  }
  GradLocalArgs gl;
  memset(&gl, 0, sizeof gl);
  gl.N = c->N;
  gl.Cfull = c->C;
  gl.Cact = c->C;
  gl.y = c->d_y;
  gl.lam = c->d_lam;
  gl.S = c->d_S;
  gl.out = c->d_out;
  gl.mus = c->d_mus;
  gl.mut = c->d_mut;
  gl.idx = c->self_lut_ok ? c->d_self_idx : nullptr;
  gl.dlut = c->d_dlut;
  gl.mom = c->d_mom;
  gl.K = c->K;
  gl.scale = c->dV / c->cm;
  gl.air_no_self = c->model == RTE_MODEL_FIM ? 1 : 0;
  for (int l = 0; l <= RTE_MAX_L; l++) gl.scat[l] = scat[l];
  gl.gt = c->d_gt;
  gl.gs = c->d_gs;
  CUDA_TRY(c, (c->launches++, rte_launch_grad_local(gl, c->st)));
  // source column and ballistic transmission (host; nz voxels)
  std::vector<int> cols;
  double scale;
  if (source_columns(c, s, cols, scale)) return fail(c, RTE_ERR_ARG, "bad source");
  for (int col : cols) {
    const int nz = c->nz, plane = c->nx * c->ny;
    std::vector<double> lamc((size_t)nz * c->C);
    for (int i = 0; i < nz; i++)
      CUDA_TRY(c, cudaMemcpyAsync(&lamc[(size_t)i * c->C], c->d_lam + ((size_t)i * plane + col) * c->C,
                                  c->C * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CUDA_TRY(c, cudaStreamSynchronize(c->st));
    std::vector<double> X(nz), Lam(nz), Tt(nz), E(nz);
    double att = 1.0;
    for (int i = 0; i < nz; i++) {
      const int r = i * plane + col;
      E[i] = exp(-mut[r] * c->dz);
      Tt[i] = att;
      att *= E[i];
      double lam = 0.0, gl2 = 1.0;
      for (int l = 0; l <= c->L; l++) {
        lam += lamc[(size_t)i * c->C + l * l + l] * scale * gl2 * sqrt((2.0 * l + 1.0) / (4.0 * M_PI)) / c->dV;
        gl2 *= c->cfg.g;
      }
      Lam[i] = lam;
      X[i] = (mus[r] / mut[r]) * Tt[i] * (1 - E[i]);
    }
    double tail = 0.0;  // sum_{i' > i} Lam X
    const double ball = s->mag * att;
    for (int i = nz - 1; i >= 0; i--) {
      const int r = i * plane + col;
      const double mt = mut[r], ms = mus[r], ma = mt - ms;
      const double common = (ms / mt) * Tt[i] * c->dz * E[i];
      ga[r] += Lam[i] * (Tt[i] * (1 - E[i]) * (-ms / (mt * mt)) + common) - c->dz * tail - rho_ball * ball * c->dz;
      gsum[r] += Lam[i] * (Tt[i] * (1 - E[i]) * (ma / (mt * mt)) + common) - c->dz * tail - rho_ball * ball * c->dz;
      tail += Lam[i] * X[i];
    }
  }
  return RTE_OK;
}

// Pass 2 of the back-projection, then the per-voxel gradient g_mua = g_t + ga, g_mus = g_t + g_s + gsum.
static int adjoint_finish(rte_ctx* c, const std::vector<double>& ga, const std::vector<double>& gsum, double* g_mua,
                          double* g_mus) {
  {
    const BpArgs bp = bp_args(c, true);
    ProfScope ps(c, 0);
    CUDA_TRY(c, (c->launches++, rte_launch_bp_walk(bp, c->precision == RTE_PREC_MIXED ? 0 : 1, c->st)));
  }
  std::vector<double> gt(c->N), gs(c->N);
  CUDA_TRY(c, cudaMemcpyAsync(gt.data(), c->d_gt, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaMemcpyAsync(gs.data(), c->d_gs, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->st));
  CUDA_TRY(c, cudaStreamSynchronize(c->st));
  int rc = check_kernel_err(c);
  if (rc) return rc;
  for (int r = 0; r < c->N; r++) {
    g_mua[r] = gt[r] + ga[r];
    g_mus[r] = gt[r] + gs[r] + gsum[r];
  }
  return RTE_OK;
}

static int gradient_sources_ok(rte_ctx* c, int nsrc, const rte_source* srcs) {
  if (c->split)
    return fail(c, RTE_ERR_UNSUPPORTED, "the exact derivative needs one tissue table (rte_set_medium_tissue_split)");
  if (c->model == RTE_MODEL_FIM)
    return fail(c, RTE_ERR_UNSUPPORTED,
                "the exact derivative is not available for the table model (RTE_MODEL_FIM): its back-projection "
                "uses exact directions; use RTE_DERIV_REFERENCE or RTE_MODEL_EXACT");
  for (int q = 0; q < nsrc && srcs; q++)
    if (srcs[q].kind != RTE_SRC_COLUMN && srcs[q].kind != RTE_SRC_FIM &&
        !(srcs[q].kind == RTE_SRC_BEAM && srcs[q].face == 0))
      return fail(c, RTE_ERR_UNSUPPORTED, "the gradient takes collimated sources on the z = 0 face");
  return RTE_OK;
}

static int gradient_setup(rte_ctx* c, std::vector<double>& mut, std::vector<double>& mus) {
  mut.resize(c->N);
  mus.resize(c->N);
  CUDA_TRY(c, cudaMemsetAsync(c->d_gt, 0, sizeof(double) * c->N, c->st));
  CUDA_TRY(c, cudaMemsetAsync(c->d_gs, 0, sizeof(double) * c->N, c->st));
  CUDA_TRY(c, cudaMemcpy(mut.data(), c->d_mut, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
  CUDA_TRY(c, cudaMemcpy(mus.data(), c->d_mus, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
  return ensure_bp_buffer(c);
}

extern "C" int rte_gradient(rte_ctx* c, int nsrc, const rte_source* srcs, const rte_stop* stop,
                            const rte_detector* d, const double* target, double* loss, double* g_mua,
                            double* g_mus) {
  if (!c || !target || !g_mua || !g_mus) return fail(c, RTE_ERR_ARG, "null argument");
  if (c->kappa != 0.0) return unsupported_modulated(c, "the adjoint gradient");
  int rc = gradient_sources_ok(c, nsrc, srcs);
  if (rc) return rc;
  rc = check_detector(c, nsrc, srcs, stop, d);
  if (rc) return rc;
  const size_t np = (size_t)c->nx * c->ny;
  const size_t npix = 2 * (np + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  const int nb = d->nbins;
  std::vector<double> J(npix), rho(npix), bins(6 * nb * nb), dbins(6 * nb * nb);
  std::vector<double> ga(c->N, 0.0), gsum(c->N, 0.0), mut, mus;
  rc = gradient_setup(c, mut, mus);
  if (rc) return rc;
  double L2 = 0.0;
  for (int sidx = 0; sidx < nsrc; sidx++) {
    const rte_source* s = &srcs[sidx];
    int terms = 0;
    rc = forward_with_flux(c, s, stop, J, &terms);
    if (rc) return rc;
    bin_faces(c, d, J, bins.data());
    const double* T = target + (size_t)sidx * 6 * nb * nb;
    for (int f = 0; f < 6; f++)
      for (int q = 0; q < nb * nb; q++) {
        const size_t i = (size_t)f * nb * nb + q;
        const double r = ((d->faces >> f) & 1) ? bins[i] - T[i] : 0.0;
        L2 += r * r;
        dbins[i] = 2.0 * r;
      }
    unbin_faces(c, d, dbins.data(), rho);
    CUDA_TRY(c, cudaMemcpyAsync(c->d_rho, rho.data(), npix * sizeof(double), cudaMemcpyHostToDevice, c->st));
    CUDA_TRY(c, cudaMemsetAsync(c->d_e, 0, (size_t)c->N * c->C * sizeof(double), c->st));
    FaceArgs fa;
    memset(&fa, 0, sizeof fa);
    fa.nx = c->nx;
    fa.ny = c->ny;
    fa.nz = c->nz;
    fa.Cfull = c->C;
    fa.vstride = c->C;
    fa.h = c->d_h;
    fa.rho = c->d_rho;
    fa.e = c->d_e;
    CUDA_TRY(c, (c->launches++, rte_launch_adjoint_seed(fa, c->st)));
    std::vector<int> cols;
    double scale;
    source_columns(c, s, cols, scale);
    const double rho_b = cols.empty() ? 0.0 : rho[np + (size_t)cols[0]];  // z+ face pixel of the column
    rc = adjoint_source_terms(c, s, stop, terms, rho_b, sidx == 0, mut, mus, ga, gsum);
    if (rc) return rc;
  }
  rc = adjoint_finish(c, ga, gsum, g_mua, g_mus);
  if (rc) return rc;
  if (loss) *loss = L2;
  return RTE_OK;
}

// Gradient of the reference's image misfit sum_j (gbar_j - g_j)^2 (compute_grad_rte.cu:314-315,
// 376-377; GPU package/src/inverse_rte.cu:365, 425) from one forward and one adjoint series.
extern "C" int rte_image_gradient(rte_ctx* c, const rte_source* s, const rte_stop* stop, int image, int deriv,
                                  const double* g, double* loss, double* g_mua, double* g_mus) {
  if (!c || !s || !stop || !g || !g_mua || !g_mus) return fail(c, RTE_ERR_ARG, "null argument");
  if (image != 0 && image != 1) return fail(c, RTE_ERR_ARG, "image must be 0 (transmission) or 1 (reflection)");
  if (deriv != RTE_DERIV_EXACT && deriv != RTE_DERIV_REFERENCE) return fail(c, RTE_ERR_ARG, "bad derivative model");
  if (c->kappa != 0.0 || s->modulation != 0.0) return unsupported_modulated(c, "the image gradient");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (stop->rule == RTE_STOP_REFERENCE && deriv == RTE_DERIV_EXACT)
    return fail(c, RTE_ERR_UNSUPPORTED, "the exact derivative takes a fixed or relative-L2 stop rule");
  int rc = deriv == RTE_DERIV_EXACT ? gradient_sources_ok(c, 1, s) : RTE_OK;
  if (rc) return rc;
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  rc = ensure_detector_buffers(c);
  if (rc) return rc;
  const size_t np = (size_t)c->nx * c->ny, NC = (size_t)c->N * c->C;
  std::vector<double> ga(c->N, 0.0), gsum(c->N, 0.0), mut, mus;
  if (deriv == RTE_DERIV_EXACT) {
    rc = gradient_setup(c, mut, mus);
    if (rc) return rc;
  }
  // forward solve: S in d_S, out = A S in d_out, the image with its ballistic term
  const size_t npix = 2 * (np + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  std::vector<double> J(npix);
  int terms = 0;
  if (s->kind == RTE_SRC_CPU) {  // several columns: the flux path takes single-column sources
    c->has_point = false;
    rc = launch_source(c, s, c->d_aux1, 0, nullptr, true, c->d_q);
    if (!rc) rc = series_start(c, c->d_aux1, c->d_q, c->d_aux3, 1, c->d_Wf, c->cpad);
    if (!rc) rc = neumann_real(c, c->d_aux3, c->d_aux1, c->d_out, 1, stop, -1, &terms, nullptr);
    if (!rc) CUDA_TRY(c, cudaMemcpyAsync(c->d_S, c->d_sum, NC * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  } else {
    rc = forward_with_flux(c, s, stop, J, &terms);
  }
  if (rc) return rc;
  std::vector<rte_cplx> gbar(np);
  rc = run_images(c, c->d_out, s, true, image == 0 ? gbar.data() : nullptr, image == 1 ? gbar.data() : nullptr);
  if (rc) return rc;
  // seed e = M^T rho on the image's voxel layer, rho_j = 2 (gbar_j - g_j), M the per-l image weights
  ImgArgs wts;
  rc = image_weights(c, s, wts);
  if (rc) return rc;
  const double* w = image == 0 ? wts.wt : wts.wr;
  std::vector<double> rho(np), layer(np * c->C, 0.0);
  double L2 = 0.0;
  for (size_t j = 0; j < np; j++) {
    const double e = gbar[j].re - g[j];
    L2 += e * e;
    rho[j] = 2.0 * e;
    for (int l = 0; l <= c->L; l++) layer[j * c->C + l * l + l] = w[l] * rho[j];
  }
  const size_t layer_off = image == 0 ? (size_t)(c->nz - 1) * np : 0;
  CUDA_TRY(c, cudaMemsetAsync(c->d_e, 0, NC * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_e + layer_off * c->C, layer.data(), layer.size() * sizeof(double),
                              cudaMemcpyHostToDevice, c->st));
  if (deriv == RTE_DERIV_REFERENCE) {
    // the reference's tangent sources -C dmu_a out and (-C + g^l) dmu_s out (C = 1, rte.h:15) paired
    // with the adjoint field: d loss / d mu(r) = <lambda_r, source_r>
    rc = adjoint_series(c, stop, terms);
    if (rc) return rc;
    double fa[RTE_MAX_L + 1], fs[RTE_MAX_L + 1];
    for (int l = 0; l <= RTE_MAX_L; l++) {
      fa[l] = -1.0;
      fs[l] = -1.0 + pow(c->cfg.g, (double)l);
    }
    CUDA_TRY(c, (c->launches++, rte_launch_tangent_pair_dots(c->d_lam, c->d_out, fa, fs, c->N, c->L, c->d_gt, c->d_gs,
                                                              c->st)));
    CUDA_TRY(c, cudaMemcpyAsync(g_mua, c->d_gt, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->st));
    CUDA_TRY(c, cudaMemcpyAsync(g_mus, c->d_gs, sizeof(double) * c->N, cudaMemcpyDeviceToHost, c->st));
    CUDA_TRY(c, cudaStreamSynchronize(c->st));
    rc = check_kernel_err(c);
    if (rc) return rc;
  } else {
    std::vector<int> cols;
    double scale;
    source_columns(c, s, cols, scale);
    // the ballistic beam reaches the transmission image at its column's pixel (dist.cu:137-145)
    const double rho_b = (image == 0 && !cols.empty()) ? rho[(size_t)cols[0]] : 0.0;
    rc = adjoint_source_terms(c, s, stop, terms, rho_b, true, mut, mus, ga, gsum);
    if (!rc) rc = adjoint_finish(c, ga, gsum, g_mua, g_mus);
    if (rc) return rc;
  }
  if (loss) *loss = L2;
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Fixed-term Neumann series of nb right-hand sides as one CUDA graph per context: the pair-kernel
// precompute (for the medium set before the replay), nterms x (pair, self, epilogue) and the final
// attenuation, recorded once and replayed for every request of this shape.  W0 and S0 must be in
// graph_w0 / graph_s0 before the replay; the result lands in d_bres (nb > 1) or d_aux2 (nb = 1).
static std::vector<uintptr_t> graph_signature(const rte_ctx* c, int nb) {
  auto u = [](const void* p) { return (uintptr_t)p; };
  const double* W = nb == 1 ? c->d_W : c->d_bW;
  const double* Wn = nb == 1 ? c->d_Wn : c->d_bWn;
  return {u(std::min(W, Wn)), u(std::max(W, Wn)), u(nb == 1 ? c->d_sum : c->d_bsum),
          u(nb == 1 ? c->d_aux2 : c->d_bres), u(nb == 1 ? (const void*)c->d_Wf : (const void*)c->d_bWf),
          u(c->d_part), u(c->d_selfp), u(c->d_self_idx), u(c->d_self_lut), u(c->d_mom), (uintptr_t)c->K,
          (uintptr_t)c->self_lut_ok, u(c->d_K), u(c->d_K64), (uintptr_t)c->Kld, u(c->d_mut), u(c->d_mutf), u(c->d_mus),
          u(c->d_red), u(c->d_err), (uintptr_t)c->bcap, (uintptr_t)(fft_eligible(c) && !c->fft_graph_failed),
          rte_fft_signature(c->fft)};
}

static bool graph_stale(const rte_ctx* c, int nb, int nterms) {
  return !c->graph[nb] || c->graph_terms[nb] != nterms || c->graph_sig[nb] != graph_signature(c, nb);
}

static int run_series_graph(rte_ctx* c, int nb, int nterms, double** d_res) {
  const int gi = nb;
  const size_t NC = (size_t)c->N * c->C;
  const int vs = nb * c->C;
  const int cp = (nb * c->cstride + 3) / 4 * 4;
  double* W = nb == 1 ? c->d_W : c->d_bW;
  double* Wn = nb == 1 ? c->d_Wn : c->d_bWn;
  double* sum = nb == 1 ? c->d_sum : c->d_bsum;
  double* res = nb == 1 ? c->d_aux2 : c->d_bres;
  float* Wf = nb == 1 ? c->d_Wf : c->d_bWf;
  const int flag_l = c->cfg.g != 0.0 ? 1 : 0;
  if (graph_stale(c, nb, nterms)) {
    if (c->graph[gi]) {
      cudaGraphExecDestroy(c->graph[gi]);
      c->graph[gi] = nullptr;
    }
    // everything that may allocate or synchronise happens before the capture
    const bool use_fft = fft_eligible(c) && !c->fft_graph_failed;
    bool stored = false;
    int rc = RTE_OK;
    if (use_fft) {  // uniform medium: table spectra and transform plans now, the transforms in the graph
      rc = ensure_fft(c);
      if (!rc) CUDA_TRY(c, rte_fft_warm(c->fft, nb * c->C));
      if (!rc && flag_l == 0) CUDA_TRY(c, rte_fft_warm(c->fft, nb));
    } else {
      rc = ensure_pair_kernel(c, &stored);
      if (rc) return rc;
      int S, chunk;
      rc = plan_split(c, 0, stored ? 1 : 0, nb, &S, &chunk);
      if (!rc) rc = plan_split(c, c->L, stored ? 1 : 0, nb, &S, &chunk);
      if (!rc && flag_l == 0) rc = plan_split(c, 0, stored ? 1 : 0, nb, &S, &chunk);
    }
    if (rc) return rc;
    c->fft_in_graph[gi] = use_fft;
    c->fft_capture_ready = use_fft;
    c->graph_w0[gi] = W;
    c->graph_s0[gi] = sum;
    const bool prof = c->profiling;
    c->profiling = false;
    c->capturing = true;
    cudaGraph_t g = nullptr;
    CUDA_TRY(c, cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    if (stored) {  // the precompute for whatever medium is set when the graph is replayed
      c->capture_store = true;
      rc = ensure_pair_kernel(c, &stored);
      c->capture_store = false;
    }
    cudaError_t e = rte_launch_to_f32_slots(W, Wf, c->d_islot, c->N, vs, cp, c->C, c->cstride, c->st);
    if (e == cudaSuccess) {
      double *w = W, *wn = Wn;
      for (int t = 0; t < nterms && !rc; t++) {
        rc = apply_term(c, w, Wf, wn, Wf, sum, flag_l, 1, nb);
        std::swap(w, wn);
      }
      if (!rc) e = rte_launch_to_f32_slots(sum, Wf, c->d_islot, c->N, vs, cp, c->C, c->cstride, c->st);
      if (!rc && e == cudaSuccess) rc = apply_term(c, sum, Wf, res, nullptr, nullptr, 1, 0, nb);
    }
    cudaError_t e2 = cudaStreamEndCapture(c->st, &g);
    c->capturing = false;
    c->fft_capture_ready = false;
    c->profiling = prof;
    if ((rc || e != cudaSuccess || e2 != cudaSuccess) && use_fft) {
      // the transforms could not be recorded: record the pair kernels instead from now on
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      c->fft_graph_failed = true;
      return run_series_graph(c, nb, nterms, d_res);
    }
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess || e2 != cudaSuccess)
      return fail(c, RTE_ERR_DEVICE, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    cudaError_t e3 = cudaGraphInstantiate(&c->graph[gi], g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return fail(c, RTE_ERR_DEVICE, "graph instantiate: %s", cudaGetErrorString(e3));
    c->graph_terms[gi] = nterms;
    c->graph_sig[gi] = graph_signature(c, nb);
  } else if (c->fft_in_graph[gi]) {
    int rc = ensure_fft(c);  // the table spectra of the current medium, outside the graph
    if (rc) return rc;
  }
  (void)NC;
  c->launches += 4 * nterms + 4;
  CUDA_TRY(c, cudaGraphLaunch(c->graph[gi], c->st));
  if (!c->fft_in_graph[gi]) c->K_valid = true;  // the graph recomputed the stored kernel
  *d_res = res;
  return RTE_OK;
}

// One request through the graph path: sources (nsrc <= 4 on the current medium), the captured
// series, images.  trans/ref: nsrc * nx * ny complex (may be null).
static int forward_graph(rte_ctx* c, int nsrc, const rte_source* srcs, int nterms, rte_cplx* trans, rte_cplx* ref,
                         float* ms_out) {
  if (nsrc > 1 && c->precision != RTE_PREC_MIXED) {  // FP64 keeps one right-hand side per series
    float tot = 0;
    const size_t np = (size_t)c->nx * c->ny;
    for (int b = 0; b < nsrc; b++) {
      float ms = 0;
      int rc = forward_graph(c, 1, srcs + b, nterms, trans ? trans + b * np : nullptr, ref ? ref + b * np : nullptr, &ms);
      if (rc) return rc;
      tot += ms;
    }
    if (ms_out) *ms_out = tot;
    return RTE_OK;
  }
  const int nb = nsrc == 1 ? 1 : (nsrc <= 2 ? 2 : 4);
  int rc = nb > 1 ? ensure_batch(c, nb) : RTE_OK;
  if (rc) return rc;
  const size_t NC = (size_t)c->N * c->C, np = (size_t)c->nx * c->ny;
  const size_t npix = 2 * (np + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  const int vs = nb * c->C;
  const int cp = (nb * c->cstride + 3) / 4 * 4;
  if (!c->ev_graph[0]) {
    CUDA_TRY(c, cudaEventCreate(&c->ev_graph[0]));
    CUDA_TRY(c, cudaEventCreate(&c->ev_graph[1]));
  }
  cudaEvent_t t0 = c->ev_graph[0], t1 = c->ev_graph[1];
  CUDA_TRY(c, cudaEventRecord(t0, c->st));
  double* dres = nullptr;
  if (graph_stale(c, nb, nterms)) {
    // first request of this shape (or buffers moved since the recording): record the graph on zero
    // inputs, then run the real one
    double* w = nb == 1 ? c->d_W : c->d_bW;
    double* sm = nb == 1 ? c->d_sum : c->d_bsum;
    CUDA_TRY(c, cudaMemsetAsync(w, 0, NC * nb * sizeof(double), c->st));
    CUDA_TRY(c, cudaMemsetAsync(sm, 0, NC * nb * sizeof(double), c->st));
    rc = run_series_graph(c, nb, nterms, &dres);
    if (rc) return rc;
  }
  double* W0 = c->graph_w0[nb];
  double* S0 = c->graph_s0[nb];
  double* q = nb == 1 ? c->d_q : c->d_bq;
  double* fb = nb == 1 ? c->d_fball : c->d_bball;
  CUDA_TRY(c, cudaMemsetAsync(S0, 0, NC * nb * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(q, 0, NC * nb * sizeof(double), c->st));
  CUDA_TRY(c, cudaMemsetAsync(fb, 0, npix * nb * sizeof(double), c->st));
  c->has_point = false;
  for (int b = 0; b < nsrc && !rc; b++)
    rc = launch_source(c, &srcs[b], S0 + b * c->C, vs, fb + b * npix, false, q + b * c->C);
  if (!rc) rc = series_start(c, S0, q, W0, nb, nb == 1 ? c->d_Wf : c->d_bWf, cp);
  if (!rc) rc = run_series_graph(c, nb, nterms, &dres);
  for (int b = 0; b < nsrc && !rc && (trans || ref); b++)
    rc = run_images(c, dres + b * c->C, &srcs[b], true, trans ? trans + b * np : nullptr,
                    ref ? ref + b * np : nullptr, vs, fb + b * npix);
  if (!rc) CUDA_TRY(c, cudaEventRecord(t1, c->st));
  if (!rc) CUDA_TRY(c, cudaStreamSynchronize(c->st));
  if (!rc) rc = check_kernel_err(c);
  float ms = 0;
  if (!rc) cudaEventElapsedTime(&ms, t0, t1);
  if (ms_out) *ms_out = ms;
  return rc;
}

extern "C" int rte_forward_graph(rte_ctx* c, int nsrc, const rte_source* srcs, int nterms, rte_cplx* trans,
                                 rte_cplx* ref, rte_report* rep) {
  if (!c || !srcs || nsrc < 1 || nsrc > kMaxBatch || nterms < 0) return fail(c, RTE_ERR_ARG, "bad argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (c->kappa != 0.0) return unsupported_modulated(c, "graph replay");
  for (int b = 0; b < nsrc; b++)
    if (srcs[b].modulation != 0.0) return unsupported_modulated(c, "graph replay");
  if (c->L >= 6 && nsrc > 2 && c->precision == RTE_PREC_MIXED) {  // as rte_forward_batch: two graphs of two
    const size_t np = (size_t)c->nx * c->ny;
    rte_report r1, r2;
    int rc = rte_forward_graph(c, 2, srcs, nterms, trans, ref, &r1);
    if (!rc) rc = rte_forward_graph(c, nsrc - 2, srcs + 2, nterms, trans ? trans + 2 * np : nullptr,
                                    ref ? ref + 2 * np : nullptr, &r2);
    if (rc) return rc;
    if (rep) {
      *rep = r2;
      rep->ms_device = r1.ms_device + r2.ms_device;
    }
    return RTE_OK;
  }
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  float ms = 0;
  int rc = forward_graph(c, nsrc, srcs, nterms, trans, ref, &ms);
  if (rc) return rc;
  if (rep) {
    rep->terms = nterms;
    rep->last_rel = 0;
    rep->ms_device = ms;
    rep->ms_setup = 0;
  }
  return RTE_OK;
}

// ---------------------------------------------------------------------------------------
// Reference-compatible region derivatives (the tangent solves of the reference's inverse and
// Fisher mains).  The forward solution `out` stays on the device (d_out); each region tangent is
// the series of the masked, per-l scaled copy of it, projected to the exitance images without the
// ballistic term (FisherInfo_IO/src/compute_grad_rte.cu:273-385, rte_fim.cu:236-331).

static int forward_to_out(rte_ctx* c, const rte_source* s, const rte_stop* stop, rte_cplx* trans, rte_cplx* ref) {
  int rc = ensure_detector_buffers(c);
  if (rc) return rc;
  c->has_point = false;
  if (s->kind == RTE_SRC_POINT) CUDA_TRY(c, cudaMemsetAsync(c->d_q, 0, (size_t)c->N * c->C * sizeof(double), c->st));
  rc = launch_source(c, s, c->d_aux1, 0, nullptr, true, c->d_q);
  if (!rc) rc = series_start(c, c->d_aux1, c->d_q, c->d_aux3, 1, c->d_Wf, c->cpad);
  if (!rc) rc = neumann_real(c, c->d_aux3, c->d_aux1, c->d_out, 1, stop, -1, nullptr, nullptr);
  if (!rc) rc = run_images(c, c->d_out, s, true, trans, ref);
  return rc;
}

static int tangent_images(rte_ctx* c, const rte_source* s, const uint8_t* mask, const double* fac,
                          const rte_stop* stop, rte_cplx* dtrans, rte_cplx* dref) {
  if (!c->d_mask) CUDA_TRY(c, dalloc(c, &c->d_mask, (size_t)c->N));
  CUDA_TRY(c, cudaMemcpyAsync(c->d_mask, mask, (size_t)c->N, cudaMemcpyHostToDevice, c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_masked_scale(c->d_out, c->d_aux1, c->d_mask, fac, c->N, c->L, c->st)));
  // Neumann(src, src, 1): W_0 = src, running sum_0 = src
  int rc = neumann_real(c, c->d_aux1, c->d_aux1, c->d_aux2, 1, stop, -1, nullptr, nullptr);
  if (!rc) rc = run_images(c, c->d_aux2, s, false, dtrans, dref);
  return rc;
}

extern "C" int rte_region_gradient(rte_ctx* c, const rte_source* s, const rte_stop* stop, const double* g,
                                   const uint8_t* tiss, int ntypes, int compat, double* grada, double* grada2,
                                   double* grads, double* grads2, double* residual, double* residual2) {
  if (!c || !s || !stop || !g || !tiss || ntypes < 2 || !grada || !grada2 || !grads || !grads2)
    return fail(c, RTE_ERR_ARG, "null argument");
  if (c->kappa != 0.0 || s->modulation != 0.0) return unsupported_modulated(c, "the region gradient");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  const size_t np = (size_t)c->nx * c->ny;
  std::vector<rte_cplx> gbar(np), dg(np);
  int rc = forward_to_out(c, s, stop, gbar.data(), nullptr);
  if (rc) return rc;
  const double Cl = 1.0;          // the FisherInfo_IO speed of light (rte.h:15)
  const float av_mua = 0.01f, av_mus = 1.0f;  // compute_grad_rte.cu:115-116
  std::vector<uint8_t> mask(c->N);
  std::vector<double> fa(c->L + 1, -Cl), fs(c->L + 1);
  for (int l = 0; l <= c->L; l++) fs[l] = -Cl + pow(c->cfg.g, (double)l);  // -C out + PropScatmu1(out)
  grada[0] = grada2[0] = grads[0] = grads2[0] = 0.0;
  for (int t = 1; t < ntypes; t++) {
    bool other = false;
    for (int r = 0; r < c->N; r++) {
      mask[r] = tiss[r] == t;
      other = other || !mask[r];
    }
    rc = tangent_images(c, s, mask.data(), fa.data(), stop, dg.data(), nullptr);
    if (rc) return rc;
    double a1 = 0, a2 = 0;
    for (size_t j = 0; j < np; j++)
      if (g[j] || gbar[j].re) {
        a1 -= 2.0 * av_mua * dg[j].re / (g[j] - gbar[j].re);
        a2 -= 2.0 * av_mua * (g[j] - gbar[j].re) * dg[j].re;
      }
    grada[t] = a1;
    grada2[t] = a2;
    // the mu_s mask of the reference tests each voxel but zeroes the voxel index left over from the
    // mu_a loop (compute_grad_rte.cu:356-363): the last voxel, whenever another tissue exists
    if (compat) {
      std::fill(mask.begin(), mask.end(), (uint8_t)1);
      if (other) mask[c->N - 1] = 0;
    }
    rc = tangent_images(c, s, mask.data(), fs.data(), stop, dg.data(), nullptr);
    if (rc) return rc;
    double s1 = 0, s2 = 0;
    for (size_t j = 0; j < np; j++)
      if (g[j] || gbar[j].re) {
        s1 -= 2.0 * av_mus * dg[j].re / (g[j] - gbar[j].re);
        s2 -= 2.0 * av_mus * (g[j] - gbar[j].re) * dg[j].re;
      }
    grads[t] = s1;
    grads2[t] = s2;
  }
  double d1 = 0, d2 = 0;  // compute_grad_rte.cu:437-444
  for (size_t j = 0; j < np; j++) {
    const double e = gbar[j].re - g[j];
    if (e != 0.0) d1 += log(e * e);
    d2 += e * e;
  }
  if (residual) *residual = d1;
  if (residual2) *residual2 = d2;
  return check_kernel_err(c);
}

extern "C" int rte_fisher_regions(rte_ctx* c, const rte_source* s, const rte_stop* stop, int P, const uint8_t* masks,
                                  int image, double* F) {
  if (!c || !s || !stop || P < 1 || !masks || !F || image < 0 || image > 2) return fail(c, RTE_ERR_ARG, "bad argument");
  if (!c->medium_set) return fail(c, RTE_ERR_STATE, "medium not set");
  if (c->kappa != 0.0 || s->modulation != 0.0) return unsupported_modulated(c, "the Fisher information");
  CUDA_TRY(c, cudaSetDevice(c->cfg.device));
  const size_t np = (size_t)c->nx * c->ny;
  std::vector<rte_cplx> gt(np), gr(np), t(np), rr(np);
  int rc = forward_to_out(c, s, stop, gt.data(), gr.data());
  if (rc) return rc;
  std::vector<double> fa(c->L + 1, -1.0);  // -C mask(out), C = 1 (rte_fim.cu:270)
  std::vector<std::vector<double>> d((size_t)P);
  for (int p = 0; p < P; p++) {
    rc = tangent_images(c, s, masks + (size_t)p * c->N, fa.data(), stop, t.data(), rr.data());
    if (rc) return rc;
    d[p].resize(2 * np);
    for (size_t j = 0; j < np; j++) {
      d[p][j] = t[j].re;
      d[p][np + j] = rr[j].re;
    }
  }
  // Poisson noise: F_ab = sum_j dg_a,j dg_b,j / gbar_j over pixels with gbar_j != 0 (rte_fim.cu:316-331);
  // image 0 transmission, 1 reflection (the reference main), 2 both
  for (int a = 0; a < P; a++)
    for (int b = 0; b < P; b++) {
      double f = 0.0;
      for (int im = 0; im < 2; im++) {
        if ((image == 0 && im == 1) || (image == 1 && im == 0)) continue;
        const std::vector<rte_cplx>& gb = im ? gr : gt;
        for (size_t j = 0; j < np; j++)
          if (gb[j].re) f += (1.0 / gb[j].re) * d[a][im * np + j] * d[b][im * np + j];
      }
      F[(size_t)a * P + b] = f;
    }
  return check_kernel_err(c);
}

// ---------------------------------------------------------------------------------------
// Fisher information of parameters of the medium, from tangent (sensitivity) solves.
// For a parameter direction (dmu_a, dmu_s) per voxel and a converged forward solution
// S = sum_k (DA)^k xi, out = A S, the discrete model's derivative is
//   dS = (I - DA)^-1 [ dxi + dD (A S) + D (dA S) ],   d out = A dS + dA S,
// dA S from k_pair_tangent (path integrals of dmu_t along every pair, the kernel recomputed or read
// from the stored FP32 copy) plus the self-term derivative; dxi and the ballistic derivative of the
// collimated beam by a complex step on the host (exact to rounding).  J = d(binned flux)/dtheta and,
// with Poisson counts, F = J^T diag(1 / flux) J.

static int tangent_dA(rte_ctx* c, const double* d_in, double* d_outT, const std::vector<double>& dmut) {
  const size_t NC = (size_t)c->N * c->C;
  int lo[3] = {c->nx, c->ny, c->nz}, hi[3] = {-1, -1, -1};
  for (int r = 0; r < c->N; r++)
    if (dmut[r] != 0.0) {
      const int v[3] = {r % c->nx, (r / c->nx) % c->ny, r / (c->nx * c->ny)};
      for (int a = 0; a < 3; a++) {
        lo[a] = std::min(lo[a], v[a]);
        hi[a] = std::max(hi[a], v[a]);
      }
    }
  if (hi[0] < 0) return cudaMemsetAsync(d_outT, 0, NC * sizeof(double), c->st) == cudaSuccess
                            ? RTE_OK : fail(c, RTE_ERR_DEVICE, "memset");
  CUDA_TRY(c, cudaMemcpyAsync(c->d_dmut, dmut.data(), sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
  const int tiles = (c->N + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS;
  const int S = std::max(1, std::min(c->max_split, (4 * 148 + tiles - 1) / tiles));
  PairArgs a = pair_args(c, d_in, nullptr, 1, S, split_chunk(c->N, S));
  a.nsplit = (c->N + a.chunk - 1) / a.chunk;
  a.Kmat = c->K_valid && c->d_K ? c->d_K : nullptr;
  a.Kmat64 = c->K_valid && c->d_K64 ? c->d_K64 : nullptr;
  a.islot = c->d_islot;
  a.dmut = c->d_dmut;
  for (int q = 0; q < 3; q++) {
    a.box_lo[q] = lo[q];
    a.box_hi[q] = hi[q];
  }
  {
    ProfScope ps(c, 0);
    CUDA_TRY(c, (c->launches++, rte_launch_pair_tangent(a, c->L, c->precision == RTE_PREC_MIXED ? 0 : 1,
                                                         c->model == RTE_MODEL_FIM ? 1 : 0, c->st)));
  }
  SelfArgs sa;
  memset(&sa, 0, sizeof sa);
  sa.N = c->N;
  sa.nb = 1;
  sa.Cfull = c->C;
  sa.Cact = c->C;
  sa.K = c->K;
  sa.W = d_in;
  sa.mut = c->d_mut;
  sa.idx = c->self_lut_ok ? c->d_self_idx : nullptr;
  sa.lut = c->d_self_lut;
  sa.mom = c->d_mom;
  sa.scale = c->dV / c->cm;
  sa.air_no_self = c->model == RTE_MODEL_FIM ? 1 : 0;
  sa.out = c->d_selfp;

  sa.dmut = c->d_dmut;
  sa.dlut = c->d_dlut;
  CUDA_TRY(c, (c->launches++, rte_launch_self(sa, c->st)));
  EpiArgs e;
  memset(&e, 0, sizeof e);
  e.N = c->N;
  e.nx = c->nx;
  e.ny = c->ny;
  e.nz = c->nz;
  e.Cfull = c->C;
  e.S = a.nsplit;
  e.nb = 1;
  e.part = c->d_part;
  e.selfp = c->d_selfp;
  e.mus = c->d_mus;
  e.flag_scat = 0;
  e.Wout = d_outT;
  e.islot = c->d_islot;
  e.red = c->d_red;
  CUDA_TRY(c, cudaMemsetAsync(c->d_red, 0, 4 * sizeof(double), c->st));
  CUDA_TRY(c, (c->launches++, rte_launch_epilogue(e, c->L, c->st)));
  return RTE_OK;
}

extern "C" int rte_fisher(rte_ctx* c, int nsrc, const rte_source* srcs, const rte_stop* stop, const rte_detector* d,
                          int P, const double* dmua, const double* dmus, double* J, double* F) {
  if (!c || P < 1 || !dmua || !dmus || !F) return fail(c, RTE_ERR_ARG, "null argument");
  if (c->kappa != 0.0) return unsupported_modulated(c, "the Fisher information");
  if (c->split)
    return fail(c, RTE_ERR_UNSUPPORTED, "the Fisher information needs one tissue table (rte_set_medium_tissue_split)");
  int rc = check_detector(c, nsrc, srcs, stop, d);
  if (rc) return rc;
  for (int q = 0; q < nsrc; q++)
    if (srcs[q].kind != RTE_SRC_COLUMN && srcs[q].kind != RTE_SRC_FIM && srcs[q].kind != RTE_SRC_BEAM)
      return fail(c, RTE_ERR_UNSUPPORTED, "the Fisher information takes collimated beams");
  const size_t NC = (size_t)c->N * c->C, np = (size_t)c->nx * c->ny;
  const size_t npix = 2 * (np + (size_t)c->nz * c->nx + (size_t)c->nz * c->ny);
  const int nb = d->nbins;
  const size_t NB2 = (size_t)6 * nb * nb;
  // tangent series run together: four at L <= 5 (the widest pair-kernel batch whose accumulators fit in
  // registers) and, with the path integrals recomputed, at L >= 6 (k_pair_mixed_grp: two thread groups
  // of two sharing each pair's walk); two otherwise.  The pair walk (and at L <= 5 the SH recurrence) of
  // every pair serves the whole group.
  const bool recompute = c->kernel_mode == RTE_KERNEL_RECOMPUTE && c->model != RTE_MODEL_FIM;
  const int nbt = c->precision == RTE_PREC_MIXED ? (c->L <= 5 || recompute ? 4 : 2) : 1;
  if (nbt > 1) {
    rc = ensure_batch(c, nbt);
    if (rc) return rc;
  }
  if (!c->d_dmut) {
    CUDA_TRY(c, dalloc(c, &c->d_dmut, (size_t)c->N));
    CUDA_TRY(c, dalloc(c, &c->d_dmus, (size_t)c->N));
    CUDA_TRY(c, dalloc(c, &c->d_T, (size_t)std::max(2, nbt) * NC));  // nbt is fixed for a context (L, precision)
    CUDA_TRY(c, dalloc(c, &c->d_cidx, (size_t)std::max(c->nx, std::max(c->ny, c->nz))));
    CUDA_TRY(c, dalloc(c, &c->d_cval, (size_t)std::max(c->nx, std::max(c->ny, c->nz)) * c->C));
  }
  std::vector<double> mut(c->N), mus(c->N);
  CUDA_TRY(c, cudaMemcpy(mut.data(), c->d_mut, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
  CUDA_TRY(c, cudaMemcpy(mus.data(), c->d_mus, sizeof(double) * c->N, cudaMemcpyDeviceToHost));
  double scat[RTE_MAX_L + 1];
  scatter_factors(c, c->cfg.g != 0.0 ? 1 : 0, scat);
  const size_t a0 = np, a1 = (size_t)c->nz * c->nx, a2 = (size_t)c->nz * c->ny;
  const size_t off[6] = {0, a0, 2 * a0, 2 * a0 + a1, 2 * a0 + 2 * a1, 2 * a0 + 2 * a1 + a2};
  std::vector<double> Jpix(npix), dJ(npix), ybar(NB2), dbin(NB2), Js(NB2 * P), dmt(c->N);
  std::vector<double> coef(c->C);
  for (int q = 0; q < P * P; q++) F[q] = 0.0;
  const double h = 1e-20;  // complex-step increment
  for (int si = 0; si < nsrc; si++) {
    const rte_source* s = &srcs[si];
    int terms = 0;
    // the forward solve (S -> d_S, out -> d_out, flux -> Jpix) by the FP64 method, path integrals
    // recomputed: F weights every bin by 1 / flux, and in the mixed series the flux of dim bins
    // (1e-6..1e-4 of the brightest) carries up to ~1e-4 relative error, which F inherits (25^3 L=5, 6
    // beams: F 5.4e-5 from FP64 with mixed forward solves, 1.9e-6 with FP64 ones; J 2.5e-6 either way)
    const int prec = c->precision, mode = c->kernel_mode;
    c->precision = RTE_PREC_FP64;
    if (prec != RTE_PREC_FP64) c->kernel_mode = RTE_KERNEL_RECOMPUTE;
    rc = forward_with_flux(c, s, stop, Jpix, &terms);
    c->precision = prec;
    c->kernel_mode = mode;
    if (rc) return rc;
    bin_faces(c, d, Jpix, ybar.data());
    std::vector<int> cols;
    double scale = 1.0;
    source_columns(c, s, cols, scale);
    const int face = source_face(s);
    const int ncol = face < 2 ? c->nz : (face < 4 ? c->ny : c->nx);
    const double dlen = face < 2 ? c->dz : (face < 4 ? c->dy : c->dx);
    beam_coefs(c, face, scale, coef.data());
    // parameters in groups of nbt: the tangent series of a group run together (mixed precision)
    for (int p0 = 0; p0 < P; p0 += nbt) {
      const int vs = nbt * c->C;
      double* q = nbt == 1 ? c->d_aux1 : c->d_bW;
      if (nbt > 1) CUDA_TRY(c, cudaMemsetAsync(q, 0, NC * nbt * sizeof(double), c->st));
      double dball[4] = {0, 0, 0, 0};
      int ball_pix = -1;
      for (int b = 0; b < nbt && p0 + b < P; b++) {
        const int p = p0 + b;
        const double* da = dmua + (size_t)p * c->N;
        const double* ds = dmus + (size_t)p * c->N;
        for (int r = 0; r < c->N; r++) dmt[r] = da[r] + ds[r];
        rc = tangent_dA(c, c->d_S, c->d_T + (size_t)b * NC, dmt);  // T = dA S
        if (rc) return rc;
        CUDA_TRY(c, cudaMemcpyAsync(c->d_dmus, ds, sizeof(double) * c->N, cudaMemcpyHostToDevice, c->st));
        CUDA_TRY(c, (c->launches++, rte_launch_tangent_rhs(q + (size_t)b * c->C, vs, c->d_T + (size_t)b * NC, c->d_out,
                                                             c->d_mus, c->d_dmus, scat, c->N, c->L, c->st)));
        // the beam's source column and ballistic transmission, differentiated by a complex step
        if (!cols.empty()) {
          std::vector<int> idx(ncol);
          std::vector<double> vals((size_t)ncol * c->C);
          std::complex<double> att(1.0, 0.0);
          for (int t = 0; t < ncol; t++) {
            const int r = face_voxel(c, face, cols[0], t);
            idx[t] = r;
            const std::complex<double> mt(mut[r], h * dmt[r]), ms(mus[r], h * ds[r]);
            const std::complex<double> e = std::exp(-mt * dlen);
            const std::complex<double> amp = ms / mt * (att * (1.0 - e)) / c->dV;
            att *= e;
            for (int k = 0; k < c->C; k++) vals[(size_t)t * c->C + k] = amp.imag() / h * coef[k];
          }
          dball[b] = s->mag * att.imag() / h;
          ball_pix = (int)(off[face ^ 1] + cols[0]);
          CUDA_TRY(c, cudaMemcpyAsync(c->d_cidx, idx.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice, c->st));
          CUDA_TRY(c, cudaMemcpyAsync(c->d_cval, vals.data(), sizeof(double) * vals.size(), cudaMemcpyHostToDevice,
                                      c->st));
          CUDA_TRY(c, (c->launches++, rte_launch_scatter_add(q + (size_t)b * c->C, vs, c->d_cidx, c->d_cval, ncol, c->C,
                                                               c->st)));
        }
      }
      // dS = (I - DA)^-1 q; the series returns A dS
      const double* res;
      if (nbt == 1) {
        rc = neumann_real(c, q, q, c->d_aux2, 1, stop, -1, nullptr, nullptr);
        res = c->d_aux2;
      } else {
        CUDA_TRY(c, cudaMemcpyAsync(c->d_bsum, q, NC * nbt * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        rc = series_batch(c, nbt, stop, nullptr, nullptr);
        res = c->d_bres;
      }
      if (rc) return rc;
      for (int b = 0; b < nbt && p0 + b < P; b++) {
        const int p = p0 + b;
        // d out = A dS + dA S
        CUDA_TRY(c, (c->launches++, rte_launch_strided_add(c->d_aux4, res + (size_t)b * c->C, vs,
                                                             c->d_T + (size_t)b * NC, c->N, c->C, c->st)));
        FaceArgs fa;
        memset(&fa, 0, sizeof fa);
        fa.nx = c->nx;
        fa.ny = c->ny;
        fa.nz = c->nz;
        fa.Cfull = c->C;
        fa.vstride = c->C;
        fa.out = c->d_aux4;
        fa.h = c->d_h;
        fa.J = c->d_J;
        CUDA_TRY(c, (c->launches++, rte_launch_face_flux(fa, c->st)));
        CUDA_TRY(c, cudaMemcpyAsync(dJ.data(), c->d_J, npix * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CUDA_TRY(c, cudaStreamSynchronize(c->st));
        if (ball_pix >= 0) dJ[ball_pix] += dball[b];
        bin_faces(c, d, dJ, dbin.data());
        for (size_t k = 0; k < NB2; k++) Js[k * P + p] = ((d->faces >> (k / ((size_t)nb * nb))) & 1) ? dbin[k] : 0.0;
      }
    }
    rc = check_kernel_err(c);
    if (rc) return rc;
    if (J) memcpy(J + (size_t)si * NB2 * P, Js.data(), sizeof(double) * NB2 * P);
    for (size_t b = 0; b < NB2; b++) {
      if (!((d->faces >> (b / ((size_t)nb * nb))) & 1) || !(ybar[b] > 0.0)) continue;
      const double w = 1.0 / ybar[b];
      const double* jb = &Js[b * P];
      for (int p = 0; p < P; p++)
        for (int q = 0; q < P; q++) F[(size_t)p * P + q] += w * jb[p] * jb[q];
    }
  }
  return RTE_OK;
}
