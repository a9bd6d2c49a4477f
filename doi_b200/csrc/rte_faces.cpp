// rte_faces.cpp -- the CPU package's boundary outputs of a final distribution: the side-face images
// (CPU package/src/Dist.c:353-532) and the photon number (Dist.c:538-989).
//
// Each output is a sum over one boundary voxel layer of w_f . W(voxel), with per-coefficient weights
//   w_f[m] = (c/n) * area * sum_{101 x 101 (theta, phi) points} Y_m(theta, phi) sin(theta) dtheta dphi (n . s)
// over a hemisphere (a left-endpoint rectangle rule, as the package integrates).  The package
// re-evaluates the quadrature for every pixel and coefficient; here the weights are computed once
// per hemisphere and applied to every pixel, the same arithmetic in a different order.  Host code:
// the work is a few face layers of the distribution.
#include <math.h>
#include <string.h>

#include <complex>
#include <vector>

#include "../../include/rte_b200.h"
#include "rte_internal.h"

namespace {

typedef std::complex<double> cd;

// Complex SH of the reference (Y_lm = N P_l^|m| e^{i|m| phi}, Y_l,-m = (-1)^m conj(Y_lm)) from
// the real basis: Y_l0 = R_l0, Y_lm = (R_l,m + i R_l,-m) / sqrt(2) for m > 0.
void sh_complex(const ShTables& t, int L, double th, double ph, cd* Y) {
  const int C = (L + 1) * (L + 1);
  std::vector<double> R(C);
  sh_real_host(t, L, sin(th) * cos(ph), sin(th) * sin(ph), cos(th), R.data());
  for (int l = 0; l <= L; l++) {
    Y[l * l + l] = R[l * l + l];
    for (int m = 1; m <= l; m++) {
      const cd y = cd(R[l * l + l + m], R[l * l + l - m]) / sqrt(2.0);
      Y[l * l + l + m] = y;
      Y[l * l + l - m] = ((m & 1) ? -1.0 : 1.0) * std::conj(y);
    }
  }
}

// The six hemisphere rules of the package: theta / phi start and range, and the direction factor
// n . s of the face normal they go with.
enum Dir { COS, NEG_COS, NEG_SINCOS, SINCOS, NEG_SINSIN, SINSIN };
struct Rule {
  double th0, thr, ph0, phr;
  Dir dir;
};
const Rule kRules[6] = {
    {0.0, M_PI / 2.0, 0.0, 2.0 * M_PI, COS},               // +z hemisphere (Dist.c:566-572)
    {M_PI / 2.0, M_PI / 2.0, 0.0, 2.0 * M_PI, NEG_COS},     // -z (Dist.c:653-659)
    {0.0, M_PI, M_PI / 2.0, M_PI, NEG_SINCOS},              // -x (Dist.c:376-381)
    {0.0, M_PI, -M_PI / 2.0, M_PI, SINCOS},                 // +x (Dist.c:412-418)
    {0.0, M_PI, M_PI, M_PI, NEG_SINSIN},                    // -y (Dist.c:449-455)
    {0.0, M_PI, 0.0, M_PI, SINSIN},                         // +y (Dist.c:489-495)
};

std::vector<cd> rule_weights(const ShTables& t, int L, const Rule& q, double area_cn, int num) {
  const int C = (L + 1) * (L + 1);
  std::vector<cd> w(C, 0.0), Y(C);
  const double dth = q.thr / num, dph = q.phr / num;
  for (int ip = 0; ip < num; ip++)
    for (int jp = 0; jp < num; jp++) {
      const double th = ip * q.thr / num + q.th0, ph = jp * q.phr / num + q.ph0;
      double d;
      switch (q.dir) {
        case COS: d = cos(th); break;
        case NEG_COS: d = -cos(th); break;
        case NEG_SINCOS: d = -sin(th) * cos(ph); break;
        case SINCOS: d = sin(th) * cos(ph); break;
        case NEG_SINSIN: d = -sin(th) * sin(ph); break;
        default: d = sin(th) * sin(ph); break;
      }
      sh_complex(t, L, th, ph, Y.data());
      const double f = area_cn * sin(th) * dth * dph * d;
      for (int m = 0; m < C; m++) w[m] += f * Y[m];
    }
  return w;
}

}  // namespace

extern "C" int rte_cpu_face_outputs(const rte_config* cfg, const rte_cplx* W, const rte_source* src, double mu_t,
                                    double mu_t_im, rte_cplx* side_x0, rte_cplx* side_x1, rte_cplx* side_y0,
                                    rte_cplx* side_y1, rte_cplx* photons) {
  if (!cfg || !W || cfg->nL < 0 || cfg->nL > RTE_MAX_L || cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1)
    return RTE_ERR_ARG;
  const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, L = cfg->nL, C = (L + 1) * (L + 1);
  const double dx = (cfg->x_max - cfg->x_min) / nx, dy = (cfg->y_max - cfg->y_min) / ny,
               dz = (cfg->z_max - cfg->z_min) / nz;
  const double cn = cfg->c / cfg->n;
  const ShTables t = make_sh_tables();
  const int num = 101;
  auto at = [&](int i, int j, int k) { return reinterpret_cast<const cd*>(W) + ((size_t)(k * ny + j) * nx + i) * C; };
  auto dot = [&](const std::vector<cd>& w, const cd* v) {
    cd s = 0.0;
    for (int m = 0; m < C; m++) s = w[m] * v[m] + s;
    return s;
  };
  cd total = 0.0;
  // z faces (photon number only): +z rule on the last layer (outgoing, with the ballistic beam) and
  // on the first layer; -z rule on the first and the last layer
  for (int r = 0; r < 2; r++) {
    const std::vector<cd> w = rule_weights(t, L, kRules[r], dx * dy * cn, num);
    for (int pass = 0; pass < 2; pass++) {
      const int k = (r == 0) == (pass == 0) ? nz - 1 : 0;
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
          cd v = 0.0;
          if (r == 0 && pass == 0 && src) {  // Dist.c:589-596
            const double xs = i * dx + cfg->x_min + dx / 2.0, ys = j * dy + cfg->y_min + dy / 2.0;
            const double zs = k * dz + cfg->z_min + dz / 2.0;
            const double rad = sqrt((xs - src->pos_x) * (xs - src->pos_x) + (ys - src->pos_y) * (ys - src->pos_y));
            if (rad <= (src->diam + 1.0e-16) / 2.0) v = src->mag * std::exp(-cd(mu_t, mu_t_im) * (zs + dz / 2.0));
          }
          total += dot(w, at(i, j, k)) + v;
        }
    }
  }
  // x and y faces: the side images (the outgoing layer of each rule) and both photon-number sums
  rte_cplx* imgs[4] = {side_x0, side_x1, side_y0, side_y1};
  for (int r = 2; r < 6; r++) {
    const bool xface = r < 4;
    const std::vector<cd> w = rule_weights(t, L, kRules[r], (xface ? dz * dy : dx * dz) * cn, num);
    const bool lowface = (r & 1) == 0;  // -x / -y rules go out through the low face
    for (int pass = 0; pass < 2; pass++) {
      const bool low = lowface == (pass == 0);
      for (int k = 0; k < nz; k++)
        for (int u = 0; u < (xface ? ny : nx); u++) {
          const int i = xface ? (low ? 0 : nx - 1) : u, j = xface ? u : (low ? 0 : ny - 1);
          const cd v = dot(w, at(i, j, k));
          total += v;
          if (pass == 0 && imgs[r - 2]) imgs[r - 2][k + (size_t)u * nz] = rte_cplx{v.real(), v.imag()};
        }
    }
  }
  if (photons) *photons = rte_cplx{total.real(), total.imag()};
  return RTE_OK;
}
