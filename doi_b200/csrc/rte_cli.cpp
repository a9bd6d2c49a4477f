// rte_cli.cpp -- the reference's command-line programs over the B200 library.
//
//   rte_gpu file.par   forward solve (FisherInfo_IO/src/rte.cu:92-236; the CPU package's
//                      RTE_uniform.c for uniform-medium files): source, Neumann series with the
//                      reference stop rule, transmission / reflection / phase images written to
//                      [Runtime] TransFile / ReflectFile / PhaseFile in the reference's layout
//   rte_inv file.par   region gradients of the transmission misfit against [Runtime] gFile
//                      (FisherInfo_IO/src/compute_grad_rte.cu:205-385), one line per tissue type
//   rte_fim file.par   Fisher information of the mu_a of a spherical region on the reflection
//                      image (FisherInfo_IO/src/rte_fim.cu:236-331)
//   rte_snr file.par   detection SNR of a mu_a lesion against depth (FisherInfo_IO/src/rte_snr.cu)
//
// One executable; the program is chosen by the name it is called under (build.py links the three
// names).  Argument and error conventions follow the reference mains: a usage line and exit status 1
// for a wrong argument count; a message and a non-zero status for unreadable inputs.
#include <libgen.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <stdint.h>

#include <algorithm>
#include <complex>
#include <string>
#include <vector>

#include "../../include/rte_b200.h"

namespace {

int die(rte_ctx* ctx, const char* what, int rc) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, rte_last_error(ctx));
  return 1;
}

struct Loaded {
  rte_par* par = nullptr;
  rte_problem pr;
  rte_ctx* ctx = nullptr;
  ~Loaded() {
    if (ctx) rte_destroy(ctx);
    rte_problem_free(&pr);
    rte_par_free(par);
  }
};

// .par -> context with the medium set.  `forward_rule` applies the forward main's diffuse-medium
// propThresh (rte.cu:116-119), which the gradient and Fisher mains do not have.
int load(const char* path, bool forward_rule, Loaded& L, int read_map = 1) {
  memset(&L.pr, 0, sizeof L.pr);
  int rc = rte_par_load(path, &L.par);
  if (rc) {
    fprintf(stderr, "cannot read parameter file %s\n", path);
    return 1;
  }
  rc = rte_par_problem(L.par, read_map, &L.pr);
  if (rc) {
    fprintf(stderr, "bad parameter file %s (%d): geometry, nL, tissue map or medium files\n", path, rc);
    return 1;
  }
  rte_config cfg = L.pr.cfg;
  if (forward_rule && L.pr.style == 0) cfg.prop_thresh = L.pr.diffuse_prop_thresh;
  rc = rte_create(&cfg, &L.ctx);
  if (rc) return die(nullptr, "rte_create", rc);
  if (L.pr.mua_vox)
    rc = rte_set_medium_voxel(L.ctx, L.pr.mua_vox, L.pr.mus_vox);
  else
    rc = rte_set_medium_tissue(L.ctx, L.pr.tiss, L.pr.ntypes, L.pr.mua, L.pr.mus);
  if (rc) return die(L.ctx, "set medium", rc);
  return 0;
}

double mut_at(const rte_problem& pr, size_t r) {
  return pr.mua_vox ? pr.mua_vox[r] + pr.mus_vox[r] : pr.mua[pr.tiss[r]] + pr.mus[pr.tiss[r]];
}

// Phase image of the forward main (dist.cu:163-226): the diffuse transmission plus the ballistic
// transmission of every column whose centre lies strictly inside the beam's diameter, then arg().
std::vector<double> phase_image(const Loaded& L, const std::vector<rte_cplx>& W) {
  const rte_config& c = L.pr.cfg;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  std::vector<rte_cplx> tr((size_t)nx * ny);
  std::vector<double> ph((size_t)nx * ny, 0.0);
  if (rte_images(L.ctx, W.data(), nullptr, tr.data(), nullptr)) return ph;
  const double dx = (c.x_max - c.x_min) / nx, dy = (c.y_max - c.y_min) / ny, dz = (c.z_max - c.z_min) / nz;
  const rte_source& s = L.pr.src;
  for (int j = 0; j < ny; j++)
    for (int k = 0; k < nx; k++) {
      std::complex<double> v(tr[(size_t)j * nx + k].re, tr[(size_t)j * nx + k].im);
      const double xs = k * dx + c.x_min + dx / 2.0, ys = j * dy + c.y_min + dy / 2.0;
      if (sqrt(pow(s.pos_x - xs, 2) + pow(s.pos_y - ys, 2)) < s.diam / 2.0) {
        double t = s.mag;
        for (int i = 0; i < nz; i++) t *= exp(-mut_at(L.pr, ((size_t)i * ny + j) * nx + k) * dz);
        v += t;
      }
      ph[(size_t)j * nx + k] = std::arg(v);
    }
  return ph;
}

typedef std::complex<double> cd;

// Source columns of the CPU package's beam (GenerateSourceBeam, Dist.c:1087-1093: voxel centres in
// the circle |xy - pos| <= diam/2; the library adds 1e-16 to diam/2 against rounding at the rim).
int cpu_columns(const rte_config& c, const rte_source& s) {
  const double dx = (c.x_max - c.x_min) / c.nx, dy = (c.y_max - c.y_min) / c.ny;
  int n = 0;
  for (int j = 0; j < c.ny; j++)
    for (int k = 0; k < c.nx; k++) {
      const double xs = k * dx + c.x_min + dx / 2.0, ys = j * dy + c.y_min + dy / 2.0;
      if (sqrt((xs - s.pos_x) * (xs - s.pos_x) + (ys - s.pos_y) * (ys - s.pos_y)) <= (s.diam + 1.0e-16) / 2.0) n++;
    }
  return n;
}

// StopIteration of the CPU package (Kernels_selfsub.c:1184-1220): real parts of all coefficients on
// the layer z = nZ-1.
bool cpu_stop(const rte_config& c, double& fi, int n, const std::vector<rte_cplx>& W, const std::vector<rte_cplx>& out) {
  const size_t C = (size_t)(c.nL + 1) * (c.nL + 1), plane = (size_t)c.nx * c.ny;
  double sw = 0.0, so = 0.0;
  for (size_t q = (size_t)(c.nz - 1) * plane * C; q < (size_t)c.nz * plane * C; q++) {
    sw += W[q].re;
    so += out[q].re;
  }
  double hi = 0.0;
  if (n > 1) {
    if (so == 0.0) return true;
    hi = 1.0 - (sw / so) * (1.0 / (1.0 - (sw / so) / fi));
    fi = sw / so;
    if (hi > 1.0 || hi < 0.0) hi = 0.0;
  }
  return hi > 0.9999;
}

// ComputePhaseImage (CPU package/src/Dist.c:71-131): the diffuse transmission with the weight
// 1/(100-1) per abscissa (the transmission image uses 1/100) plus the ballistic beam with the package's
// current mu_t and magnitude, then arg() in degrees.
std::vector<double> cpu_phase_image(rte_ctx* ctx, const rte_config& c, const std::vector<rte_cplx>& W,
                                    const rte_source& s, double mag, cd mut) {
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  std::vector<rte_cplx> tr((size_t)nx * ny);
  std::vector<double> ph((size_t)nx * ny, 0.0);
  if (rte_images(ctx, W.data(), nullptr, tr.data(), nullptr)) return ph;
  const double dx = (c.x_max - c.x_min) / nx, dy = (c.y_max - c.y_min) / ny, dz = (c.z_max - c.z_min) / nz;
  const double zs = (nz - 1) * dz + c.z_min + dz / 2.0;
  for (int j = 0; j < ny; j++)
    for (int k = 0; k < nx; k++) {
      cd v = cd(tr[(size_t)j * nx + k].re, tr[(size_t)j * nx + k].im) * (100.0 / 99.0);
      const double xs = k * dx + c.x_min + dx / 2.0, ys = j * dy + c.y_min + dy / 2.0;
      if (sqrt((xs - s.pos_x) * (xs - s.pos_x) + (ys - s.pos_y) * (ys - s.pos_y)) <= s.diam / 2.0)
        v += mag * std::exp(-mut * (zs + dz / 2.0));
      ph[(size_t)j * nx + k] = std::arg(v) * 180.0 / M_PI;
    }
  return ph;
}

int write_cpu_faces(const Loaded& L, const std::vector<rte_cplx>& W, const rte_source& s, cd mut) {
  const rte_config& c = L.pr.cfg;
  const size_t np = (size_t)c.nx * c.ny;
  std::vector<rte_cplx> sx0((size_t)c.nz * c.ny), sx1(sx0.size()), sy0((size_t)c.nz * c.nx), sy1(sy0.size());
  rte_cplx ph{0, 0};
  int rc = rte_cpu_face_outputs(&c, W.data(), &s, mut.real(), mut.imag(), sx0.data(), sx1.data(), sy0.data(),
                                sy1.data(), &ph);
  if (rc) return die(L.ctx, "rte_cpu_face_outputs", rc);
  const char* names[4] = {"SideFace1(-X).out", "SideFace2(+X).out", "SideFace3(-Y).out", "SideFace4(+Y).out"};
  std::vector<rte_cplx>* imgs[4] = {&sx0, &sx1, &sy0, &sy1};
  for (int q = 0; q < 4; q++) {
    // the package writes these buffers through its z-face writer (nX x nY values read in order)
    std::vector<rte_cplx> buf(np, rte_cplx{0, 0});
    for (size_t e = 0; e < np && e < imgs[q]->size(); e++) buf[e] = (*imgs[q])[e];
    if ((rc = rte_write_image(names[q], c.nx, c.ny, buf.data(), 1))) return die(L.ctx, names[q], rc);
  }
  printf("Number of photons total: %f\n", ph.re);
  return 0;
}

// The CPU package's main (RTE_uniform.c:64-196) on a uniform-medium file.  Steady state: source,
// Neumann series with the package's stop rule, final A.  With [Source] modulation != 0 the package
// continues as written: the source is built again with the real mu_a (GenerateSourceBeam divides the
// magnitude by the column count once more, Dist.c:1113-1114), mu_a gains i modulation/(c/n), the
// modulated terms (D A)^n src are added to the steady-state result itself under its stop rule, the
// modulated output is A src alone, its phase image is written, and the images come from
// CombineOuts = 0.5 out + 0.25 out2 + 0.25 conj(out2) (Dist.c:1294-1303).  Reproduced step by step.
int forward_cpu_package(Loaded& L, std::vector<rte_cplx>& W, std::vector<rte_cplx>& tr, std::vector<rte_cplx>& rf,
                        rte_report& rep) {
  const rte_config& c = L.pr.cfg;
  const size_t N = (size_t)c.nx * c.ny * c.nz, C = (size_t)(c.nL + 1) * (c.nL + 1);
  const double modulation = L.pr.src.modulation;
  rte_source s = L.pr.src;
  s.modulation = 0.0;
  int rc = rte_forward(L.ctx, &s, &L.pr.stop, W.data(), tr.data(), rf.data(), &rep);
  if (rc) return die(L.ctx, "rte_forward", rc);
  printf("Neumann series: %d terms, %.3f ms on the device\n", rep.terms, rep.ms_device);
  const int cols = std::max(1, cpu_columns(c, s));
  const double mut = L.pr.mua[1] + L.pr.mus[1];
  s.mag = L.pr.src.mag / cols;  // source->mag after GenerateSourceBeam
  std::vector<rte_cplx> out2 = W;
  cd mutc(mut, 0.0);
  if (modulation != 0.0) {
    std::vector<rte_cplx> xi(N * C), Wn(N * C);
    if ((rc = rte_source_beam(L.ctx, &s, xi.data()))) return die(L.ctx, "rte_source_beam", rc);
    if ((rc = rte_set_modulation(L.ctx, modulation))) return die(L.ctx, "rte_set_modulation", rc);
    s.mag /= cols;  // the second GenerateSourceBeam
    s.modulation = modulation;
    mutc = cd(mut, modulation / (c.c / c.n));
    std::vector<rte_cplx> Wk = xi;
    const int flag = c.g != 0.0 ? 1 : 0;
    double fi = 1.0;
    int n = 1;
    while (!cpu_stop(c, fi, n, Wk, W) && n <= 10000) {
      if ((rc = rte_prop_abs(L.ctx, Wk.data(), Wn.data(), flag, 1))) return die(L.ctx, "rte_prop_abs", rc);
      Wk.swap(Wn);
      for (size_t q = 0; q < N * C; q++) {
        W[q].re += Wk[q].re;
        W[q].im += Wk[q].im;
      }
      n++;
    }
    printf("Neumann series (modulated): %d terms\n", n - 1);
    if ((rc = rte_prop_abs(L.ctx, xi.data(), out2.data(), 1, 0))) return die(L.ctx, "rte_prop_abs", rc);
  }
  if (L.pr.phase_file[0]) {
    const std::vector<double> ph = cpu_phase_image(L.ctx, c, out2, s, s.mag, mutc);
    if ((rc = rte_write_phase_image(L.pr.phase_file, c.nx, c.ny, ph.data(), 1))) return die(L.ctx, L.pr.phase_file, rc);
  }
  if (modulation != 0.0) {
    for (size_t q = 0; q < N * C; q++) {  // CombineOuts: out2 = 0.5 out + 0.5 Re(out2) per coefficient
      W[q].re = 0.5 * W[q].re + 0.5 * out2[q].re;
      W[q].im = 0.5 * W[q].im;
    }
    rte_source si = s;
    si.mag = s.mag * cols;  // the library divides by the column count itself
    if ((rc = rte_images(L.ctx, W.data(), &si, tr.data(), rf.data()))) return die(L.ctx, "rte_images", rc);
  }
  return write_cpu_faces(L, W, s, mutc);
}

int main_forward(const char* path) {
  Loaded L;
  if (load(path, true, L)) return 1;
  const rte_config& c = L.pr.cfg;
  const size_t N = (size_t)c.nx * c.ny * c.nz, C = (size_t)(c.nL + 1) * (c.nL + 1), np = (size_t)c.nx * c.ny;
  std::vector<rte_cplx> W(N * C), tr(np), rf(np);
  rte_report rep;
  int rc;
  const int cpu_layout = L.pr.style == 1;
  if (L.pr.style == 1) {
    if ((rc = forward_cpu_package(L, W, tr, rf, rep))) return rc;
  } else {
    // FisherInfo_IO reads [Source] modulation and does not use it; the exact model solves with it
    if (c.model == RTE_MODEL_FIM) L.pr.src.modulation = 0.0;
    rc = rte_forward(L.ctx, &L.pr.src, &L.pr.stop, W.data(), tr.data(), rf.data(), &rep);
    if (rc) return die(L.ctx, "rte_forward", rc);
    printf("Neumann series: %d terms, %.3f ms on the device\n", rep.terms, rep.ms_device);
  }
  if (L.pr.trans_file[0] && (rc = rte_write_image(L.pr.trans_file, c.nx, c.ny, tr.data(), cpu_layout)))
    return die(L.ctx, L.pr.trans_file, rc);
  if (L.pr.ref_file[0] && (rc = rte_write_image(L.pr.ref_file, c.nx, c.ny, rf.data(), cpu_layout)))
    return die(L.ctx, L.pr.ref_file, rc);
  if (L.pr.phase_file[0] && L.pr.style == 0) {
    std::vector<double> ph;
    if (L.pr.src.modulation != 0.0) {  // the modulated transmission (ballistic included): its phase delay
      ph.resize(np);
      for (size_t q = 0; q < np; q++) ph[q] = std::arg(cd(tr[q].re, tr[q].im));
    } else {
      ph = phase_image(L, W);
    }
    if ((rc = rte_write_phase_image(L.pr.phase_file, c.nx, c.ny, ph.data(), 0))) return die(L.ctx, L.pr.phase_file, rc);
  }
  if (L.pr.flux_file[0] && L.pr.detector_bins > 0) {  // binned exitant flux on all six faces
    rte_stop st = L.pr.stop;
    if (st.rule == RTE_STOP_REFERENCE) st = rte_stop{RTE_STOP_FIXED, rep.terms, 0.0};
    rte_detector det{L.pr.detector_bins, 63};
    std::vector<double> flux((size_t)6 * det.nbins * det.nbins);
    if ((rc = rte_detector_flux(L.ctx, 1, &L.pr.src, &st, &det, flux.data()))) return die(L.ctx, "rte_detector_flux", rc);
    FILE* f = fopen(L.pr.flux_file, "wb");
    if (!f || fwrite(flux.data(), sizeof(double), flux.size(), f) != flux.size()) {
      fprintf(stderr, "cannot write %s\n", L.pr.flux_file);
      if (f) fclose(f);
      return 1;
    }
    fclose(f);
  }
  return 0;
}

int main_inverse(const char* path) {
  Loaded L;
  if (load(path, false, L)) return 1;
  const rte_config& c = L.pr.cfg;
  const size_t np = (size_t)c.nx * c.ny;
  std::vector<double> g(np);
  int rc = L.pr.g_file[0] ? rte_read_image(L.pr.g_file, c.nx, c.ny, g.data()) : RTE_ERR_IO;
  if (rc) {
    fprintf(stderr, "Error in opening gfile. Exiting \n");
    return 1;
  }
  const int nt = L.pr.ntypes;
  std::vector<double> ga(nt), ga2(nt), gs(nt), gs2(nt), mua(L.pr.mua, L.pr.mua + nt), mus(L.pr.mus, L.pr.mus + nt);
  // [Algorithm] ReferenceQuirks = 1 (default): the main's device tissue table keeps the .par values
  // (populate_info_dev()'s result is dropped, compute_grad_rte.cu:431), so the path integrals and the
  // scatter use them while the source, self-voxel term and images take the swept values; 0: the swept
  // values throughout
  const int quirks = rte_par_get_int(L.par, "Algorithm:ReferenceQuirks", 1);
  FILE* resf = fopen("Residual.out", "wb");
  // the main sweeps tissue 1 over a fixed grid of values, one gradient evaluation per iteration
  // (compute_grad_rte.cu:207-209); its parameter update is disabled in the reference
  for (int itt = 0; itt < L.pr.num_iterations; itt++) {
    mus[1] = 0.8 + round(itt / 2.0) * 0.05;
    mua[1] = 0.008 + floor(itt / 2.0) * 0.0005;
    rc = quirks ? rte_set_medium_tissue_split(L.ctx, L.pr.tiss, nt, mua.data(), mus.data(), L.pr.mua, L.pr.mus)
                : rte_set_medium_tissue(L.ctx, L.pr.tiss, nt, mua.data(), mus.data());
    if (rc) return die(L.ctx, "set medium", rc);
    double res = 0, res2 = 0;
    rc = rte_region_gradient(L.ctx, &L.pr.src, &L.pr.stop, g.data(), L.pr.tiss, nt, 1, ga.data(), ga2.data(),
                             gs.data(), gs2.data(), &res, &res2);
    if (rc) return die(L.ctx, "rte_region_gradient", rc);
    printf("Iteration No %d \n", itt);
    for (int t = 1; t < nt; t++) {
      printf("Value of mua = %e mus = %e \n", mua[t], mus[t]);
      printf("Value of mua grad1 = %e musgrad1 = %e \n", ga[t], gs[t]);
      printf("Value of mua grad2 = %e musgrad2 = %e \n", ga2[t], gs2[t]);
    }
    printf("Residual = %e\n", res);
    printf("Residual2 = %e\n", res2);
    if (resf) fwrite(&res, sizeof(double), 1, resf);
  }
  if (resf) fclose(resf);
  return 0;
}

// rte_snr (FisherInfo_IO/src/rte_snr.cu:80-385): squared detection SNR of a spherical mu_a lesion
// (radius 3 fov / (2 nX), tissue 2, mu_a 0.35 against 0.25, mu_s 1) at depths z index 2 .. 15 on the
// reflection image, SNR^2 = sum_j (g1_j - g0_j)^2 / g0_j, written to snr_terms.dat (nZ - 2 doubles).
// The reference steps its depth loop with `loc_indz = loc_indz++` (undefined in C; under gcc the index
// never advances); here it steps by one and stops at the last layer of small grids.
// [Algorithm] ReferenceQuirks = 1 (default) reproduces what the main computes at each depth: its device
// tissue table keeps the .par values (rte_snr.cu:239 drops populate_info_dev()'s result), so the path
// integrals and the scatter use them while the source, self-voxel term and images take the lesion's
// values, and its z coordinate array is filled only for indices below nX (rte_snr.cu:175-179; the rest
// read as 0).  0: the lesion's values throughout and every z coordinate.
int main_snr(const char* path) {
  Loaded L;
  if (load(path, false, L)) return 1;
  const rte_config& c = L.pr.cfg;
  const size_t N = (size_t)c.nx * c.ny * c.nz, np = (size_t)c.nx * c.ny;
  FILE* gf = L.pr.g_file[0] ? fopen(L.pr.g_file, "rb") : nullptr;
  if (!gf) {
    printf("Error in opening gfile. Exiting \n");
    return 0;
  }
  fclose(gf);
  if (L.pr.ntypes < 3) {
    fprintf(stderr, "rte_snr needs NoTiss >= 2 (the lesion is tissue 2)\n");
    return 1;
  }
  const int max_ind = 10;
  double mua_tab[max_ind], mus_tab[max_ind];
  for (int q = 0; q < max_ind; q++) {
    mus_tab[q] = q * 0.25 + 0.25;
    mua_tab[q] = q * 0.0025 + 0.0025;
  }
  auto dump = [](const char* name, const double* v, size_t n) {
    FILE* f = fopen(name, "wb");
    if (f) {
      if (n) fwrite(v, sizeof(double), n, f);
      fclose(f);
    }
  };
  dump("abs_co_fim.dat", mua_tab, max_ind);
  dump("sc_co_fim.dat", mus_tab, max_ind);
  for (const char* nm : {"grada_terms_fim.dat", "grads_terms_fim.dat", "res_terms_fim.dat", "fim_terms.dat"})
    dump(nm, nullptr, 0);
  const double fov = c.x_max - c.x_min;
  auto X = [&](int i) { return i * fov / c.nx - fov / 2 + fov / (2 * c.nx); };
  auto Y = [&](int i) { return i * fov / c.ny - fov / 2 + fov / (2 * c.ny); };
  const int quirks = rte_par_get_int(L.par, "Algorithm:ReferenceQuirks", 1);
  auto Z = [&](int i) { return (quirks && i >= c.nx) ? 0.0 : i * fov / c.nz + fov / (2 * c.nz); };
  const float rad = (float)(3 * fov / (2 * c.nx));
  const float rad2 = rad * rad;
  const int initz = 2, lx = c.nx / 2, ly = c.ny / 2;
  std::vector<double> snr(c.nz > initz ? c.nz - initz : 0, 0.0);
  std::vector<uint8_t> tiss(N);
  std::vector<double> ta(L.pr.mua, L.pr.mua + L.pr.ntypes), ts(L.pr.mus, L.pr.mus + L.pr.ntypes);
  std::vector<rte_cplx> tr(np), g1(np), g0(np);
  for (int lz = initz; lz < 16 && lz < c.nz; lz++) {
    for (int i = 0; i < c.nz; i++)
      for (int j = 0; j < c.ny; j++)
        for (int k = 0; k < c.nx; k++) {
          const double d2 = (X(k) - X(lx)) * (X(k) - X(lx)) + (Y(j) - Y(ly)) * (Y(j) - Y(ly)) + (Z(i) - Z(lz)) * (Z(i) - Z(lz));
          tiss[((size_t)i * c.ny + j) * c.nx + k] = d2 < (double)rad2 ? 2 : 1;
        }
    for (int hyp = 1; hyp >= 0; hyp--) {
      ta[2] = 0.25 + 0.1 * hyp;
      ts[2] = 1.0;
      int rc = quirks ? rte_set_medium_tissue_split(L.ctx, tiss.data(), L.pr.ntypes, ta.data(), ts.data(), L.pr.mua,
                                                    L.pr.mus)
                      : rte_set_medium_tissue(L.ctx, tiss.data(), L.pr.ntypes, ta.data(), ts.data());
      if (!rc) rc = rte_forward(L.ctx, &L.pr.src, &L.pr.stop, nullptr, tr.data(), hyp ? g1.data() : g0.data(), nullptr);
      if (rc) return die(L.ctx, "rte_forward", rc);
    }
    for (size_t q = 0; q < np; q++) snr[lz - initz] += (g1[q].re - g0[q].re) * (g1[q].re - g0[q].re) / g0[q].re;
    printf("%e is the SNR^2 for the lesion at z index %d \n", snr[lz - initz], lz);
  }
  dump("snr_terms.dat", snr.data(), snr.size());
  return 0;
}

int main_fisher(const char* path) {
  Loaded L;
  if (load(path, false, L, 0)) return 1;  // LoadPhantom(ini, 0): no tissue map (rte_fim.cu:104)
  const rte_config& c = L.pr.cfg;
  const size_t N = (size_t)c.nx * c.ny * c.nz;
  // the main sets mu_a = 0.01, mu_s = 1 for every tissue type before its solves (rte_fim.cu:226-230)
  std::vector<double> ta(L.pr.ntypes, 0.01), ts(L.pr.ntypes, 1.0);
  ta[0] = ts[0] = 0.0;
  int rc = rte_set_medium_tissue(L.ctx, L.pr.tiss, L.pr.ntypes, ta.data(), ts.data());
  if (rc) return die(L.ctx, "set medium", rc);
  // region: the voxels within rad_sig[0] = fov/(2 nX) of voxel (nX/2, nY/2, 1), on the main's own
  // coordinate arrays, which use the x extent for every axis (rte_fim.cu:135-206).  The reference
  // fills its z array only for indices below nX; with ReferenceQuirks (default) the others read as 0, as
  // in the reference's run (the region about z index 1 is the same either way).
  const double fov = c.x_max - c.x_min;
  auto X = [&](int i) { return i * fov / c.nx - fov / 2 + fov / (2 * c.nx); };
  auto Y = [&](int i) { return i * fov / c.ny - fov / 2 + fov / (2 * c.ny); };
  const int quirks = rte_par_get_int(L.par, "Algorithm:ReferenceQuirks", 1);
  auto Z = [&](int i) { return (quirks && i >= c.nx) ? 0.0 : i * fov / c.nz + fov / (2 * c.nz); };
  const float rad = (float)(1 * fov / (2 * c.nx));
  const float rad2 = rad * rad;  // a float product, compared against the double distance
  const int lx = c.nx / 2, ly = c.ny / 2, lz = 1;
  std::vector<uint8_t> mask(N);
  for (int i = 0; i < c.nz; i++)
    for (int j = 0; j < c.ny; j++)
      for (int k = 0; k < c.nx; k++) {
        const double d2 = (X(k) - X(lx)) * (X(k) - X(lx)) + (Y(j) - Y(ly)) * (Y(j) - Y(ly)) + (Z(i) - Z(lz)) * (Z(i) - Z(lz));
        mask[((size_t)i * c.ny + j) * c.nx + k] = !(d2 > (double)rad2);
      }
  double F = 0;
  for (int t = 1; t < L.pr.ntypes; t++) {  // the main repeats the same solve per tissue type
    rc = rte_fisher_regions(L.ctx, &L.pr.src, &L.pr.stop, 1, mask.data(), 1, &F);
    if (rc) return die(L.ctx, "rte_fisher_regions", rc);
  }
  printf("%e is fisher abs for %d as z index and %f as radius \n", F, lz, rad);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::string name = basename(argv[0]);
  if (argc != 2) {
    if (name == "rte_gpu") {
      printf("\n RTE_uniform file.ini\n");
      printf("     file.ini is the initialization.\n\n");
    } else {
      printf("\n InverseRTE file.par\n");
      printf("     file.par is the parameter file.\n\n");
    }
    return 1;
  }
  if (name == "rte_inv" || name == "rte_test") return main_inverse(argv[1]);
  if (name == "rte_fim") return main_fisher(argv[1]);
  if (name == "rte_snr") return main_snr(argv[1]);
  return main_forward(argv[1]);
}
