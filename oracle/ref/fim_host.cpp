// fim_host.cpp -- runs the reference FisherInfo_IO forward path on the CPU.
//
// TEST INFRASTRUCTURE ONLY (the oracle's pin).  The reference's own sources
// (kernels.cu lines 1-418 -- the device functions and kernels, no host launch
// code --, dist.cu, sph_harm.cu, inits.cu, neumann.cu, rte.cu with main renamed,
// iniparser.cu, dictionary.cu) are compiled as host C++ under fim_emu.h by
// oracle/build.sh, straight from where they lie in the reference tree.  This file
// replaces only the one function that needs a GPU: prop_abs()
// (FisherInfo_IO/src/kernels.cu:704-811), re-enacted here launch by launch: the
// same grid (nX/10, nY/10), blocks of 10x10x5, the same four kernels in the same
// order, each kernel body run once per emulated CUDA thread.
//
// usage:
//   fim_host forward <file.par> <out_prefix>
//       writes <prefix>_src.bin (xi), <prefix>_out.bin (final distribution),
//       <prefix>_trans.bin, <prefix>_ref.bin (complex images), <prefix>_meta.txt
//   fim_host apply <file.par> <in.bin> <flag> <flag_scat> <out.bin>
//       one prop_abs pass over all slabs (flag = all-L, flag_scat = scatter)
//   fim_host diag <file.par> <out.bin>
//       the self-voxel table diag_terms_host (MAX_TISS_NUM*MAX_NL^4 complex, dist.cu:362-533)
//   fim_host program <file.par>
//       the reference main linked into this binary (rte.cu in fim_host, rte_fim.cu in fim_fisher,
//       rte_snr.cu in fim_snr, compute_grad_rte.cu in fim_grad; oracle/build.sh renames each main
//       to fim_prog_main), run as
//       `<main> file.par`, so it reads the file and writes its outputs as the program does
//   fim_host downsample <file.par> <in.bin> <ds> <out.bin>
//       downsample_image (dist.cu:271-289) of an nX*nY complex image; writes the (nX/ds)*(nY/ds)
//       values its loops assign.  The function sums into a fresh malloc block without clearing it,
//       so the allocator is told to hand out zero-filled blocks (M_PERTURB 0xff fills each block
//       with 0xff ^ 0xff; run with GLIBC_TUNABLES=glibc.malloc.tcache_count=0 so that no block
//       bypasses the fill), which makes its result the zero-started sum.
#include <malloc.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "rte.h"

thread_local emu_dim3 threadIdx, blockIdx;

// CUDA fast-math intrinsics named by complex_arith.cu's cexp_dev (never called on this path)
extern "C" float __powf(float a, float b) { return powf(a, b); }
extern "C" float __cosf(float a) { return cosf(a); }
extern "C" float __sinf(float a) { return sinf(a); }

// reference globals (rte.cu:14-21) and device constants (kernels.cu:20-22)
extern Geometry* geom;
extern Phantom* phan;
extern Source* beam_src;
extern complex_double* diag_terms_host;
extern complex_double* sph_harm;
extern Info_Stat* info_stat_host;
extern SHORT nL;
extern int nTerms;
extern Info_Stat info_stat;
extern SHORT nL_dev;
extern complex_double diag_terms_dev[MAX_TISS_NUM * MAX_NL * MAX_NL * MAX_NL * MAX_NL];
Info_Stat* populate_info_dev();

// kernels compiled from kernels.cu
void compute_diagonal_abs(doublecomplex* src_dist, doublecomplex* out_dist, Info_Dyn info_dyn, int cnt,
                          SHORT block_dep, SHORT layer_start, SHORT flag);
void compute_propabs(complex_double* src_dist_dev, complex_double* out_dist_dev, Info_Dyn info_dyn,
                     complex_double* sph_harm_dev, SHORT cnt, SHORT blk_dep, SHORT start_layer, SHORT flag);
void scale_dist_dev(doublecomplex* W, double scale_fac, SHORT cnt, SHORT block_dep);
void prop_scat_dev(doublecomplex* out_dist, Info_Dyn info_dyn, short layer_start, SHORT block_dep, SHORT flag);

static std::mutex g_launch_mu;
static int g_prop_abs_calls = 0;

template <class F>
static void launch(int gx, int gy, F body) {
  const int bx = BLK_SIZE, by = BLK_SIZE, bz = BLK_SIZE_Z;
  const int nthr = gx * gy * bx * by * bz;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < nthr; t++) {
    int k = t % bx, j = (t / bx) % by, i = (t / (bx * by)) % bz, b = t / (bx * by * bz);
    blockIdx.x = b % gx;
    blockIdx.y = b / gx;
    blockIdx.z = 0;
    threadIdx.x = k;
    threadIdx.y = j;
    threadIdx.z = i;
    body();
  }
}

// Host re-enactment of prop_abs (kernels.cu:704-811).
void* prop_abs(void* arg) {
  std::lock_guard<std::mutex> lk(g_launch_mu);
  g_prop_abs_calls++;
  const THREAD_PARAMETERS parameters = *((THREAD_PARAMETERS*)arg);
  int size_layer = (geom->nX + 2 * geom->bounX) * (geom->nY + 2 * geom->bounY) * (nL + 1) * (nL + 1);
  int size = size_layer * (geom->nZ + 2 * geom->bounZ);
  if (geom->nX % BLK_SIZE || geom->nY % BLK_SIZE || parameters.num_layers % BLK_SIZE_Z) {
    fprintf(stderr, "fim_host: grid not supported by the reference launch shape\n");
    exit(3);
  }
  std::vector<complex_double> src(size), out((size_t)size_layer * parameters.num_layers);
  memcpy(src.data(), parameters.src_host, sizeof(complex_double) * size);
  memset(out.data(), 0, sizeof(complex_double) * out.size());
  Info_Dyn info_dyn;
  info_dyn.tiss_type = phan->tiss_type;
  info_stat = *info_stat_host;  // cudaMemcpyToSymbol(info_stat, ...)
  nL_dev = nL;
  memcpy(diag_terms_dev, diag_terms_host,
         sizeof(complex_double) * MAX_TISS_NUM * MAX_NL * MAX_NL * MAX_NL * MAX_NL);
  int gx = geom->nX / BLK_SIZE, gy = geom->nY / BLK_SIZE;
  SHORT cnt = 0;
  for (SHORT bd = 0; bd < parameters.num_layers; bd = bd + BLK_SIZE_Z)
    launch(gx, gy, [&] {
      compute_diagonal_abs(src.data(), out.data(), info_dyn, cnt, bd, parameters.layer_start, parameters.flag);
    });
  for (SHORT bd = 0; bd < parameters.num_layers; bd = bd + BLK_SIZE_Z)
    launch(gx, gy, [&] {
      compute_propabs(src.data(), out.data(), info_dyn, sph_harm, cnt, bd, parameters.layer_start,
                      parameters.flag);
    });
  for (SHORT bd = 0; bd < parameters.num_layers; bd = bd + BLK_SIZE_Z)
    launch(gx, gy, [&] { scale_dist_dev(out.data(), geom->delX * geom->delY * geom->delZ, cnt, bd); });
  if (parameters.flag_scat)
    for (SHORT bd = 0; bd < parameters.num_layers; bd = bd + BLK_SIZE_Z)
      launch(gx, gy, [&] { prop_scat_dev(out.data(), info_dyn, parameters.layer_start, bd, parameters.flag); });
  memcpy(parameters.out_host, out.data(), sizeof(complex_double) * out.size());
  return NULL;
}

static void write_dist(const char* name, const complex_double* d, size_t n) {
  FILE* f = fopen(name, "wb");
  fwrite(d, sizeof(complex_double), n, f);
  fclose(f);
}

// the reference's setup sequence, rte.cu:110-166
static void setup(const char* par) {
  dictionary* ini = iniparser_load((char*)par);
  geom = LoadGeometry(ini);
  phan = LoadPhantom(ini, 1);
  beam_src = LoadSource(ini);
  if (((phan->mut_mean).real() * (geom->z_max - geom->z_min)) > 4)
    geom->prop_thresh = -log(THRESH_PROP) / (phan->mut_mean.real());
  nL = iniparser_getint(ini, (char*)"Algorithm:nL", 1000);
  nTerms = iniparser_getint(ini, (char*)"Algorithm:nTerms", 1);
  info_stat_host = populate_info_dev();
  generate_sph_harm_terms();
  generate_diag_terms_host();
}

int fim_prog_main(int argc, char** argv);

int main(int argc, char** argv) {
  if (argc >= 3 && !strcmp(argv[1], "program")) return fim_prog_main(argc - 1, argv + 1);
  if (argc < 4) {
    fprintf(stderr, "usage: fim_host forward <par> <prefix> | apply <par> <in> <flag> <flag_scat> <out>\n");
    return 1;
  }
  setup(argv[2]);
  size_t ndist = (size_t)geom->no_vox * (nL + 1) * (nL + 1);
  if (!strcmp(argv[1], "forward")) {
    complex_double* src = alloc_dist();
    complex_double* out = alloc_dist();
    complex_double* W = alloc_dist();
    generate_source_beam(src);
    copy_dist(src, out);
    copy_dist(src, W);
    Neumann(W, out, 1);
    complex_double* trans = generate_trans_image(out, 1);
    complex_double* ref = generate_ref_image(out);
    char name[4096];
    snprintf(name, sizeof name, "%s_src.bin", argv[3]);
    write_dist(name, src, ndist);
    snprintf(name, sizeof name, "%s_out.bin", argv[3]);
    write_dist(name, out, ndist);
    snprintf(name, sizeof name, "%s_trans.bin", argv[3]);
    write_dist(name, trans, (size_t)geom->nX * geom->nY);
    snprintf(name, sizeof name, "%s_ref.bin", argv[3]);
    write_dist(name, ref, (size_t)geom->nX * geom->nY);
    snprintf(name, sizeof name, "%s_meta.txt", argv[3]);
    FILE* f = fopen(name, "w");
    // prop_abs runs once per device per term, plus once per device for the final A
    fprintf(f, "terms %d\nprop_thresh %.17g\ncm %.17g\ndelX %.17g\ndelY %.17g\ndelZ %.17g\n",
            g_prop_abs_calls / NUM_DEVICES - 1, (double)geom->prop_thresh, (double)info_stat_host->cm,
            geom->delX, geom->delY, geom->delZ);
    fclose(f);
    return 0;
  }
  if (!strcmp(argv[1], "diag")) {
    write_dist(argv[3], diag_terms_host, (size_t)MAX_TISS_NUM * MAX_NL * MAX_NL * MAX_NL * MAX_NL);
    return 0;
  }
  if (!strcmp(argv[1], "apply") && argc >= 7) {
    std::vector<complex_double> in(ndist), res(ndist);
    FILE* f = fopen(argv[3], "rb");
    if (!f || fread(in.data(), sizeof(complex_double), ndist, f) != ndist) {
      fprintf(stderr, "fim_host: cannot read %s\n", argv[3]);
      return 2;
    }
    fclose(f);
    int flag = atoi(argv[4]), flag_scat = atoi(argv[5]);
    // the per-device slab split of neumann.cu:38-51 and :65-82
    int per = geom->nZ / NUM_DEVICES, rem = geom->nZ % NUM_DEVICES, start = 0;
    int size_layer = geom->nX * geom->nY * (nL + 1) * (nL + 1);
    for (int d = 0; d < NUM_DEVICES; d++) {
      THREAD_PARAMETERS tp;
      tp.device_index = d;
      tp.src_host = in.data();
      tp.num_layers = per + (rem > d ? 1 : 0);
      tp.layer_start = start;
      tp.out_host = res.data() + (size_t)start * size_layer;
      tp.flag = flag;
      tp.flag_scat = flag_scat;
      prop_abs(&tp);
      start += tp.num_layers;
    }
    write_dist(argv[6], res.data(), ndist);
    return 0;
  }
  if (!strcmp(argv[1], "downsample") && argc >= 6) {
    const size_t np = (size_t)geom->nX * geom->nY;
    std::vector<complex_double> img(np);
    FILE* f = fopen(argv[3], "rb");
    if (!f || fread(img.data(), sizeof(complex_double), np, f) != np) {
      fprintf(stderr, "fim_host: cannot read %s\n", argv[3]);
      return 2;
    }
    fclose(f);
    const int ds = atoi(argv[4]);
    if (ds < 1 || ds > geom->nX || ds > geom->nY) return 2;
    mallopt(M_PERTURB, 0xff);
    complex_double* res = downsample_image(img.data(), ds);
    write_dist(argv[5], res, (size_t)(geom->nX / ds) * (geom->nY / ds));
    return 0;
  }
  fprintf(stderr, "fim_host: unknown command %s\n", argv[1]);
  return 1;
}
