// rte_par.cpp -- the reference's parameter-file interface and image files, for drop-in use.
//
// Parameter files follow the iniparser dialect the reference links (FisherInfo_IO/src/iniparser.cu
// :455-620): lines are stripped; '#' starts a comment line; "[name]" opens a section; "key = value"
// with the value optionally in double or single quotes, an unquoted value ending at ';' or '#';
// "key =" gives an empty value; a trailing backslash joins the next line; keys and sections are
// case-insensitive and looked up as "section:key"; a repeated key keeps its last value; integers
// convert like strtol(s, NULL, 0) and doubles like atof (iniparser.cu:268-337).  Malformed lines
// are reported and skipped, as the reference does.
//
// rte_par_problem derives the solver inputs the way the reference mains do: LoadGeometry /
// LoadPhantom / LoadSource (FisherInfo_IO/src/inits.cu:22-269) for tissue-map files, the CPU
// package's loaders (CPU package/src/Inits.c:24-131, RTE_uniform.c:51-66) for uniform media, plus
// optional keys for what this library adds (per-voxel media, face and point sources, precision,
// stop rule, detector bins).  No device work happens here.
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/rte_b200.h"

struct rte_par {
  std::map<std::string, std::string> kv;
  std::string path;
};

namespace {

std::string lower(std::string s) {
  for (char& ch : s) ch = (char)tolower((unsigned char)ch);
  return s;
}

std::string strip(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && isspace((unsigned char)s[a])) a++;
  while (b > a && isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

// One logical line -> (kind, key, value): 0 empty/comment, 1 section, 2 key/value, -1 error.
int parse_line(const std::string& raw, std::string& section, std::string& key, std::string& val) {
  const std::string line = strip(raw);
  if (line.empty() || line[0] == '#') return 0;
  if (line[0] == '[' && line.back() == ']') {
    section = lower(strip(line.substr(1, line.find(']') - 1)));
    return 1;
  }
  const size_t eq = line.find('=');
  if (eq == std::string::npos || eq == 0) return -1;
  key = lower(strip(line.substr(0, eq)));
  std::string rest = strip(line.substr(eq + 1));
  if (!rest.empty() && (rest[0] == '"' || rest[0] == '\'')) {
    const size_t close = rest.find(rest[0], 1);
    if (close != std::string::npos) {
      val = rest.substr(1, close - 1);
      return 2;
    }
  }
  const size_t cut = rest.find_first_of(";#");
  val = strip(cut == std::string::npos ? rest : rest.substr(0, cut));
  if (val == "\"\"" || val == "''") val.clear();
  return 2;
}

bool read_file(const char* path, std::vector<unsigned char>& buf, size_t n) {
  FILE* f = fopen(path, "rb");
  if (!f) return false;
  buf.resize(n);
  const size_t got = n ? fread(buf.data(), 1, n, f) : 0;
  fclose(f);
  return got == n;
}

void copy_str(char* dst, size_t cap, const char* src) {
  if (!src) {
    dst[0] = 0;
    return;
  }
  snprintf(dst, cap, "%s", src);
}

}  // namespace

extern "C" {

int rte_par_load(const char* path, rte_par** out) {
  if (!path || !out) return RTE_ERR_ARG;
  *out = nullptr;
  FILE* f = fopen(path, "r");
  if (!f) return RTE_ERR_IO;
  rte_par* p = new rte_par;
  p->path = path;
  std::string section, key, val, acc;
  char buf[4096];
  int lineno = 0;
  while (fgets(buf, sizeof buf, f)) {
    lineno++;
    std::string line(buf);
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r' || isspace((unsigned char)line.back())))
      line.pop_back();
    if (!line.empty() && line.back() == '\\') {  // continued on the next line
      line.pop_back();
      acc += line;
      continue;
    }
    acc += line;
    const int kind = parse_line(acc, section, key, val);
    if (kind == 2) p->kv[section + ":" + key] = val;
    if (kind == -1) fprintf(stderr, "par: syntax error in %s (%d): %s\n", path, lineno, acc.c_str());
    acc.clear();
  }
  fclose(f);
  *out = p;
  return RTE_OK;
}

void rte_par_free(rte_par* p) { delete p; }

const char* rte_par_get_string(const rte_par* p, const char* key, const char* def) {
  if (!p || !key) return def;
  auto it = p->kv.find(lower(key));
  return it == p->kv.end() ? def : it->second.c_str();
}

int rte_par_get_int(const rte_par* p, const char* key, int def) {
  const char* s = rte_par_get_string(p, key, nullptr);
  return s ? (int)strtol(s, nullptr, 0) : def;
}

double rte_par_get_double(const rte_par* p, const char* key, double def) {
  const char* s = rte_par_get_string(p, key, nullptr);
  return s ? atof(s) : def;
}

int rte_par_problem(const rte_par* p, int read_map, rte_problem* pr) {
  if (!p || !pr) return RTE_ERR_ARG;
  memset(pr, 0, sizeof *pr);
  rte_config& c = pr->cfg;
  const bool cpu_style = !rte_par_get_string(p, "Phantom:TissMapFile", nullptr) &&
                         rte_par_get_string(p, "Phantom:mua", nullptr) != nullptr;
  pr->style = cpu_style ? 1 : 0;
  // [Geometry]: the reference keeps the extents and thresholds as float (rte.h:61-70)
  c.nx = rte_par_get_int(p, "Geometry:nX", -1);
  c.ny = rte_par_get_int(p, "Geometry:nY", -1);
  c.nz = rte_par_get_int(p, "Geometry:nZ", -1);
  if (c.nx < 1 || c.ny < 1 || c.nz < 1) return RTE_ERR_ARG;
  auto ext = [&](const char* lo, const char* hi, double& a, double& b) {
    const double vlo = rte_par_get_double(p, lo, -1.0), vhi = rte_par_get_double(p, hi, -1.0);
    if (cpu_style) {
      a = vlo;
      b = vhi;
    } else {  // float extents; the width is a float difference (inits.cu:217-219)
      a = (double)(float)vlo;
      b = a + (double)((float)vhi - (float)vlo);
    }
  };
  ext("Geometry:xMin", "Geometry:xMax", c.x_min, c.x_max);
  ext("Geometry:yMin", "Geometry:yMax", c.y_min, c.y_max);
  ext("Geometry:zMin", "Geometry:zMax", c.z_min, c.z_max);
  const double prop = rte_par_get_double(p, "Geometry:propThresh", 0.0);
  c.prop_thresh = cpu_style ? prop : (double)(float)prop;
  c.self_sub_vox = cpu_style ? 1 : (int)rte_par_get_double(p, "Geometry:selfsubVox", 1.0);
  c.nL = rte_par_get_int(p, "Algorithm:nL", -1);
  if (c.nL < 0) return RTE_ERR_ARG;
  c.g = rte_par_get_double(p, "Phantom:g", -1.0);
  c.n = rte_par_get_double(p, "Phantom:n", -1.0);
  c.c = cpu_style ? rte_par_get_double(p, "Phantom:c", 2.9979e10) : 1.0;  // rte.h:15 (#define C 1)
  // optional keys of this library
  const std::string model = lower(rte_par_get_string(p, "Algorithm:Model", cpu_style ? "cpu" : "fim"));
  c.model = model == "exact" ? RTE_MODEL_EXACT : (model == "cpu" ? RTE_MODEL_CPU : RTE_MODEL_FIM);
  const std::string prec = lower(rte_par_get_string(p, "Algorithm:Precision", "fp64"));
  c.precision = prec == "mixed" ? RTE_PREC_MIXED : RTE_PREC_FP64;
  const std::string km = lower(rte_par_get_string(p, "Algorithm:KernelMode", "auto"));
  c.kernel_mode = km == "store" ? RTE_KERNEL_STORE : (km == "recompute" ? RTE_KERNEL_RECOMPUTE : RTE_KERNEL_AUTO);
  c.device = rte_par_get_int(p, "Algorithm:Device", 0);
  pr->nterms = rte_par_get_int(p, "Algorithm:nTerms", 1);
  const std::string rule = lower(rte_par_get_string(p, "Algorithm:StopRule", "reference"));
  pr->stop.rule = rule == "fixed" ? RTE_STOP_FIXED : (rule == "rel_l2" ? RTE_STOP_REL_L2 : RTE_STOP_REFERENCE);
  pr->stop.max_terms = rte_par_get_int(p, "Algorithm:MaxTerms", pr->stop.rule == RTE_STOP_FIXED ? pr->nterms : 30);
  pr->stop.tol = rte_par_get_double(p, "Algorithm:Tol", 1e-7);
  pr->detector_bins = rte_par_get_int(p, "Algorithm:DetectorBins", 0);
  // [Source]
  rte_source& s = pr->src;
  s.pos_x = rte_par_get_double(p, "Source:posX", 0.0);
  s.pos_y = rte_par_get_double(p, "Source:posY", 0.0);
  s.pos_z = rte_par_get_double(p, "Source:posZ", 0.0);
  s.diam = rte_par_get_double(p, "Source:diam", 0.2);
  s.theta = rte_par_get_double(p, "Source:theta", 0.0);
  s.phi = rte_par_get_double(p, "Source:phi", 0.0);
  s.mag = rte_par_get_double(p, "Source:magnitude", 1.0);
  s.modulation = rte_par_get_double(p, "Source:modulation", 0.0);
  const std::string kind = lower(rte_par_get_string(p, "Source:Kind", cpu_style ? "cpu" : "fim"));
  s.kind = kind == "column" ? RTE_SRC_COLUMN
         : kind == "cpu"    ? RTE_SRC_CPU
         : kind == "beam"   ? RTE_SRC_BEAM
         : kind == "point"  ? RTE_SRC_POINT
                            : RTE_SRC_FIM;
  s.face = rte_par_get_int(p, "Source:Face", 0);
  // [Runtime]
  copy_str(pr->trans_file, sizeof pr->trans_file, rte_par_get_string(p, "Runtime:TransFile", nullptr));
  copy_str(pr->ref_file, sizeof pr->ref_file, rte_par_get_string(p, "Runtime:ReflectFile", nullptr));
  copy_str(pr->phase_file, sizeof pr->phase_file, rte_par_get_string(p, "Runtime:PhaseFile", nullptr));
  copy_str(pr->g_file, sizeof pr->g_file, rte_par_get_string(p, "Runtime:gFile", nullptr));
  copy_str(pr->flux_file, sizeof pr->flux_file, rte_par_get_string(p, "Runtime:FluxFile", nullptr));
  pr->num_iterations = rte_par_get_int(p, "Runtime:numIterations", 1);
  pr->step_a = rte_par_get_double(p, "Runtime:stepsizea", 1e3);
  pr->step_s = rte_par_get_double(p, "Runtime:stepsizes", 1e3);
  // [Phantom] medium
  const size_t N = (size_t)c.nx * c.ny * c.nz;
  double mut_sum = 0.0;
  if (cpu_style) {
    pr->ntypes = 2;
    pr->mua[1] = rte_par_get_double(p, "Phantom:mua", -1.0);
    pr->mus[1] = rte_par_get_double(p, "Phantom:mus", -1.0);
    pr->tiss = (uint8_t*)malloc(N);
    if (!pr->tiss) return RTE_ERR_NOMEM;
    memset(pr->tiss, 1, N);
    mut_sum = (pr->mua[1] + pr->mus[1]) * (double)N;
  } else {
    const int notiss = rte_par_get_int(p, "Phantom:NoTiss", 1);
    if (notiss < 1 || notiss + 1 > RTE_PAR_MAX_TISS) return RTE_ERR_UNSUPPORTED;
    pr->ntypes = notiss + 1;  // + type 0, outside the object (inits.cu:44)
    for (int t = 1; t < pr->ntypes; t++) {
      char ka[64], ks[64];
      snprintf(ka, sizeof ka, "Phantom:TissAbs%d", t);
      snprintf(ks, sizeof ks, "Phantom:TissSc%d", t);
      pr->mua[t] = rte_par_get_double(p, ka, 0.01);
      pr->mus[t] = rte_par_get_double(p, ks, 1.0);
    }
    pr->tiss = (uint8_t*)malloc(N);
    if (!pr->tiss) return RTE_ERR_NOMEM;
    if (read_map) {
      const char* map = rte_par_get_string(p, "Phantom:TissMapFile", nullptr);
      std::vector<unsigned char> buf;
      if (!map || !read_file(map, buf, N)) {
        rte_problem_free(pr);
        return RTE_ERR_IO;
      }
      memcpy(pr->tiss, buf.data(), N);
    } else {
      memset(pr->tiss, 1, N);  // LoadPhantom(ini, 0): every voxel tissue 1 (inits.cu:112-128)
    }
    for (size_t r = 0; r < N; r++) {
      if (pr->tiss[r] >= pr->ntypes) {
        rte_problem_free(pr);
        return RTE_ERR_ARG;
      }
      mut_sum += pr->mua[pr->tiss[r]] + pr->mus[pr->tiss[r]];
    }
  }
  pr->mut_mean = mut_sum / (double)N;
  // per-voxel media (new): N doubles each, z-major, x fastest
  const char* fa = rte_par_get_string(p, "Phantom:MuaFile", nullptr);
  const char* fs = rte_par_get_string(p, "Phantom:MusFile", nullptr);
  if (fa && fs) {
    std::vector<unsigned char> ba, bs;
    if (!read_file(fa, ba, N * sizeof(double)) || !read_file(fs, bs, N * sizeof(double))) {
      rte_problem_free(pr);
      return RTE_ERR_IO;
    }
    pr->mua_vox = (double*)malloc(N * sizeof(double));
    pr->mus_vox = (double*)malloc(N * sizeof(double));
    if (!pr->mua_vox || !pr->mus_vox) {
      rte_problem_free(pr);
      return RTE_ERR_NOMEM;
    }
    memcpy(pr->mua_vox, ba.data(), N * sizeof(double));
    memcpy(pr->mus_vox, bs.data(), N * sizeof(double));
    mut_sum = 0.0;
    for (size_t r = 0; r < N; r++) mut_sum += pr->mua_vox[r] + pr->mus_vox[r];
    pr->mut_mean = mut_sum / (double)N;
  }
  // the forward main's diffuse-medium threshold (FisherInfo_IO/src/rte.cu:116-119), float as stored
  pr->diffuse_prop_thresh = pr->mut_mean * (c.z_max - c.z_min) > 4.0
                                ? (double)(float)(-log(0.01) / pr->mut_mean)
                                : c.prop_thresh;
  return RTE_OK;
}

void rte_problem_free(rte_problem* pr) {
  if (!pr) return;
  free(pr->tiss);
  free(pr->mua_vox);
  free(pr->mus_vox);
  pr->tiss = nullptr;
  pr->mua_vox = pr->mus_vox = nullptr;
}

int rte_write_image(const char* path, int nx, int ny, const rte_cplx* img, int cpu_layout) {
  if (!path || !img || nx < 1 || ny < 1) return RTE_ERR_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return RTE_ERR_IO;
  // FisherInfo_IO/src/dist.cu:316-345 writes (nY, nX); CPU package/src/Dist.c:16-40 (nX, nY)
  const int hdr[2] = {cpu_layout ? nx : ny, cpu_layout ? ny : nx};
  bool ok = fwrite(hdr, sizeof(int), 2, f) == 2;
  const size_t np = (size_t)nx * ny;
  std::vector<double> plane(np);
  for (int part = 0; part < 2 && ok; part++) {
    for (size_t q = 0; q < np; q++) plane[q] = part ? img[q].im : img[q].re;
    ok = fwrite(plane.data(), sizeof(double), np, f) == np;
  }
  ok = fclose(f) == 0 && ok;
  return ok ? RTE_OK : RTE_ERR_IO;
}

int rte_write_phase_image(const char* path, int nx, int ny, const double* phase, int cpu_layout) {
  if (!path || !phase || nx < 1 || ny < 1) return RTE_ERR_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return RTE_ERR_IO;
  int hdr[2] = {ny, nx};  // dist.cu:291-314
  if (cpu_layout) {       // Dist.c:54-55
    hdr[0] = nx;
    hdr[1] = ny;
  }
  const size_t np = (size_t)nx * ny;
  bool ok = fwrite(hdr, sizeof(int), 2, f) == 2 && fwrite(phase, sizeof(double), np, f) == np;
  ok = fclose(f) == 0 && ok;
  return ok ? RTE_OK : RTE_ERR_IO;
}

int rte_read_image(const char* path, int nx, int ny, double* out) {
  if (!path || !out || nx < 1 || ny < 1) return RTE_ERR_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return RTE_ERR_IO;
  int hdr[2];
  const size_t np = (size_t)nx * ny;
  // two ints, then nX*nY doubles (compute_grad_rte.cu:151-161 reads exactly that much)
  const bool ok = fread(hdr, sizeof(int), 2, f) == 2 && fread(out, sizeof(double), np, f) == np;
  fclose(f);
  return ok ? RTE_OK : RTE_ERR_IO;
}

// FisherInfo_IO/src/dist.cu:271-289 (downsample_image): sums of ds x ds pixel blocks.  The index
// arithmetic is the reference's: output (i, j), i < nX/ds, j < nY/ds, is out[i*(nY/ds) + j] and adds
// img[(i*ds + a)*nY + j*ds + b] for a, b < ds; on the square images the callers pass this is the block
// sum of the y*nX + x image layout.  The reference accumulates into an uninitialised malloc block; the
// sums here start at zero.  Rows and columns beyond the last whole block are dropped, as there.
int rte_downsample_image(const rte_cplx* img, int nx, int ny, int ds, rte_cplx* out) {
  if (!img || !out || nx < 1 || ny < 1 || ds < 1 || ds > nx || ds > ny) return RTE_ERR_ARG;
  const int mx = nx / ds, my = ny / ds;
  for (int i = 0; i < mx; i++)
    for (int j = 0; j < my; j++) {
      double re = 0.0, im = 0.0;
      for (int a = 0; a < ds; a++)
        for (int b = 0; b < ds; b++) {
          const rte_cplx& v = img[(size_t)(i * ds + a) * ny + (size_t)j * ds + b];
          re += v.re;
          im += v.im;
        }
      out[(size_t)i * my + j] = rte_cplx{re, im};
    }
  return RTE_OK;
}

}  // extern "C"
