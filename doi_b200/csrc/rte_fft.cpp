// rte_fft.cpp -- the attenuation operator of a uniform medium as a convolution.
//
// In a uniform medium the pair kernel exp(-mu_t |d|) dV / (cm |d|^2) and the SH of the direction
// depend only on the displacement d = r - r', so the off-diagonal operator is a linear convolution
//   out_c[r] = sum_{d != 0} sum_c' T_cc'(d) W_c'[r - d],   T_cc'(d) = k(d) R_c(d/|d|) R_c'(d/|d|),
// over displacements inside the grid and the coupling distance (the CPU package builds the same
// shift-invariant table, CPU package/src/Kernels_selfsub.c:710-1084, and sums it directly).  Here
// it runs through FP64 FFTs on a grid zero-padded to at least 2n - 1 per axis: the spectra of the
// C(C+1)/2 distinct T_cc' are built once per medium; each application transforms the C input
// fields, forms the C x C spectral products (memory-bound on the table spectra, which are real or
// imaginary by the parity of T_cc' and stored as one real number each) and transforms back.
// cuFFT does the transforms; the sampling, padding, product and cropping kernels are in
// rte_kernels.cu.
#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <map>
#include <utility>

#include "rte_internal.h"

namespace {

int fft_size(int n) {  // >= 2n - 1, with prime factors 2, 3, 5, 7 only
  int m = 2 * n - 1;
  for (;; ++m) {
    int v = m;
    for (int f : {2, 3, 5, 7})
      while (v % f == 0) v /= f;
    if (v == 1) return m;
  }
}

cudaError_t cufft_err(cufftResult r) { return r == CUFFT_SUCCESS ? cudaSuccess : cudaErrorUnknown; }

}  // namespace

struct FftState {
  FftTabArgs a;
  int L = -1, table = 0;
  size_t M = 0, Mk = 0;
  int npair = 0;
  double* tau = nullptr;    // table spectra [npair][Mk]: one real number each, or complex (FIM table)
  double* F = nullptr;      // padded real fields [cap][M]
  double2* Fh = nullptr;    // their spectra [cap][Mk]
  double2* Oh = nullptr;    // product spectra [cap][Mk]
  int cap = 0;              // fields the buffers hold
  std::map<int, std::pair<cufftHandle, cufftHandle>> plans;  // fields -> (forward, inverse)
  bool valid = false;
  double mut = -1.0;
};

void rte_fft_destroy(FftState* s) {
  if (!s) return;
  for (auto& kv : s->plans) {
    cufftDestroy(kv.second.first);
    cufftDestroy(kv.second.second);
  }
  cudaFree(s->tau);
  cudaFree(s->F);
  cudaFree(s->Fh);
  cudaFree(s->Oh);
  delete s;
}

size_t rte_fft_bytes(int nx, int ny, int nz, int L, int nbmax) {
  const size_t Mx = fft_size(nx), My = fft_size(ny), Mz = fft_size(nz);
  const size_t M = Mx * My * Mz, Mk = Mz * My * (Mx / 2 + 1);
  const size_t C = (size_t)(L + 1) * (L + 1), npair = C * (C + 1) / 2;
  return npair * Mk * 16 + (size_t)nbmax * C * (M * 8 + 2 * Mk * 16);  // (a complex table at most)
}

// Table spectra for a uniform medium of attenuation mut (rebuilt when mut or the order changes).
cudaError_t rte_fft_prepare(FftState** ps, const FftTabArgs& args, int L, int table, int nbmax, cudaStream_t st) {
  FftState* s = *ps;
  if (!s) {
    s = new FftState;
    *ps = s;
  }
  FftTabArgs a = args;
  a.Mx = fft_size(a.nx);
  a.My = fft_size(a.ny);
  a.Mz = fft_size(a.nz);
  const size_t M = (size_t)a.Mx * a.My * a.Mz, Mk = (size_t)a.Mz * a.My * (a.Mx / 2 + 1);
  const int C = (L + 1) * (L + 1), npair = C * (C + 1) / 2;
  cudaError_t e = cudaSuccess;
  if (!s->tau || s->M != M || s->L != L || s->table != table) {
    cudaFree(s->tau);
    s->tau = nullptr;
    e = cudaMalloc(&s->tau, sizeof(double) * (table ? 2 : 1) * (size_t)npair * Mk);
    if (e != cudaSuccess) return e;
    s->valid = false;
  }
  if (s->cap < nbmax * C || s->M != M) {
    cudaFree(s->F);
    cudaFree(s->Fh);
    cudaFree(s->Oh);
    s->F = nullptr;
    s->Fh = s->Oh = nullptr;
    for (auto& kv : s->plans) {
      cufftDestroy(kv.second.first);
      cufftDestroy(kv.second.second);
    }
    s->plans.clear();
    s->cap = nbmax * C;
    if ((e = cudaMalloc(&s->F, sizeof(double) * (size_t)s->cap * M)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->Fh, sizeof(double2) * (size_t)s->cap * Mk)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->Oh, sizeof(double2) * (size_t)s->cap * Mk)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(s->F, 0, sizeof(double) * (size_t)s->cap * M, st)) != cudaSuccess) return e;
  }
  s->M = M;
  s->Mk = Mk;
  s->npair = npair;
  if (s->valid && s->mut == a.mut && s->L == L && s->table == table && s->a.prop_thresh == a.prop_thresh &&
      s->a.kscale == a.kscale)
    return cudaSuccess;
  s->a = a;
  s->L = L;
  s->table = table;
  s->mut = a.mut;
  // table fields in chunks that fit the padded-field buffer, each transformed in place into That
  const int chunk = s->cap;
  int dims[3] = {a.Mz, a.My, a.Mx};
  cufftHandle plan;
  if (cufftPlanMany(&plan, 3, dims, nullptr, 1, (int)M, nullptr, 1, (int)Mk, CUFFT_D2Z, chunk) != CUFFT_SUCCESS)
    return cudaErrorUnknown;
  cufftSetStream(plan, st);
  for (int p0 = 0; p0 < npair && e == cudaSuccess; p0 += chunk) {
    FftTabArgs b = a;
    b.p0 = p0;
    b.p1 = p0 + chunk < npair ? p0 + chunk : npair;
    if (b.p1 - b.p0 < chunk) e = cudaMemsetAsync(s->F, 0, sizeof(double) * (size_t)chunk * M, st);
    if (e == cudaSuccess) e = rte_launch_fft_table(b, L, table, s->F, M, st);
    if (e == cudaSuccess) e = cufft_err(cufftExecD2Z(plan, s->F, reinterpret_cast<cufftDoubleComplex*>(s->Fh)));
    if (e == cudaSuccess)
      e = table ? cudaMemcpyAsync(reinterpret_cast<double2*>(s->tau) + (size_t)p0 * Mk, s->Fh,
                                  sizeof(double2) * (size_t)(b.p1 - b.p0) * Mk, cudaMemcpyDeviceToDevice, st)
                : rte_launch_fft_extract(s->Fh, s->tau, p0, b.p1 - b.p0, C, Mk, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // before the plan goes
  cufftDestroy(plan);
  // the padded fields must start from zero outside the grid for the applications
  if (e == cudaSuccess) e = cudaMemsetAsync(s->F, 0, sizeof(double) * (size_t)s->cap * M, st);
  s->valid = e == cudaSuccess;
  return e;
}

static cudaError_t plans_for(FftState* s, int nf, std::pair<cufftHandle, cufftHandle>** out) {
  auto it = s->plans.find(nf);
  if (it == s->plans.end()) {
    int dims[3] = {s->a.Mz, s->a.My, s->a.Mx};
    cufftHandle f, i;
    if (cufftPlanMany(&f, 3, dims, nullptr, 1, (int)s->M, nullptr, 1, (int)s->Mk, CUFFT_D2Z, nf) != CUFFT_SUCCESS)
      return cudaErrorUnknown;
    if (cufftPlanMany(&i, 3, dims, nullptr, 1, (int)s->Mk, nullptr, 1, (int)s->M, CUFFT_Z2D, nf) != CUFFT_SUCCESS) {
      cufftDestroy(f);
      return cudaErrorUnknown;
    }
    it = s->plans.emplace(nf, std::make_pair(f, i)).first;
  }
  *out = &it->second;
  return cudaSuccess;
}

// Plans for nf transformed fields made ahead of a stream capture (planning allocates).
cudaError_t rte_fft_warm(FftState* s, int nf) {
  if (!s || !s->valid || nf > s->cap) return cudaErrorInvalidValue;
  std::pair<cufftHandle, cufftHandle>* pl;
  return plans_for(s, nf, &pl);
}

// Every device address the transforms and kernels of an application use (a recorded graph holds them).
uintptr_t rte_fft_signature(const FftState* s) {
  if (!s) return 0;
  return (uintptr_t)s->tau ^ ((uintptr_t)s->F << 1) ^ ((uintptr_t)s->Fh << 2) ^ ((uintptr_t)s->Oh << 3) ^ s->M;
}

// out (split-K partial layout, one split) = off-diagonal operator applied to W [N][vstride], nb
// right-hand sides, coefficients below Cact.
cudaError_t rte_fft_apply(FftState* s, const double* W, int vstride, int Cfull, int LA, int nb, double* part,
                          cudaStream_t st) {
  if (!s || !s->valid) return cudaErrorInvalidValue;
  const int Cact = (LA + 1) * (LA + 1);
  const int nf = nb * Cact;
  if (nf > s->cap) return cudaErrorInvalidValue;
  std::pair<cufftHandle, cufftHandle>* pl = nullptr;
  cudaError_t e0 = plans_for(s, nf, &pl);
  if (e0 != cudaSuccess) return e0;
  cufftSetStream(pl->first, st);
  cufftSetStream(pl->second, st);
  cudaError_t e = rte_launch_fft_pad(W, vstride, Cfull, Cact, nb, s->a, s->F, s->M, st);
  if (e == cudaSuccess) e = cufft_err(cufftExecD2Z(pl->first, s->F, reinterpret_cast<cufftDoubleComplex*>(s->Fh)));
  if (e != cudaSuccess) return e;
  e = rte_launch_fft_product(s->tau, s->Fh, s->Oh, (s->L + 1) * (s->L + 1), Cact, nb, s->Mk, s->table, st);
  if (e != cudaSuccess) return e;
  // the inverse overwrites the padded buffer; the crop below reads only the grid, and the padding
  // is restored to zero for the next application
  e = cufft_err(cufftExecZ2D(pl->second, reinterpret_cast<cufftDoubleComplex*>(s->Oh), s->F));
  if (e != cudaSuccess) return e;
  e = rte_launch_fft_crop(s->F, Cfull, Cact, nb, s->a, part, s->M, st);
  if (e != cudaSuccess) return e;
  return cudaMemsetAsync(s->F, 0, sizeof(double) * (size_t)nf * s->M, st);
}
