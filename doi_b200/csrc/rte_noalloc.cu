// rte_noalloc.cu -- one entry point of the library that never allocates device memory.
//
// Who needs it: callers that are not allowed to call cudaMalloc at the point where they run the
// solver.  Examples: code recorded into a CUDA graph (allocation is illegal during stream capture),
// plug-ins living inside a host application that owns every byte of device memory through its own
// pool, and real-time loops that must not block on the allocator.  rte_create() allocates the
// context's buffers, so such callers cannot use the context API at that point.
//
// What it computes: one application of the off-diagonal attenuation operator of the reference
// (the compute_propabs + scale_dist_dev part of prop_abs, FisherInfo_IO/src/kernels.cu:289-383),
// i.e. the exact FP64 pair sum without the self-voxel term and without scatter, on caller-owned
// device buffers in the reference's complex coefficient layout.
//
// Where its scratch lives: a file-scope __device__ array of RTE_NOALLOC_SCRATCH_BYTES (64 MiB),
// part of the module image, so every GPU that loads this library holds it until the process
// exits.  Host code cannot use the array's name as a device address; the first call on each
// device looks the address up with cudaGetSymbolAddress (and uploads the spherical-harmonic
// recurrence tables), with that device current.  That first call should therefore be made before
// any stream capture.  All calls share the one array and it keeps the previous call's contents;
// everything that must start at zero is cleared by each call, and two calls whose GPU work overlaps
// (different streams, or host threads) race on it.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "../../include/rte_b200.h"
#include "rte_internal.h"

#define RTE_NOALLOC_SCRATCH_BYTES (64ull << 20)
#define RTE_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double g_noalloc_scratch[RTE_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {
std::mutex g_mu;
double* g_addr[RTE_NOALLOC_MAX_DEVICES];

int set_err(int code, const char* msg) {
  rte_set_global_error(msg);  // reported by rte_last_error(NULL)
  return code;
}

// once per device, with that device current: the scratch array's device address and the SH tables
int setup(int dev, double** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= RTE_NOALLOC_MAX_DEVICES) return set_err(RTE_ERR_ARG, "device ordinal out of range");
  if (!g_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_err(RTE_ERR_DEVICE, cudaGetErrorString(e));
    e = rte_upload_sh_tables(make_sh_tables());  // the context path's tables (rte_host.cpp)
    if (e != cudaSuccess) return set_err(RTE_ERR_DEVICE, cudaGetErrorString(e));
    g_addr[dev] = (double*)p;
  }
  *out = g_addr[dev];
  return RTE_OK;
}

__global__ void k_identity(int* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}
}  // namespace

extern "C" int rte_attenuate_noalloc(int nx, int ny, int nz, double dx, double dy, double dz, int nL,
                                     double prop_thresh, double cm, const double* d_mut, const rte_cplx* d_in,
                                     rte_cplx* d_out, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || nL < 0 || nL > RTE_MAX_L || !(dx > 0) || !(dy > 0) || !(dz > 0) ||
      !(cm > 0) || !d_mut || !d_in || !d_out)
    return set_err(RTE_ERR_ARG, "rte_attenuate_noalloc: bad argument");
  const long long N = (long long)nx * ny * nz;
  const long long C = (long long)(nL + 1) * (nL + 1);
  const long long NC = N * C;
  // scratch layout in doubles: [partials S*NC][u1 NC][u2 NC][o1 NC][o2 NC][red 8][perm N ints]
  const long long cap = (long long)(RTE_NOALLOC_SCRATCH_BYTES / sizeof(double));
  const long long fixed = 4 * NC + 8 + (N + 1) / 2;
  if (N > (1ll << 26) || fixed + NC > cap) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "rte_attenuate_noalloc: %lld voxels x %lld coefficients needs %.1f MiB of scratch, the limit is %llu MiB",
             N, C, (double)(fixed + NC) * 8.0 / 1048576.0, RTE_NOALLOC_SCRATCH_BYTES >> 20);
    return set_err(RTE_ERR_UNSUPPORTED, msg);
  }
  int S = (int)std::min<long long>(8, (cap - fixed) / NC);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(RTE_ERR_DEVICE, cudaGetErrorString(e));
  double* base = nullptr;
  int rc = setup(dev, &base);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  double* part = base;
  double* u1 = part + (size_t)S * NC;
  double* u2 = u1 + NC;
  double* o1 = u2 + NC;
  double* o2 = o1 + NC;
  double* red = o2 + NC;
  int* perm = (int*)(red + 8);
  const int Ni = (int)N;
  const int tiles = (Ni + RTE_PAIR_THREADS - 1) / RTE_PAIR_THREADS;
  int chunk = ((Ni + S - 1) / S + RTE_PAIR_TS - 1) / RTE_PAIR_TS * RTE_PAIR_TS;
  S = (Ni + chunk - 1) / chunk;
  (void)tiles;
  // nothing below depends on earlier contents of the scratch array except what is written first
  k_identity<<<(Ni + 255) / 256, 256, 0, st>>>(perm, Ni);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemsetAsync(red, 0, 8 * sizeof(double), st);
  if (e == cudaSuccess) e = rte_launch_to_real((const double*)d_in, u1, u2, Ni, nL, red, st);
  for (int part_k = 0; part_k < 2 && e == cudaSuccess; part_k++) {
    PairArgs a;
    memset(&a, 0, sizeof a);
    a.N = Ni;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.Cfull = (int)C;
    a.dx = dx;
    a.dy = dy;
    a.dz = dz;
    a.prop_thresh = prop_thresh;
    a.kscale = dx * dy * dz / cm;
    a.perm = perm;
    a.mut = d_mut;
    a.Win = part_k ? u2 : u1;
    a.part = part;
    a.chunk = chunk;
    a.nsplit = S;
    e = rte_launch_pair(a, nL, 0, 0, 0, st);
    if (e != cudaSuccess) break;
    // partial sums -> output coefficients (the epilogue with no self term and no scatter)
    EpiArgs ep;
    memset(&ep, 0, sizeof ep);
    ep.N = Ni;
    ep.nx = nx;
    ep.ny = ny;
    ep.nz = nz;
    ep.Cfull = (int)C;
    ep.S = S;
    ep.nb = 1;
    ep.part = part;
    ep.selfp = nullptr;
    ep.mus = d_mut;
    ep.Wout = part_k ? o2 : o1;
    ep.red = red;
    e = rte_launch_epilogue(ep, nL, st);
  }
  if (e == cudaSuccess) e = rte_launch_to_cplx(o1, o2, (double*)d_out, Ni, nL, st);
  if (e != cudaSuccess) return set_err(RTE_ERR_DEVICE, cudaGetErrorString(e));
  return RTE_OK;
}
