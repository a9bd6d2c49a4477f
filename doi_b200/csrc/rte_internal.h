// rte_internal.h -- shared declarations between the host context (rte_host.cpp) and the
// sm_100a kernels (rte_kernels.cu).  Not part of the public ABI (include/rte_b200.h).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define RTE_MAX_L 7
#define RTE_PAIR_THREADS 128  // destination voxels per CTA (one per thread)
#define RTE_PAIR_TS 64        // source voxels staged in shared memory per step
#define RTE_MAX_MOM 48        // self-term power-series terms

// Stored FP32 pair kernel layout: blocks of 128 destination slots, each block [source slot][128
// destinations] with ld (>= N) source rows.  The kernel values of a run of consecutive sources for one
// pair-kernel CTA's 128 destinations are then one contiguous block (a single bulk copy).
#define RTE_KBLK 128
__host__ __device__ inline size_t kmat_index(size_t s, size_t d, size_t ld) {
  return ((d / RTE_KBLK) * ld + s) * RTE_KBLK + (d % RTE_KBLK);
}

struct PairArgs {
  int N, nx, ny, nz, Cfull;
  double dx, dy, dz;
  double prop_thresh;
  double kscale;        // dV / cm folded into the pair kernel
  const int* perm;      // destination slot -> voxel index (spatially compact order)
  const double* mut;    // mu_t per voxel, FP64
  const float* mutf;    // mu_t per voxel, FP32
  const double* Win;    // current term, real basis, N x Cfull, FP64
  const float* Winf;    // current term, FP32 copy in slot order, coefficient c times N_c (sh_eval_monic)
  float* Kmat;          // stored pair kernel K(source slot, destination slot), blocked (kmat_index, ld = Kld)
  double* Kmat64;       // FP64 stored kernel (FP64 method), row-major [source slot][destination slot], stride Kld
  size_t Kld;
  double* part;         // split-K partial sums, [S][N][Cfull], indexed by voxel
  float* partf;         // FP32 partial sums in the same layout (tile-staged kernel: raw chunk sums, no N_c)
  int chunk;            // source voxels per blockIdx.y
  int nsplit;           // S
  int nb;               // right-hand sides sharing the medium (mixed kernels), layout [N][nb][Cfull]
  const float4* slot_xyz;  // per slot: (x, y, z) voxel coordinates as exact floats, w = voxel index
  int cpad;             // FP32 source row length in floats: nb*cstride rounded up to a multiple of 4
  int cstride;          // FP32 row stride of one right-hand side: Cfull rounded up to a multiple of 4
  int* err;             // set to 1 when a bounded wait runs out (kernel result invalid)
  // tangent pass (k_pair_tangent): derivative of mu_t along a parameter direction, and the voxel
  // bounding box of its support (pairs whose segment misses the box have no path derivative)
  const double* dmut;
  int box_lo[3], box_hi[3];  // (x, y, z) voxel indices
  const int* islot;          // voxel -> slot (row of the stored kernel)
  // intensity modulation: mu_t has the uniform imaginary part kappa, so every pair kernel gains the
  // phase exp(-i kappa |r - r'|); the right-hand sides are complex, (real, imaginary) pairs of rows
  double kappa;
  // transposed operator of the table model: each pair's table direction is snapped from the reverse
  // displacement (source minus destination).  Snapping does not commute with negation, so for the
  // FisherInfo_IO table A^T != P A P; with exact SH the parity form is used instead.
  int transpose;
  int tile;  // staged stored-kernel launch: 0 = 32-source tiles, 1 = 64-source tiles (autotuned)
};

struct EpiArgs {
  int N, nx, ny, nz, Cfull, S, nb;  // nb right-hand sides, layout [N][nb][Cfull]
  const double* part;   // [S][N][nb][Cfull]
  const float* partf;   // or FP32 chunk sums of the tile-staged kernel, times N_c here (then part is unused)
  const double* selfp;  // self-voxel term [N][nb][Cfull] (may be null)
  const double* mus;
  int flag_scat;
  double scat[RTE_MAX_L + 1];  // per-l scatter factor (times mu_s of the voxel)
  double* Wout;         // FP64 result (may alias nothing else)
  float* Woutf;         // FP32 copy in slot order (times N_c), rows of cpad floats (may be null)
  const int* islot;     // voxel -> slot
  int cpad, cstride;
  double* sum;          // running sum (null = do not accumulate)
  double* red;          // [0] ||Wout||^2 [1] ||sum||^2 [2] stop-layer sum of Wout [3] of sum
  int cplx;             // right-hand sides are (real, imaginary) pairs: odd ones are imaginary parts
};

struct SelfArgs {
  int N, nb, Cfull, Cact, K;
  const double* W;      // [N][nb][Cfull]
  const double* mut;
  const int* idx;       // voxel -> row of lut (null: power series)
  const double* lut;    // [ndistinct][Cfull][Cfull]
  const double* mom;    // [K][Cfull][Cfull]
  double scale;         // dV / cm
  int air_no_self;
  double* out;          // [N][nb][Cfull]
  // derivative mode: out = scale * dmut(r) * dD/dmu(mu_t(r)) W (dlut rows, or the series' derivative)
  const double* dmut;   // null: the self term itself
  const double* dlut;   // [ndistinct][Cfull][Cfull]
  // complex mu_t = mu_t + i kappa (intensity modulation): W holds (real, imaginary) pairs of rows,
  // lut_im the imaginary parts of the table (the power series takes the complex mu_t directly)
  double kappa;
  const double* lut_im;
};

struct ImgArgs {
  int nx, ny, nz, Cfull, L, vstride;
  const double* out;
  double wt[RTE_MAX_L + 1];  // transmission weights per l (m = 0 coefficient)
  double wr[RTE_MAX_L + 1];  // reflection weights per l
  const double* fball;       // ballistic flux per face pixel (z- first, z+ next); may be null
  const double* fball_im;    // its imaginary part under intensity modulation (may be null)
  const double* out_im;      // imaginary-part distribution, same layout as out (may be null)
  double* trans;  // nx*ny complex (re, im)
  double* ref;
};

// SH recurrence tables (host-computed, see rte_host.cpp) uploaded to __constant__.
struct ShTables {
  double A[64], B[64];   // q_l^m = A z q_{l-1}^m - B q_{l-2}^m, index l*(l+1)/2 + m
  double Q0[RTE_MAX_L + 1];  // q_m^m
};

#define RTE_MAX_SRC_COLS 512

struct SrcArgs {
  int nx, ny, nz, Cfull, L, kind, ncols;
  int face;                   // entry face (detector order: z-, z+, y-, y+, x-, x+)
  int cols[RTE_MAX_SRC_COLS]; // pixels of the entry face (row-major in the face) hit by the beam
  double coef[64];            // per real coefficient: scale * g^l * R_lm(beam direction)
  double scale, mag, dlen, dV, z_min, dz;
  int vstride;   // elements between consecutive voxels of W (Cfull for one right-hand side)
  const double* mut;
  const double* mus;
  double* W;     // N x vstride, zeroed by the caller
  double* fball; // ballistic exitant flux per face pixel (all six faces), zeroed by the caller
  // intensity modulation: attenuation with mu_t + i kappa; the imaginary part of the source goes to
  // W + Cfull (the second row of each voxel's pair) and that of the ballistic flux to fball_im
  double kappa;
  double* fball_im;
};

// detector faces and the adjoint gradient
struct FaceArgs {
  int nx, ny, nz, Cfull, vstride;
  const double* out;   // real basis [N][vstride]
  const double* h;     // [6][Cfull] exitant-flux weights of each face (area and cm included)
  const double* fball; // ballistic flux per face pixel, same layout as J (may be null)
  double* J;           // fluxes of all face pixels (z-, z+, y-, y+, x-, x+ concatenated)
  const double* rho;   // adjoint seed: dL/dJ per face pixel
  double* e;           // adjoint seed field [N][Cfull]
};

struct BpArgs {
  int N, nx, ny, nz, Cfull;
  double dx, dy, dz, prop_thresh, kscale;
  const int* perm;
  const int* islot;
  const double* mut;
  const float* mutf;
  const double* y;     // destination-side field [N][Cfull] (voxel order)
  const double* S;     // source-side field [N][Cfull] (voxel order)
  const float* Kmat;   // stored pair kernel (null: recompute the path integral)
  const double* Kmat64;  // FP64 stored pair kernel (FP64 contexts in stored-kernel mode)
  size_t Kld;
  double* g;           // gradient w.r.t. mu_t, accumulated [N]
  int use_smem;        // per-CTA private accumulator of N entries in shared memory (set by the launcher)
  void* Q;             // per unordered pair weight [source slot][destination slot] (row stride Kld), T
  int accumulate;      // k_bp_weights: add to Q (later sources) instead of overwriting
};

struct GradLocalArgs {
  int N, Cfull, Cact;
  const double* y;      // e + D lambda
  const double* lam;    // adjoint field
  const double* S;      // forward running sum
  const double* out;    // A S
  const double* mus;
  const double* mut;
  const int* idx;       // voxel -> distinct mu_t (null: power series)
  const double* dlut;   // d Dself / d mu_t per distinct value [nd][C][C]
  const double* mom;
  int K;
  double scale;         // dV / cm
  int air_no_self;
  double scat[RTE_MAX_L + 1];
  double* gt;           // += self-term part of dL/dmu_t
  double* gs;           // += scatter part of dL/dmu_s
};

extern "C++" {
cudaError_t rte_launch_face_flux(const FaceArgs& a, cudaStream_t st);
cudaError_t rte_launch_adjoint_seed(const FaceArgs& a, cudaStream_t st);
cudaError_t rte_launch_parity(double* x, int N, int L, int vstride, cudaStream_t st);
cudaError_t rte_launch_axpy(double* y, const double* x, double alpha, size_t n, cudaStream_t st);
// ga[r] = sum_c fa[l] lam[r][c] out[r][c], gs[r] likewise with fs (N voxels, rows of (L+1)^2)
cudaError_t rte_launch_tangent_pair_dots(const double* lam, const double* out, const double* fa, const double* fs, int N,
                                         int L, double* ga, double* gs, cudaStream_t st);
cudaError_t rte_launch_y_field(double* y, const double* e, const double* lam, const double* mus, const double* scat,
                               int N, int L, int Cfull, cudaStream_t st);
// Symmetric back-projection in two passes: pair weights of one source added into Q, then one walk
// over every unordered pair scattering Q * length into the gradient.
cudaError_t rte_launch_bp_weights(const BpArgs& a, int LA, int fp64, cudaStream_t st);
cudaError_t rte_launch_bp_walk(const BpArgs& a, int fp64, cudaStream_t st);
cudaError_t rte_launch_pair_tangent(const PairArgs& a, int LA, int fp64, int table, cudaStream_t st);
// q = mus * scat_l * T + dmus * scat_l * out (per voxel and coefficient; q rows qstride apart)
cudaError_t rte_launch_tangent_rhs(double* q, int qstride, const double* T, const double* out, const double* mus,
                                   const double* dmus, const double* scat, int N, int L, cudaStream_t st);
cudaError_t rte_launch_scatter_add(double* dst, int dstride, const int* idx, const double* vals, int n, int C,
                                   cudaStream_t st);
cudaError_t rte_launch_strided_add(double* dst, const double* a, int astride, const double* b, int N, int C,
                                   cudaStream_t st);
cudaError_t rte_launch_masked_scale(const double* in, double* out, const uint8_t* mask, const double* fac, int N,
                                    int L, cudaStream_t st);
cudaError_t rte_launch_grad_local(const GradLocalArgs& a, cudaStream_t st);
// message returned by rte_last_error(NULL) on this thread
__attribute__((visibility("hidden"))) void rte_set_global_error(const char* msg);
cudaError_t rte_launch_source(const SrcArgs& a, cudaStream_t st);
cudaError_t rte_launch_medium(const double* mua, const double* mus, double* mut, double* mus_out, float* mutf,
                              int N, double* red_max, cudaStream_t st);
cudaError_t rte_launch_fma_peak(int fp64, int iters, float* sink, cudaStream_t st, int blocks);
cudaError_t rte_upload_sh_tables(const ShTables& t);
// Uniform-medium convolution path (rte_fft.cpp): grid, padded grid, spacing, coupling distance,
// kernel scale, mu_t, and the pair range [p0, p1) of one sampling launch.
struct FftTabArgs {
  int nx, ny, nz, Mx, My, Mz;
  double dx, dy, dz, prop_thresh, kscale, mut;
  int p0, p1;
};
cudaError_t rte_launch_fft_table(const FftTabArgs& a, int L, int table, double* T, size_t M, cudaStream_t st);
cudaError_t rte_launch_fft_pad(const double* W, int vstride, int Cfull, int Cact, int nb, const FftTabArgs& a, double* F,
                               size_t M, cudaStream_t st);
cudaError_t rte_launch_fft_extract(const void* spec, double* tau, int p0, int np, int C, size_t Mk, cudaStream_t st);
cudaError_t rte_launch_fft_product(const void* That, const void* Wh, void* Oh, int C, int Cact, int nb, size_t Mk,
                                   int complex_table, cudaStream_t st);
cudaError_t rte_launch_fft_crop(const double* F, int Cfull, int Cact, int nb, const FftTabArgs& a, double* part,
                                size_t M, cudaStream_t st);
struct FftState;
cudaError_t rte_fft_prepare(FftState** s, const FftTabArgs& a, int L, int table, int nbmax, cudaStream_t st);
cudaError_t rte_fft_apply(FftState* s, const double* W, int vstride, int Cfull, int LA, int nb, double* part,
                          cudaStream_t st);
size_t rte_fft_bytes(int nx, int ny, int nz, int L, int nbmax);
cudaError_t rte_fft_warm(FftState* s, int nf);
uintptr_t rte_fft_signature(const FftState* s);
void rte_fft_destroy(FftState* s);

// host copies: the recurrence tables and the real SH R_c at a unit direction (index l*l + l + m)
ShTables make_sh_tables();
void sh_real_host(const ShTables& t, int L, double x, double y, double z, double* R);
cudaError_t rte_launch_pair(const PairArgs& a, int LA, int precision, int table, int stored, cudaStream_t st);
// fp64 = 1: FP64 path sums and exp into a.Kmat64; else FP32 into a.Kmat
cudaError_t rte_launch_store_kernel(const PairArgs& a, cudaStream_t st, int fp64 = 0);
cudaError_t rte_pair_occupancy(int LA, int precision, int table, int stored, int nb, int cpad, int* blocks_per_sm,
                               int cplx = 0, int tile = 0);
cudaError_t rte_launch_epilogue(const EpiArgs& a, int LA, cudaStream_t st);
cudaError_t rte_launch_images(const ImgArgs& a, cudaStream_t st);
cudaError_t rte_launch_self(const SelfArgs& a, cudaStream_t st);
// complex basis -> real parts; u1/u2 rows ostride apart (0: C)
cudaError_t rte_launch_to_real(const double* cplx, double* u1, double* u2, int N, int L, double* red,
                               cudaStream_t st, int ostride = 0);
cudaError_t rte_launch_to_cplx(const double* u1, const double* u2, double* cplx, int N, int L,
                               cudaStream_t st, int ustride = 0);
cudaError_t rte_launch_layer_sums(const double* W, const double* S, int N, int nx, int ny, int nz, int Cfull,
                                  double* red, cudaStream_t st, int cplx = 0);
cudaError_t rte_launch_f64_to_f32(const double* a, float* b, size_t n, cudaStream_t st);
// FP64 [N][vstride] (voxel order) -> FP32 [slot][cpad] (slot order), coefficient c scaled by the monic
// SH normalisation N_c that the mixed pair kernels factor out of their per-pair recurrence
cudaError_t rte_launch_to_f32_slots(const double* a, float* b, const int* islot, int N, int vstride, int cpad,
                                    int Cfull, int cstride, cudaStream_t st);
}
