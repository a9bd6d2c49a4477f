/* rte_b200.h -- C ABI of the B200 Neumann-series radiative transport solver.
 *
 * Drop-in boundary for the forward, inverse-gradient and Fisher-information paths of
 * the reference research code (ajha4/DOI, FisherInfo_IO and GPU package).  Plain C
 * types only: caller-owned host buffers, opaque context, int status codes.  Nothing
 * here ever calls exit().
 *
 * Distributions crossing this boundary use the reference layout: complex double
 * (re, im) pairs, W[r*C + cnt] with voxel r = (z*nY + y)*nX + x and coefficient
 * cnt = l*l + l + m (l = 0..nL, m = -l..l), C = (nL+1)^2, in the reference's complex
 * orthonormal spherical-harmonic basis (FisherInfo_IO/src/sph_harm.cu:19-102).
 * Images are nX*nY complex values, x fastest (FisherInfo_IO/src/dist.cu:316-345 writes
 * the same order).
 */
#ifndef RTE_B200_H
#define RTE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define RTE_OK 0
#define RTE_ERR_ARG 1         /* bad argument or configuration */
#define RTE_ERR_STATE 2       /* call out of order (e.g. no medium set) */
#define RTE_ERR_DEVICE 3      /* CUDA error */
#define RTE_ERR_NOMEM 4       /* device allocation failed / admission refused */
#define RTE_ERR_IO 5          /* file could not be read or written */
#define RTE_ERR_UNSUPPORTED 6 /* feature outside this build's limits */
#define RTE_ERR_TIMEOUT 7     /* a bounded device wait ran out */
#define RTE_ERR_CANCELLED 8   /* the request was cancelled before it ran */

/* ---- discretisation models (which reference the numbers follow) ------------------- */
#define RTE_MODEL_EXACT 0 /* exact Y_lm, exact path integral, 200x200 self term, exact exitance */
#define RTE_MODEL_FIM 1   /* FisherInfo_IO kernels as shipped: 100x100 SH table, g truncated ... */
#define RTE_MODEL_CPU 2   /* CPU package (uniform medium) discretisation */

#define RTE_PREC_FP64 0  /* plain FP64 method: every pair recomputed in FP64 each term */
#define RTE_PREC_MIXED 1 /* FP32 path integrals + SH projection, FP64 sums and norms */

#define RTE_KERNEL_AUTO 0      /* mixed precision: store the voxel-pair kernel when it fits, else recompute;
                                  FP64: recompute (the plain method) */
#define RTE_KERNEL_STORE 1     /* store exp(-tau)/r^2 per voxel pair in HBM (FP32 for mixed precision,
                                  FP64 for the FP64 method: 8 N^2 bytes) */
#define RTE_KERNEL_RECOMPUTE 2 /* recompute path integrals every term */

#define RTE_SRC_COLUMN 0 /* collimated pencil on the z=0 face, column containing (pos_x,pos_y) */
#define RTE_SRC_FIM 1    /* FisherInfo_IO rule: column x == nX/2.0 && y == nY/2.0 (even grids only) */
#define RTE_SRC_CPU 2    /* CPU package rule: columns within diam/2, normalised by column count */
#define RTE_SRC_BEAM 3   /* collimated beam entering through `face` along its inward normal (new) */
#define RTE_SRC_POINT 4  /* isotropic point source in the first voxel layer behind `face` (new) */

#define RTE_STOP_REFERENCE 0 /* reference lambda > 0.9999 rule (dist.cu:1132-1172) */
#define RTE_STOP_FIXED 1     /* exactly max_terms terms */
#define RTE_STOP_REL_L2 2    /* ||W_k|| < tol * ||sum|| or max_terms */

typedef struct {
  double re, im;
} rte_cplx;

/* Mirror of the reference Geometry / Phantom-optics / Algorithm .par keys
 * (FisherInfo_IO/src/inits.cu:198-269, :22-153; rte.cu:123-128). */
typedef struct {
  int nx, ny, nz;                 /* [Geometry] nX nY nZ */
  double x_min, x_max;            /* [Geometry] xMin xMax (delX = (xMax-xMin)/nX) */
  double y_min, y_max;
  double z_min, z_max;
  int nL;                         /* [Algorithm] nL (0..7) */
  double prop_thresh;             /* [Geometry] propThresh: pairs with |r-r'| < propThresh couple */
  int self_sub_vox;               /* [Geometry] selfsubVox */
  double g;                       /* [Phantom] g */
  double n;                       /* [Phantom] n */
  double c;                       /* speed of light; the FIM model uses 1 (rte.h:15) */
  int model;                      /* RTE_MODEL_* */
  int precision;                  /* RTE_PREC_* */
  int kernel_mode;                /* RTE_KERNEL_* */
  int device;                     /* CUDA device ordinal */
} rte_config;

/* [Source] section (FisherInfo_IO/src/inits.cu:167-185). */
typedef struct {
  double pos_x, pos_y, pos_z;
  double diam;
  double theta, phi; /* read by the reference, unused */
  double mag;
  double modulation; /* intensity modulation (CPU package/src/RTE_uniform.c:120-176): rte_forward and
                        rte_forward_batch solve at the source's modulation (rte_set_modulation); other
                        calls take a source whose modulation is 0 or the context's */
  int kind;          /* RTE_SRC_* */
  int face;          /* RTE_SRC_BEAM / RTE_SRC_POINT: 0 z=0, 1 z=nZ-1, 2 y=0, 3 y=nY-1, 4 x=0, 5 x=nX-1;
                        the position on the face comes from the two in-face coordinates of pos_* */
} rte_source;

typedef struct {
  int rule;      /* RTE_STOP_* */
  int max_terms; /* RTE_STOP_FIXED / RTE_STOP_REL_L2 cap (the reference rule is capped at 10000) */
  double tol;    /* RTE_STOP_REL_L2 tolerance */
} rte_stop;

typedef struct {
  int terms;             /* Neumann terms taken (scatter-propagate applications) */
  double last_rel;       /* ||W_last|| / ||sum|| */
  double ms_device;      /* device time of the solve, CUDA events */
  double ms_setup;       /* pair-kernel precompute time (0 when not stored) */
} rte_report;

typedef struct rte_ctx rte_ctx;

/* ---- context -------------------------------------------------------------------- */
int rte_create(const rte_config* cfg, rte_ctx** out);
void rte_destroy(rte_ctx* ctx);
const char* rte_last_error(const rte_ctx* ctx); /* message of the last failed call */
size_t rte_device_bytes(const rte_ctx* ctx);    /* HBM held by this context */

/* ---- medium ----------------------------------------------------------------------
 * Tissue map form of LoadPhantom (FisherInfo_IO/src/inits.cu:22-153): tiss is nX*nY*nZ
 * uint8, z-major, x fastest; types index mua[]/mus[] of length ntypes (type 0 = air,
 * mua[0] = mus[0] = 0 in the reference). */
int rte_set_medium_tissue(rte_ctx* ctx, const uint8_t* tiss, int ntypes, const double* mua,
                          const double* mus);
/* Two tissue tables on one tissue map (compat form of the FisherInfo_IO SNR and region-gradient mains,
 * FisherInfo_IO/src/rte_snr.cu:239 and compute_grad_rte.cu:431: they change tissue values on the host but
 * drop the result of populate_info_dev(), so the device's table keeps the .par values): the pair
 * kernels' path integrals and the scatter D take mua_kernel / mus_kernel, the self-voxel term, the source
 * and its ballistic beam take mua / mus.  Forward solves, Neumann, prop_abs, images and the region
 * derivatives accept it; rte_gradient, rte_image_gradient (exact), rte_fisher and modulation return
 * RTE_ERR_UNSUPPORTED.  Any other rte_set_medium_* call returns the context to one table. */
int rte_set_medium_tissue_split(rte_ctx* ctx, const uint8_t* tiss, int ntypes, const double* mua,
                                const double* mus, const double* mua_kernel, const double* mus_kernel);
/* Per-voxel form (new): mua, mus of length nX*nY*nZ in cm^-1. */
int rte_set_medium_voxel(rte_ctx* ctx, const double* mua, const double* mus);
/* Same with DEVICE pointers (on the context's GPU), for callers whose media are already in HBM. */
int rte_set_medium_device(rte_ctx* ctx, const double* d_mua, const double* d_mus);

/* Intensity modulation, the reference's [Source] modulation (CPU package/src/RTE_uniform.c:120-176):
 * mu_a -> mu_a + i * modulation / (c/n) in every voxel, so mu_t gains a uniform imaginary part and
 * every distribution becomes complex (frequency-domain radiance; its phase is the delay).  While it
 * is non-zero, rte_source_beam, rte_prop_abs, rte_neumann, rte_images and rte_forward work with the
 * complex mu_t (pair kernels exp(-(tau + i kappa r)), self term and ballistic terms with the complex
 * mu_t); the uniform-medium convolution path is not used.  Models RTE_MODEL_EXACT and RTE_MODEL_CPU
 * (RTE_ERR_UNSUPPORTED for FIM, which reads the key and ignores it); detectors, gradients, Fisher
 * information and graph replay return RTE_ERR_UNSUPPORTED until it is set back to 0.  The self-term
 * series needs |mu_t + i kappa| * (half voxel diagonal) <= 12. */
int rte_set_modulation(rte_ctx* ctx, double modulation);

/* ---- reference entry points ----------------------------------------------------- */
/* generate_source_beam (FisherInfo_IO/src/dist.cu:66-101): xi = D A (collimated beam). */
int rte_source_beam(rte_ctx* ctx, const rte_source* src, rte_cplx* xi);

/* One prop_abs pass (FisherInfo_IO/src/kernels.cu:704-808): out = [D] A in.  flag = 1 uses
 * all orders, flag = 0 only l = 0; flag_scat = 1 applies the scatter D. */
int rte_prop_abs(rte_ctx* ctx, const rte_cplx* in, rte_cplx* out, int flag, int flag_scat);

/* Adjoint of prop_abs without scatter (new): out = A^H in, so that sum conj(y) (A x) = sum conj(A^H y) x
 * over all voxels and coefficients.  The adjoint of flag_scat = 1 is A^H D, D the real diagonal scatter.
 * Not under intensity modulation. */
int rte_prop_abs_adjoint(rte_ctx* ctx, const rte_cplx* in, rte_cplx* out, int flag);

/* Neumann (FisherInfo_IO/src/neumann.cu:23-120).  flag = 1: W_0 = src, sum_0 = out (the
 * caller passes out = src as rte.cu:148-149 does), W_{k+1} = D A W_k, sum += W_{k+1} until
 * the stop rule, then out = A sum.  flag = 0: out = A out.  src is not modified (the
 * reference used it as scratch).  nterms may be NULL. */
int rte_neumann(rte_ctx* ctx, const rte_cplx* src, rte_cplx* out, int flag, const rte_stop* stop,
                int* nterms);

/* generate_trans_image / generate_ref_image (FisherInfo_IO/src/dist.cu:103-161, 229-268)
 * of a final distribution; trans/ref are nX*nY complex (either may be NULL). */
int rte_images(rte_ctx* ctx, const rte_cplx* out, const rte_source* src, rte_cplx* trans,
               rte_cplx* ref);

/* Whole forward solve (rte.cu:139-210): source, Neumann, images.  W_out (N*C complex),
 * trans, ref and report may each be NULL. */
int rte_forward(rte_ctx* ctx, const rte_source* src, const rte_stop* stop, rte_cplx* W_out,
                rte_cplx* trans, rte_cplx* ref, rte_report* report);

/* ---- detectors and derivatives (new entry points) -------------------------------- */
typedef struct {
  int nbins; /* bins per face edge: nbins x nbins bins per face (area-weighted pixel binning) */
  int faces; /* bit mask of faces: 1 z=0, 2 z=nZ-1, 4 y=0, 8 y=nY-1, 16 x=0, 32 x=nX-1 */
} rte_detector;

/* Exitant flux per detector bin of each source: flux[src][6 faces][nbins][nbins] (faces outside
 * the mask are 0).  Fluxes integrate the exitant radiance over the outward hemisphere of each
 * face, with the ballistic beam on the z = nZ-1 face.  Single-column sources only. */
int rte_detector_flux(rte_ctx* ctx, int nsrc, const rte_source* srcs, const rte_stop* stop,
                      const rte_detector* det, double* flux);

/* Adjoint gradient of loss = sum (flux - target)^2 (target laid out as rte_detector_flux's
 * output) with respect to the per-voxel mu_a and mu_s of the current medium (N each).  One forward
 * and one adjoint Neumann series per source plus one back-projection through the path integrals;
 * exact for the discrete model when the series has converged (use RTE_STOP_REL_L2 with a small
 * tolerance for derivative checks).  The reference computes region derivatives by forward
 * sensitivity solves instead (FisherInfo_IO/src/compute_grad_rte.cu:273-385). */
int rte_gradient(rte_ctx* ctx, int nsrc, const rte_source* srcs, const rte_stop* stop,
                 const rte_detector* det, const double* target, double* loss, double* g_mua,
                 double* g_mus);

/* Gradient of the reference's image misfit, loss = sum_j (gbar_j - g_j)^2 over one exitance image of
 * one source (image 0: the transmission image with its ballistic term, the gbar of
 * FisherInfo_IO/src/compute_grad_rte.cu:257 and GPU package/src/inverse_rte.cu; 1: the reflection
 * image), with respect to the per-voxel mu_a and mu_s (N each), from ONE forward and ONE adjoint
 * Neumann series (new: the reference takes one tangent solve per tissue, or per voxel in the GPU
 * package).  g: nX*nY target image.  deriv:
 *   RTE_DERIV_EXACT      the exact derivative of the discrete model, as rte_gradient (collimated z = 0
 *                        sources; fixed or relative-L2 stop rule);
 *   RTE_DERIV_REFERENCE  the reference's tangent model: a change of mu in voxel r acts as the source
 *                        -C dmu_a out(r) (mu_a) or (-C + g^l) dmu_s out(r) (mu_s), C = 1, of a tangent
 *                        solve whose transmission (or reflection) image without ballistic term is dgbar
 *                        (compute_grad_rte.cu:288-325, 343-377; per voxel in GPU package/src/
 *                        inverse_rte.cu:293-433).  g_mua[r] = sum_j 2 (gbar_j - g_j) dgbar_j(r), so
 *                        av * (sum of g_mua over tissue t) is the reference's grad2[t] (av = 0.01 for
 *                        mu_a, 1 for mu_s) and g_mua[r] the GPU package's per-voxel grada[r].  The adjoint
 *                        series takes the forward solve's term count (exact for RTE_STOP_FIXED).
 * loss may be NULL. */
#define RTE_DERIV_EXACT 0
#define RTE_DERIV_REFERENCE 1
int rte_image_gradient(rte_ctx* ctx, const rte_source* src, const rte_stop* stop, int image, int deriv,
                       const double* g, double* loss, double* g_mua, double* g_mus);

/* Region derivatives of the reference's inverse main (FisherInfo_IO/src/compute_grad_rte.cu:205-385),
 * one evaluation at the current medium: forward solve, gbar = transmission image; for every tissue
 * type t >= 1 a tangent solve of -C mask_t(out) (mu_a) and of mask(-C out + g^l out) (mu_s), C = 1,
 * projected to the transmission image dgbar without the ballistic term, and
 *   grad[t]  = -2 av sum_j dgbar_j / (g_j - gbar_j),   grad2[t] = -2 av sum_j (g_j - gbar_j) dgbar_j
 * over pixels with g_j or gbar_j non-zero (av = 0.01 for mu_a, 1 for mu_s); residual = sum log((gbar-g)^2)
 * over non-zero differences, residual2 = sum (gbar-g)^2.  compat = 1 reproduces the reference's mu_s
 * mask, which zeroes only the last voxel (a stale index, compute_grad_rte.cu:363) whenever another
 * tissue exists; compat = 0 uses the tissue mask.  g: nX*nY measured image; tiss: N tissue types;
 * output arrays have ntypes entries (entry 0 is 0). */
int rte_region_gradient(rte_ctx* ctx, const rte_source* src, const rte_stop* stop, const double* g,
                        const uint8_t* tiss, int ntypes, int compat, double* grada, double* grada2,
                        double* grads, double* grads2, double* residual, double* residual2);

/* Fisher information of P region parameters (mu_a of the voxels in masks[p*N .. p*N+N-1]) under
 * Poisson noise, F[a*P+b] = sum_j dg_a,j dg_b,j / gbar_j over pixels with gbar_j != 0, from one forward
 * and P tangent solves of -C mask_p(out) (FisherInfo_IO/src/rte_fim.cu:236-331).  image: 0
 * transmission, 1 reflection (the reference main's choice), 2 both. */
int rte_fisher_regions(rte_ctx* ctx, const rte_source* src, const rte_stop* stop, int P, const uint8_t* masks,
                       int image, double* F);

/* Fisher information of P parameters of the medium (new).  dmua, dmus: P x N arrays, the
 * derivative of each voxel's mu_a / mu_s with respect to each parameter (e.g. the position and
 * contrast of an inclusion through a smooth partial-volume rasterisation).  For every collimated
 * source: one forward solve and P tangent solves of the discrete model (the derivative of the
 * attenuation operator recomputes the path integral of the parameter direction along every voxel
 * pair), giving J = d(binned exitant flux)/d(parameter) on the detector of rte_detector_flux; with
 * Poisson counts F = sum over sources and bins with flux > 0 of J_b,p J_b,q / flux_b.  Exact for the
 * discrete model when the series converge (RTE_STOP_REL_L2 with a small tolerance).  In a
 * mixed-precision context the forward solves (whose fluxes weight every bin) run by the FP64 method
 * with the path integrals recomputed, and the tangent solves in mixed precision.  J (may be NULL):
 * nsrc * 6 * nbins^2 rows of P.  F: P x P.  Sources: RTE_SRC_COLUMN, RTE_SRC_FIM, RTE_SRC_BEAM. */
int rte_fisher(rte_ctx* ctx, int nsrc, const rte_source* srcs, const rte_stop* stop, const rte_detector* det,
               int P, const double* dmua, const double* dmus, double* J, double* F);

/* Batched forward solves (new): nsrc <= 4 sources on the current medium, propagated together so
 * each voxel pair's direction, spherical harmonics and kernel value serve every source.  Outputs
 * are the nsrc single-source results back to back (W_out nsrc*N*C, trans/ref nsrc*nX*nY, each may
 * be NULL).  Stop rule RTE_STOP_FIXED or RTE_STOP_REL_L2 (norms over all sources). */
int rte_forward_batch(rte_ctx* ctx, int nsrc, const rte_source* srcs, const rte_stop* stop,
                      rte_cplx* W_out, rte_cplx* trans, rte_cplx* ref, rte_report* report);

/* One forward solve of nsrc <= 4 sources on the current medium with a fixed number of terms,
 * recorded once per context as a CUDA graph (pair-kernel precompute, series, final attenuation)
 * and replayed afterwards; the first call on a context records the graph.  Images as
 * rte_forward_batch.  The serving path uses it. */
int rte_forward_graph(rte_ctx* ctx, int nsrc, const rte_source* srcs, int nterms, rte_cplx* trans,
                      rte_cplx* ref, rte_report* report);

/* ---- serving: continuous batching of forward solves (new) ---------------------------
 * Requests of any grid, order, medium and sources are admitted as execution slots and HBM
 * (budget) free up and run concurrently on the device, one context (and CUDA stream) per
 * admitted request; contexts are kept per shape and reused (idle ones of other shapes are
 * evicted when HBM is short).  Latency = submit to completion. */
typedef struct {
  int n;             /* voxels per edge of the cubic grid */
  double dx;         /* voxel edge (cm); x and y centred on 0, z from 0 */
  int nL;            /* SH order */
  double g, n_index; /* anisotropy, refractive index */
  int precision;     /* RTE_PREC_MIXED (stored pair kernel) or RTE_PREC_FP64 */
  int terms;         /* Neumann terms */
  int nsrc;          /* 1..4 sources solved together */
  rte_source src[4];
  const double* mua; /* n^3 values each, copied by rte_server_submit */
  const double* mus;
} rte_request;

typedef struct {
  int status;        /* RTE_OK or the failure code */
  double latency_ms; /* submit -> done */
  double queue_ms;   /* submit -> admitted */
  double service_ms; /* admitted -> done */
  double device_ms;  /* CUDA-event time of the solve on the device */
} rte_result_info;

typedef struct {
  long long submitted, completed, failed, cancelled, inflight, pending;
  int contexts;        /* contexts alive (busy or idle) */
  size_t hbm_reserved; /* HBM reserved by admitted shapes */
  double p50_ms, p99_ms, mean_ms; /* latency of completed requests */
  double wall_s;       /* first submit -> last completion */
} rte_server_info;

typedef struct rte_server rte_server;

/* hbm_budget_gb <= 0: 85% of the free memory; nworkers = requests in flight at most.  A failed
 * rte_server_create / rte_server_submit / rte_server_wait leaves its reason for rte_last_error(NULL)
 * on the calling thread (for a failed request: the admission or context error that stopped it). */
int rte_server_create(int device, double hbm_budget_gb, int nworkers, rte_server** out);
int rte_server_submit(rte_server* srv, const rte_request* req, long long* ticket);
/* Waits up to timeout_s (0, negative or NaN: poll; +inf or anything above 1e8 s: 1e8 s); trans/ref
 * get nsrc*n*n complex values.  Returns the request status (RTE_ERR_TIMEOUT if it is still running,
 * and the ticket stays valid).  A finished ticket can be waited for once. */
int rte_server_wait(rte_server* srv, long long ticket, double timeout_s, rte_cplx* trans, rte_cplx* ref,
                    rte_result_info* info);
int rte_server_cancel(rte_server* srv, long long ticket); /* only before it starts */
int rte_server_stats(rte_server* srv, rte_server_info* out);
void rte_server_destroy(rte_server* srv);

/* ---- reference parameter and image files (drop-in for the reference programs) -------
 * .par files in the reference's iniparser dialect (FisherInfo_IO/src/iniparser.cu:455-620): '#'
 * comment lines, [section], key = value (quoted, or cut at ';' / '#'), trailing '\' joins lines,
 * case-insensitive "section:key" lookup, last repeat wins; ints as strtol(s, 0, 0), doubles as
 * atof. */
typedef struct rte_par rte_par;
int rte_par_load(const char* path, rte_par** out); /* RTE_ERR_IO if the file cannot be opened */
void rte_par_free(rte_par* p);
const char* rte_par_get_string(const rte_par* p, const char* key, const char* def);
int rte_par_get_int(const rte_par* p, const char* key, int def);
double rte_par_get_double(const rte_par* p, const char* key, double def);

#define RTE_PAR_MAX_TISS 256
/* Solver inputs as the reference mains derive them from a .par file: LoadGeometry / LoadPhantom /
 * LoadSource (FisherInfo_IO/src/inits.cu:22-269; float extents and thresholds as the reference
 * stores them) when [Phantom] TissMapFile is given, else the CPU package's uniform-medium keys
 * (CPU package/src/Inits.c:24-131: [Phantom] mua, mus, c).  Optional keys of this library:
 * [Algorithm] Model = fim|cpu|exact, Precision = fp64|mixed, KernelMode = auto|store|recompute,
 * StopRule = reference|fixed|rel_l2, MaxTerms, Tol, Device, DetectorBins; [Phantom] MuaFile /
 * MusFile (N doubles each, per-voxel media); [Source] Kind = fim|column|cpu|beam|point, Face;
 * [Runtime] FluxFile.  Defaults reproduce the reference. */
typedef struct {
  rte_config cfg;
  rte_source src;
  rte_stop stop;                 /* StopRule / MaxTerms / Tol (default: the reference rule) */
  int style;                     /* 0: FisherInfo_IO tissue-map file, 1: CPU-package uniform file */
  int ntypes;                    /* tissue types including type 0 (outside, mu = 0) */
  double mua[RTE_PAR_MAX_TISS], mus[RTE_PAR_MAX_TISS];
  uint8_t* tiss;                 /* nX*nY*nZ tissue map (owned; rte_problem_free) */
  double* mua_vox;               /* per-voxel media from MuaFile / MusFile, or NULL */
  double* mus_vox;
  double mut_mean;               /* mean mu_t over the voxels (inits.cu:136-147) */
  double diffuse_prop_thresh;    /* propThresh after the forward main's diffuse-medium rule (rte.cu:116-119) */
  int nterms;                    /* [Algorithm] nTerms (read; the reference's auto-stop ignores it) */
  int detector_bins;             /* [Algorithm] DetectorBins (0: no flux file) */
  int num_iterations;            /* [Runtime] numIterations */
  double step_a, step_s;         /* [Runtime] stepsizea, stepsizes */
  char trans_file[1024], ref_file[1024], phase_file[1024], g_file[1024], flux_file[1024];
} rte_problem;
/* read_map = 1 reads [Phantom] TissMapFile (RTE_ERR_IO when missing); 0 makes every voxel tissue 1,
 * as LoadPhantom(ini, 0) does for the Fisher main.  No device work. */
int rte_par_problem(const rte_par* p, int read_map, rte_problem* out);
void rte_problem_free(rte_problem* pr);

/* Image files: 2 ints then the real and the imaginary nX*nY planes (doubles, x fastest); the
 * header is (nY, nX) as FisherInfo_IO/src/dist.cu:316-345 writes it, or (nX, nY) with cpu_layout
 * as CPU package/src/Dist.c:16-40 does.  Phase images: 2 ints + nX*nY doubles (dist.cu:291-314).
 * rte_read_image reads a measured image (gFile): 2 ints + nX*nY doubles
 * (compute_grad_rte.cu:151-161). */
int rte_write_image(const char* path, int nx, int ny, const rte_cplx* img, int cpu_layout);
/* phase images: FisherInfo_IO layout (cpu_layout = 0: nY, nX then the values) or the CPU package's
 * OutputPhaseImage (cpu_layout = 1: nX, nY, then the values x fastest, Dist.c:47-65) */
int rte_write_phase_image(const char* path, int nx, int ny, const double* phase, int cpu_layout);
int rte_read_image(const char* path, int nx, int ny, double* out);
/* Detector downsampling of an nX x nY image by ds (replaces downsample_image,
 * FisherInfo_IO/src/dist.cu:271-289): out[i*(nY/ds) + j] = sum over a, b < ds of
 * img[(i*ds + a)*nY + j*ds + b], i < nX/ds, j < nY/ds; the caller provides (nX/ds)*(nY/ds) values.
 * Sums start at zero (the reference's start from uninitialised memory).  Host-only. */
int rte_downsample_image(const rte_cplx* img, int nx, int ny, int ds, rte_cplx* out);

/* The CPU package's boundary outputs of a final distribution W (N*C complex, reference layout;
 * host code, no context): the side-face images of ComputeSideFaceImages (CPU package/src/Dist.c:
 * 353-532; x faces nZ*nY values at k + j*nZ, y faces nZ*nX at k + i*nZ; each pointer may be NULL) and
 * the photon number of ComputePhotonNumber (Dist.c:538-989: outgoing and "incoming" hemisphere sums
 * on all six faces plus the ballistic beam, with the package's 101 x 101 rectangle rule and its uniform
 * mu_t, whose imaginary part mu_t_im is the modulation's).  cfg gives the geometry, nL and c / n. */
int rte_cpu_face_outputs(const rte_config* cfg, const rte_cplx* W, const rte_source* src, double mu_t,
                         double mu_t_im, rte_cplx* side_x0, rte_cplx* side_x1, rte_cplx* side_y0,
                         rte_cplx* side_y1, rte_cplx* photons);

/* ---- allocation-free entry point (no counterpart in the reference) ------------------
 * For callers that must not allocate device memory when they run the solver: work recorded
 * into a CUDA graph (cudaMalloc is illegal during stream capture), plug-ins whose host
 * application owns all device memory through its own pool, real-time loops that cannot
 * wait on the allocator.  It needs no context (rte_create allocates).
 *
 * One application of the off-diagonal attenuation operator in exact FP64 (the pair sum of
 * compute_propabs x dV, without the self-voxel term and without scatter):
 *   out[r] = sum_{r' != r, |r-r'| < prop_thresh} conj(Y(w)) (Y(w) . in[r']) exp(-tau) dV/(cm |r-r'|^2)
 * on caller-owned DEVICE buffers: d_mut (N doubles, mu_a + mu_s), d_in and d_out (N*C complex,
 * reference layout), queued on `stream` (a cudaStream_t, may be NULL).  Scratch memory is a fixed
 * 64 MiB array inside the library, held on every GPU that loads it; problems whose
 * (4 + 1) * N * C doubles plus N ints exceed it are rejected with RTE_ERR_UNSUPPORTED (33^3
 * voxels at nL = 5 fit; the message from rte_last_error(NULL) gives the need).  The first call
 * on a device looks up the scratch address and uploads constant tables: make it before any
 * stream capture.  Calls share the scratch array, so calls whose GPU work overlaps race. */
int rte_attenuate_noalloc(int nx, int ny, int nz, double dx, double dy, double dz, int nL,
                          double prop_thresh, double cm, const double* d_mut, const rte_cplx* d_in,
                          rte_cplx* d_out, void* stream);

/* ---- measurement helpers (no reference counterpart) ------------------------------ */
typedef struct {
  long long launches;     /* kernels launched by this context since the last reset */
  double ms_pair;         /* summed device time of the pair (A operator) kernels */
  long long n_pair;
  double ms_store;        /* pair-kernel precompute */
  long long n_store;
  double ms_epi;          /* epilogue (self term, scatter, sums) */
  long long n_epi;
} rte_stats;

/* The CUDA stream (cudaStream_t) all of this context's work is queued on. */
void* rte_get_stream(rte_ctx* ctx);
/* on = 1: time every pair / precompute / epilogue launch with CUDA events on that stream. */
int rte_set_profiling(rte_ctx* ctx, int on);
/* Synchronises the stream, returns the counters and resets them. */
int rte_get_stats(rte_ctx* ctx, rte_stats* out);

/* FP32 (fp64 = 0) or FP64 (fp64 = 1) FMA throughput of the device in TFLOP/s, measured with an
 * 8-chain FMA loop: the denominator of the roofline of the CUDA-core-bound kernels.  FP32 takes the
 * faster of a scalar and a packed (f32x2) stream; fp64 = 2, 3 and 4 time one FP32 stream alone: scalar,
 * packed, and packed with three distinct operand registers per instruction.  Other values: RTE_ERR_ARG. */
int rte_measure_fma_peak(int device, int fp64, double* tflops);

#ifdef __cplusplus
}
#endif
#endif /* RTE_B200_H */
