/* neumann_b200_gpu_package.cu -- Neumann() of the reference's GPU package programs over librte_b200.
 *
 * Drop-in for GPU package/src/neumann.cu: the two-argument form declared at GPU package/src/rte.h:168
 * and called by rte.cu:174 and inverse_rte.cu:256, 334, 419.  It always runs the full series (the
 * FisherInfo_IO form's flag = 1).  The package's tissue tables are complex (rte.h:63, filled with zero
 * imaginary parts by inits.cu:53-60), so their real parts are passed.  Model RTE_MODEL_FIM reproduces
 * the table spherical harmonics both packages use; the GPU package's propagation of only l = 0 in the
 * intermediate terms (GPU package/src/neumann.cu:80) is not reproduced.  Failure: a message and exit(1),
 * as the reference does.  src_host is left unchanged.
 */
#include <stdio.h>
#include <stdlib.h>

#include "rte.h"
#include "rte_b200.h"

extern Geometry* geom;
extern Phantom* phan;
extern SHORT nL;

static rte_ctx* b200_ctx = NULL;

static rte_ctx* b200_context_for_globals(void) {
  if (b200_ctx) return b200_ctx;
  rte_config c;
  c.nx = geom->nX;
  c.ny = geom->nY;
  c.nz = geom->nZ;
  c.x_min = geom->x_min;
  c.x_max = geom->x_max;
  c.y_min = geom->y_min;
  c.y_max = geom->y_max;
  c.z_min = geom->z_min;
  c.z_max = geom->z_max;
  c.nL = nL;
  c.prop_thresh = geom->prop_thresh;
  c.self_sub_vox = geom->self_sub_vox;
  c.g = phan->g;
  c.n = phan->n;
  c.c = 1.0; /* rte.h: #define C 1 */
  c.model = RTE_MODEL_FIM;
  c.precision = RTE_PREC_FP64;
  c.kernel_mode = RTE_KERNEL_AUTO;
  c.device = 0;
  if (rte_create(&c, &b200_ctx) != RTE_OK) {
    fprintf(stderr, "Neumann: %s\n", rte_last_error(NULL));
    exit(1);
  }
  return b200_ctx;
}

void Neumann(complex_double* src_host, complex_double* out_host) {
  rte_ctx* ctx = b200_context_for_globals();
  rte_stop stop;
  stop.rule = RTE_STOP_REFERENCE;
  stop.max_terms = 0;
  stop.tol = 0.0;
  double mua[RTE_PAR_MAX_TISS], mus[RTE_PAR_MAX_TISS];
  if (phan->no_tiss < 1 || phan->no_tiss > RTE_PAR_MAX_TISS) {
    fprintf(stderr, "Neumann: %d tissue types (1..%d supported)\n", (int)phan->no_tiss, RTE_PAR_MAX_TISS);
    exit(1);
  }
  for (int t = 0; t < phan->no_tiss; t++) {
    mua[t] = phan->mu_abs[t].real();
    mus[t] = phan->mu_sc[t].real();
  }
  if (rte_set_medium_tissue(ctx, phan->tiss_type, phan->no_tiss, mua, mus) != RTE_OK ||
      rte_neumann(ctx, (const rte_cplx*)src_host, (rte_cplx*)out_host, 1, &stop, NULL) != RTE_OK) {
    fprintf(stderr, "Neumann: %s\n", rte_last_error(ctx));
    exit(1);
  }
}
