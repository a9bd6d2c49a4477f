/* neumann_b200.cu -- Neumann() of the reference's FisherInfo_IO programs over librte_b200.
 *
 * Drop-in for FisherInfo_IO/src/neumann.cu: the same signature as the declaration at
 * FisherInfo_IO/src/rte.h:187, called by the reference's mains (rte.cu:182, compute_grad_rte.cu:249,
 * 299, 369, rte_fim.cu:237, 276, 309, rte_snr.cu).  Build it in place of neumann.cu and link with
 * -lrte_b200; the rest of the reference (parameter reading, source, images) stays as it is.
 *
 * The problem comes from the reference's globals (geom, phan, nL), as neumann.cu reads them.  The
 * context is created on the first call (FisherInfo_IO discretisation, FP64 method, device 0) and
 * reused; the tissue table is re-sent on every call because the inverse mains edit phan->mu_abs and
 * phan->mu_sc between calls.  The reference's convention on failure is kept: a message and exit(1).
 * One difference a caller can see: src_host is left unchanged (neumann.cu used it as scratch).
 * The `cudacomplex` of the reference is two doubles, the same bytes as rte_cplx.
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
  c.c = 1.0; /* the speed of light of FisherInfo_IO (rte.h: #define C 1) */
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

void Neumann(complex_double* src_host, complex_double* out_host, int flag) {
  rte_ctx* ctx = b200_context_for_globals();
  rte_stop stop;
  stop.rule = RTE_STOP_REFERENCE; /* StopIteration's lambda rule (dist.cu:1132-1172) */
  stop.max_terms = 0;
  stop.tol = 0.0;
  if (rte_set_medium_tissue(ctx, phan->tiss_type, phan->no_tiss, phan->mu_abs, phan->mu_sc) != RTE_OK ||
      rte_neumann(ctx, (const rte_cplx*)src_host, (rte_cplx*)out_host, flag, &stop, NULL) != RTE_OK) {
    fprintf(stderr, "Neumann: %s\n", rte_last_error(ctx));
    exit(1);
  }
}
