/*
 * sparc_oracle.h -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A CPU (C++17, FP64, OpenMP) restatement of the reference SPARC time step
 * over the global domain.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference arm of bench.py load it, and only as the checker
 * or the timed CPU baseline.  The product (libsparc_gpu.so) never links it.
 *
 * Parity is unpinned by the reference's own tests: the reference has no
 * tests, golden vectors or fixtures, and it cannot be built here (Fortran,
 * MPI, parallel HDF5 are absent).  The restatement is pinned by analytic
 * known-answer tests and by committed golden fixtures of its own output.
 *
 * Every function names the reference file:line it restates.
 */
#ifndef SPARC_ORACLE_H
#define SPARC_ORACLE_H

#include <stdint.h>
#include "../include/sparc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_handle orc_handle;

/* INIT_MPI + INITANDALLOCATE + READ_IN_HDF5 + INITIALISE_RHS +
 * INITIALIZE_STEP.  Returns NULL on error (message in err). */
orc_handle *orc_create(const sparc_params *p, const double *rho0,
                       const double *pre0, const double *cs0,
                       const double *bx0, const double *by0,
                       const double *bz0, const double *zaxis_mm,
                       const double *grav, char *err, int errlen);
void orc_destroy(orc_handle *h);
int  orc_set_source(orc_handle *h, const sparc_source *src);
int  orc_sizes(orc_handle *h, int64_t *n_state, int64_t *n_psi);
int  orc_set_state(orc_handle *h, const double *a, const double *psi);
int  orc_get_state(orc_handle *h, double *a, double *psi);
/* forcing of iteration nn + STEP + diagnostics (driver.f90:125-183) */
int  orc_step(orc_handle *h, int64_t nn);
/* FILTER_VARS after iteration nn (driver.f90:200) */
int  orc_filter_vars(orc_handle *h, int64_t nn);
/* driver iterations first .. first+count-1 */
int  orc_run(orc_handle *h, int64_t first, int64_t count);
int  orc_diagnostics(orc_handle *h, sparc_diag *out);
int  orc_derivative(orc_handle *h, int dir, int bc, const double *in,
                    double *out);
int  orc_filter_field(orc_handle *h, int dir, const double *in,
                      double *out);
int  orc_get_coeff(orc_handle *h, const char *name, double *out,
                   int64_t *count);
int  orc_get_scalars(orc_handle *h, double *out12);
/* forcing_p of iteration nn (nx*ny*nz) */
int  orc_forcing(orc_handle *h, int64_t nn, double *out);
/* one RHS evaluation (MP_QUIET_3D / MP_MHD_3D) of stage fields temp
 * (V*N) and stage CPML fields psi, with the forcing of iteration nn;
 * writes scr (V*N) and the CPML right-hand sides scr_psi */
int  orc_rhs(orc_handle *h, int64_t nn, const double *temp,
             const double *psi, double *scr, double *scr_psi);
void orc_set_threads(int n);
int  orc_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
