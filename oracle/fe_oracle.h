/* fe_oracle.h -- TEST INFRASTRUCTURE ONLY: serial FP64 CPU restatement of the FastEddy
 * hot path (one BuildFrhs tendency evaluation + the WS2002 RK3 stage commit).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference legs may
 * load this; the product path never does. It is the checker, not the thing measured.
 * See fe_oracle.c for the reference file:line each routine restates.
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H

#include "fasteddy_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_domain ora_domain;

int ora_create(const fe_config *cfg, ora_domain **out);
void ora_destroy(ora_domain *o);
int ora_set_grid(ora_domain *o, const float *zPos, const float *J31, const float *J32, const float *J33,
                 const float *D_Jac, const float *invD_Jac);
int ora_set_base_state(ora_domain *o, const float *baseStateFlds);
int ora_set_state(ora_domain *o, const float *hydroFlds, const float *sgstke, const float *moist);
int ora_set_state_f64(ora_domain *o, const double *hydroFlds, const double *sgstke, const double *moist);
int ora_set_surface(ora_domain *o, const float *z0m, const float *z0t, const float *htFlux, const float *tskin,
                    const float *fricVel, const float *qFlux, const float *qskin);
int ora_set_clock(ora_domain *o, double simTime, int simTime_it);
/* Slab of a decomposed domain: x (y) halo columns are written by the caller before each
 * stage instead of being periodic images. */
int ora_set_decomposition(ora_domain *o, int peerX, int peerY);
/* Tendency of RK stage `stage` (0..2) from the current state (updates the stateful
 * surface-layer arrays on the last stage exactly as the device path does). */
int ora_build_frhs(ora_domain *o, int stage);
/* One RK stage: build_frhs + commit. */
int ora_rk_stage(ora_domain *o, int stage);
/* nsteps full RK3 steps, advancing the clock. */
int ora_step(ora_domain *o, int nsteps);
int ora_get_state(ora_domain *o, double *hydroFlds, double *sgstke, double *moist, double *pres);
int ora_get_frhs(ora_domain *o, double *hydroFrhs, double *sgstkeFrhs, double *moistFrhs, double *taus);
int ora_get_surface(ora_domain *o, double *cd, double *ch, double *fricVel, double *htFlux, double *invOblen,
                    double *tskin, double *qFlux, double *qskin);

#ifdef __cplusplus
}
#endif
#endif
