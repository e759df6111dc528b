/* fe_refabi.c -- the reference-named drop-in entry points (fasteddy_b200.h section A).
 *
 * The FastEddy driver (reference SRC/FEMAIN/FastEddy.c) calls its CUDA layer through
 * argument-less wrappers that read global host symbols. These functions keep those
 * names, signatures, call order and global-symbol contract, and run the B200 engine
 * underneath:
 *   fecuda_Init                 -> device = mpi_rank_world % device count (fecuda_Device.cu:59)
 *   cuda_gridInit               -> engine domain from the physics globals + grid upload
 *   cuda_hydroCoreInit          -> base-state upload
 *   cuda_timeIntInit            -> prognostic state, surface arrays and clock upload
 *   cuda_timeIntCommence(it)    -> NtBatch RK3 steps, then state/pressure/surface copied back
 *                                  to the host globals (cuda_timeIntDevice.cu:105-157, :198-257),
 *                                  with the last stage's tendencies when hydroForcingWrite or
 *                                  hydroForcingLog is set and the SGS stresses and moisture SGS
 *                                  fluxes when hydroSubGridWrite is set (:210-251)
 * Differences from the reference: errors are returned (never exit()); hydroPres returned
 * after a batch is the perturbation pressure of the returned state (the reference returns
 * the one of the last stage's input).
 */
#include <stdio.h>

#include "fasteddy_b200.h"
#include "fe_refglobals.h"

static fe_domain *g_dom = NULL;
static int g_device = 0;
static float *g_pinned[4] = {NULL, NULL, NULL, NULL};

/* Page-lock the host state arrays the batch copies move (undone at cleanup). */
static void pin_host_state(void) {
  size_t n = (size_t)(Nxp + 2 * Nh) * (Nyp + 2 * Nh) * (Nzp + 2 * Nh);
  float *bufs[4] = {hydroFlds, hydroPres, TKESelector > 0 ? sgstkeScalars : NULL, moistureSelector > 0 ? moistScalars : NULL};
  size_t nf[4] = {5, 1, (size_t)TKESelector, (size_t)moistureNvars};
  int b;
  for (b = 0; b < 4; b++) {
    if (g_pinned[b] == bufs[b]) continue;
    if (g_pinned[b]) fe_host_unregister(g_pinned[b]);
    g_pinned[b] = NULL;
    if (bufs[b] && nf[b] > 0 && fe_host_register(bufs[b], n * nf[b] * sizeof(float)) == FE_OK) g_pinned[b] = bufs[b];
  }
}

static void unpin_host_state(void) {
  int b;
  for (b = 0; b < 4; b++) {
    if (g_pinned[b]) fe_host_unregister(g_pinned[b]);
    g_pinned[b] = NULL;
  }
}

static void fill_config(fe_config *c) {
  fe_config_defaults(c);
  c->Nx = Nxp; c->Ny = Nyp; c->Nz = Nzp; c->Nh = Nh;
  c->dX = dX; c->dY = dY; c->dZ = dZ;
  c->dt = dt;
  c->simTime_itRestart = simTime_itRestart;
  c->hydroBCs = hydroBCs;
  c->pgfSelector = pgfSelector; c->buoyancySelector = buoyancySelector; c->coriolisSelector = coriolisSelector;
  c->turbulenceSelector = turbulenceSelector; c->TKESelector = TKESelector; c->TKEAdvSelector = TKEAdvSelector;
  c->TKEAdvSelector_b_hyb = TKEAdvSelector_b_hyb; c->c_s = c_s; c->c_k = c_k;
  c->advectionSelector = advectionSelector; c->b_hyb = b_hyb;
  c->diffusionSelector = diffusionSelector; c->filterSelector = filterSelector; c->lsfSelector = lsfSelector;
  c->filter_6th_coeff = filter_6th_coeff;
  c->lsf_horMnSubTerms = lsf_horMnSubTerms; c->lsf_freq = lsf_freq;
  c->lsf_w_surf = lsf_w_surf; c->lsf_w_lev1 = lsf_w_lev1; c->lsf_w_lev2 = lsf_w_lev2;
  c->lsf_w_zlev1 = lsf_w_zlev1; c->lsf_w_zlev2 = lsf_w_zlev2;
  c->lsf_th_surf = lsf_th_surf; c->lsf_th_lev1 = lsf_th_lev1; c->lsf_th_lev2 = lsf_th_lev2;
  c->lsf_th_zlev1 = lsf_th_zlev1; c->lsf_th_zlev2 = lsf_th_zlev2;
  c->lsf_qv_surf = lsf_qv_surf; c->lsf_qv_lev1 = lsf_qv_lev1; c->lsf_qv_lev2 = lsf_qv_lev2;
  c->lsf_qv_zlev1 = lsf_qv_zlev1; c->lsf_qv_zlev2 = lsf_qv_zlev2;
  c->surflayerSelector = surflayerSelector;
  c->surflayer_z0 = surflayer_z0; c->surflayer_z0t = surflayer_z0t; c->surflayer_wth = surflayer_wth;
  c->surflayer_tr = surflayer_tr; c->surflayer_wq = surflayer_wq; c->surflayer_qr = surflayer_qr;
  c->surflayer_qskin_input = surflayer_qskin_input; c->surflayer_stab = surflayer_stab;
  c->surflayer_idealsine = surflayer_idealsine;
  c->surflayer_ideal_ts = surflayer_ideal_ts; c->surflayer_ideal_te = surflayer_ideal_te;
  c->surflayer_ideal_amp = surflayer_ideal_amp; c->surflayer_ideal_qts = surflayer_ideal_qts;
  c->surflayer_ideal_qte = surflayer_ideal_qte; c->surflayer_ideal_qamp = surflayer_ideal_qamp;
  c->moistureSelector = moistureSelector; c->moistureNvars = moistureNvars;
  c->moistureAdvSelectorQv = moistureAdvSelectorQv; c->moistureAdvSelectorQv_b = moistureAdvSelectorQv_b;
  c->moistureAdvSelectorQi = moistureAdvSelectorQi; c->moistureSGSturb = moistureSGSturb;
  c->moistureCond = moistureCond; c->moistureCondTscale = moistureCondTscale;
  c->moistureCondBasePres = moistureCondBasePres; c->moistureMPcallTscale = moistureMPcallTscale;
  c->dampingLayerSelector = dampingLayerSelector; c->dampingLayerDepth = dampingLayerDepth;
  c->U_g = U_g; c->V_g = V_g; c->z_Ug = z_Ug; c->z_Vg = z_Vg; c->Ug_grad = Ug_grad; c->Vg_grad = Vg_grad;
  c->physics_oneRKonly = physics_oneRKonly;
  c->temp_grnd = temp_grnd; c->pres_grnd = pres_grnd;
  /* constants come from the host module, not re-derived (hydro_core.c:941-967) */
  c->R_gas = R_gas; c->R_vapor = R_vapor; c->Rv_Rg = Rv_Rg; c->cp_gas = cp_gas; c->cv_gas = cv_gas;
  c->accel_g = accel_g; c->R_cp = R_cp; c->cp_R = cp_R; c->cp_cv = cp_cv; c->refPressure = refPressure;
  c->kappa = kappa; c->L_v = L_v;
  c->corioConstHorz = corioConstHorz; c->corioConstVert = corioConstVert; c->corioLS_fact = corioLS_fact;
}

/* The reference's parameter reader, when the program that loads this library links it (the
 * FastEddy driver does); absent in programs built on the repository's own host layer. */
extern int queryIntegerParameter(char *name, int *var, int min, int max, int reqStatus) __attribute__((weak));

int fecuda_GetParams(void) {
  /* tBx, tBy, tBz stay mandatory keys of the parameter file (fecuda.c:38-47); the engine picks
   * its own launch shapes, so the values are only read (2 = the reference's PARAM_MANDATORY) */
  static int tbx, tby, tbz;
  int rc = 0;
  if (!queryIntegerParameter) return FE_OK;
  rc |= queryIntegerParameter("tBx", &tbx, 1, 2147483647, 2);
  rc |= queryIntegerParameter("tBy", &tby, 1, 2147483647, 2);
  rc |= queryIntegerParameter("tBz", &tbz, 1, 2147483647, 2);
  return rc ? FE_ERR_CONFIG : FE_OK;
}

int fecuda_Init(void) {
  int n = fe_device_count();
  if (n <= 0) return FE_ERR_NO_DEVICE;
  g_device = mpi_rank_world % n;
  return FE_OK;
}

int fecuda_SetBlocksPerGrid(int nx, int ny, int nz) {
  (void)nx; (void)ny; (void)nz;
  return FE_OK;
}

int fecuda_AllocateHaloBuffers(int nxp, int nyp, int nzp, int nh) {
  (void)nxp; (void)nyp; (void)nzp; (void)nh;
  return FE_OK;
}

int fecuda_DeallocateHaloBuffers(void) { return FE_OK; }
int fecuda_Cleanup(void) { return FE_OK; }

int cuda_gridInit(void) {
  fe_config c;
  int rc;
  if (numProcsX != 1 || numProcsY != 1) return FE_ERR_CONFIG;
  if (g_dom) {
    fe_destroy(g_dom);
    g_dom = NULL;
  }
  fill_config(&c);
  rc = fe_create(&c, g_device, &g_dom);
  if (rc) return rc;
  /* the batch copy-back of the tendencies needs the last stage's tendencies kept */
  rc = fe_set_forcing_capture(g_dom, hydroForcingWrite == 1 || hydroForcingLog == 1);
  if (rc) return rc;
  return fe_set_grid(g_dom, zPos, J31, J32, J33, D_Jac, invD_Jac);
}

int cuda_gridCleanup(void) { return FE_OK; }

int cuda_hydroCoreInit(void) {
  if (!g_dom) return FE_ERR_STATE;
  return fe_set_base_state(g_dom, hydroBaseStateFlds);
}

int cuda_hydroCoreCleanup(void) {
  int rc = FE_OK;
  unpin_host_state();
  if (g_dom) rc = fe_destroy(g_dom);
  g_dom = NULL;
  return rc;
}

int cuda_timeIntHydroInitDevice(void) {
  int rc;
  if (!g_dom) return FE_ERR_STATE;
  rc = fe_set_state(g_dom, hydroFlds, TKESelector > 0 && turbulenceSelector > 0 ? sgstkeScalars : NULL,
                    moistureSelector > 0 ? moistScalars : NULL);
  if (!rc && surflayerSelector > 0)
    rc = fe_set_surface(g_dom, z0m, z0t, htFlux, tskin, fricVel, moistureSelector > 0 ? qFlux : NULL,
                        moistureSelector > 0 ? qskin : NULL);
  if (!rc) rc = fe_set_clock(g_dom, simTime, simTime_it);
  return rc;
}

int cuda_timeIntHydroSynchFromDevice(void) {
  int rc;
  if (!g_dom) return FE_ERR_STATE;
  rc = fe_get_state(g_dom, hydroFlds, TKESelector > 0 ? sgstkeScalars : NULL, moistureSelector > 0 ? moistScalars : NULL,
                    hydroPres);
  if (!rc && surflayerSelector > 0)
    rc = fe_get_surface(g_dom, NULL, NULL, fricVel, htFlux, invOblen, tskin, moistureSelector > 0 ? qFlux : NULL,
                        moistureSelector > 0 ? qskin : NULL);
  /* the last stage's tendencies (kept by the engine for the last step of the batch) */
  if (!rc && (hydroForcingWrite == 1 || hydroForcingLog == 1))
    rc = fe_get_frhs(g_dom, hydroFldsFrhs, TKESelector > 0 ? sgstkeScalarsFrhs : NULL,
                     moistureSelector > 0 ? moistScalarsFrhs : NULL, NULL);
  /* SGS stresses and heat fluxes; moisture SGS fluxes (allocated on the host only in this case,
   * hydro_core.c:897-898) */
  if (!rc && hydroSubGridWrite == 1 && turbulenceSelector > 0)
    rc = fe_get_sgs_fluxes(g_dom, hydroTauFlds,
                           (moistureSGSturb == 1 && moistureSelector > 0) ? moistTauFlds : NULL);
  return rc;
}

int cuda_timeIntInit(void) {
  pin_host_state();
  return cuda_timeIntHydroInitDevice();
}

int cuda_timeIntCleanup(void) { return FE_OK; }

int cuda_timeIntCommence(int it) {
  int rc, s;
  long long bad = 0;
  if (!g_dom) return FE_ERR_STATE;
  if (it == simTime_itRestart) {
    rc = cuda_timeIntHydroInitDevice();
    if (rc) return rc;
  }
  rc = fe_advance(g_dom, NtBatch);
  if (!rc) rc = fe_sync(g_dom);
  if (rc) return rc;
  for (s = 0; s < NtBatch; s++) {
    simTime = simTime + dt;
    simTime_it = simTime_it + 1;
  }
  rc = cuda_timeIntHydroSynchFromDevice();
  if (rc) return rc;
  if (fe_count_nonfinite(g_dom, &bad) == FE_OK && bad > 0) return FE_ERR_NONFINITE;
  return FE_OK;
}

int cuda_hydroCoreDeviceBuildFrhs(float st, int st_it, int st_itRestart, float dtt, int timeStage, int nstages) {
  int rc;
  (void)st_itRestart; (void)dtt; (void)nstages;
  if (!g_dom) return FE_ERR_STATE;
  rc = fe_set_clock(g_dom, st, st_it);
  if (!rc) rc = fe_build_frhs(g_dom, timeStage);
  if (!rc)
    rc = fe_get_frhs(g_dom, hydroFldsFrhs, TKESelector > 0 ? sgstkeScalarsFrhs : NULL,
                     moistureSelector > 0 ? moistScalarsFrhs : NULL, hydroSubGridWrite == 1 ? hydroTauFlds : NULL);
  return rc;
}

/* Handle of the domain the drop-in entry points manage (for callers that mix both APIs). */
fe_domain *fe_refabi_domain(void) { return g_dom; }

/* Engine configuration assembled from the FastEddy globals (what cuda_gridInit uses). */
void fe_refabi_fill_config(fe_config *c) { fill_config(c); }
