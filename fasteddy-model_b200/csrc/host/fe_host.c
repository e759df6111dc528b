/* fe_host.c -- host C layer: parameters, grid and metrics, FP64 hydrostatic base state,
 * seeded initial conditions and surface-layer initialisation.
 *
 * This is the repository's own replacement of the reference's host modules for the
 * inputs of the hot path. It defines the global host symbols of fe_refglobals.h (the
 * names are fixed by the drop-in ABI) and fills them the way the reference's
 * FastEddy.c:72-280 initialisation sequence does:
 *   fe_host_load_params_*  ~ *GetParams of every module (hydro_core.c:197-395,
 *                            grid.c:68-88, time_integration.c:51-64, fempi.c:80-94,
 *                            fecuda.c:35-44, io.c:65-77)
 *   fe_host_init           ~ gridInit + hydro_coreInit + timeInit + gridSecondaryPreparations
 *                            + hydro_coreSetBaseState
 * Differences by design:
 *   - the base state is integrated entirely in FP64 and rounded once to float
 *     (the reference mixes float storage and double pow, hydro_core.c:1053-1190);
 *   - theta perturbations come from a seeded splitmix64 stream, not rand();
 *   - single rank only (numProcsX = numProcsY = 1): the hot path is single-GPU;
 *   - nothing calls exit(); errors are return codes.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <float.h>

#include "fe_params.h"
#include "fe_refglobals.h"
#include "fe_host.h"

/* ------------------------------------------------------------------ global symbols */
int mpi_size_world = 1, mpi_rank_world = 0;
int numProcsX = 1, numProcsY = 1;
int Nxp, Nyp, Nzp;
int Nh;
int Nx, Ny, Nz;
int iMin, iMax, jMin, jMax, kMin, kMax;
float dX, dY, dZ, dXi, dYi, dZi;
float *xPos, *yPos, *zPos, *topoPos;
float *J31, *J32, *J33, *D_Jac, *invD_Jac;
int tBx = 1, tBy = 4, tBz = 64;
int Nhydro = 5, hydroBCs;
int hydroForcingWrite, hydroForcingLog, hydroSubGridWrite;
float *hydroFlds, *hydroFldsFrhs, *hydroBaseStateFlds, *hydroPres, *hydroBaseStatePres;
float *hydroTauFlds;
float R_gas, R_vapor, Rv_Rg, cp_gas, cv_gas, accel_g, R_cp, cp_R, cp_cv, refPressure, kappa, L_v;
int pgfSelector, buoyancySelector, coriolisSelector;
float coriolisLatitude, corioConstHorz, corioConstVert, corioLS_fact;
int turbulenceSelector, TKESelector, TKEAdvSelector;
float TKEAdvSelector_b_hyb, c_s, c_k;
float *sgstkeScalars, *sgstkeScalarsFrhs;
int diffusionSelector;
int advectionSelector;
float b_hyb;
int surflayerSelector;
float surflayer_z0, surflayer_z0t, surflayer_wth, surflayer_tr, surflayer_wq, surflayer_qr;
int surflayer_qskin_input, surflayer_stab;
float *fricVel, *htFlux, *tskin, *invOblen, *z0m, *z0t, *qFlux, *qskin;
int surflayer_idealsine;
float surflayer_ideal_ts, surflayer_ideal_te, surflayer_ideal_amp;
float surflayer_ideal_qts, surflayer_ideal_qte, surflayer_ideal_qamp;
int lsfSelector;
int lsf_horMnSubTerms;
float lsf_freq;
float lsf_w_surf, lsf_w_lev1, lsf_w_lev2, lsf_w_zlev1, lsf_w_zlev2;
float lsf_th_surf, lsf_th_lev1, lsf_th_lev2, lsf_th_zlev1, lsf_th_zlev2;
float lsf_qv_surf, lsf_qv_lev1, lsf_qv_lev2, lsf_qv_zlev1, lsf_qv_zlev2;
int moistureSelector, moistureNvars, moistureAdvSelectorQv;
float moistureAdvSelectorQv_b;
int moistureSGSturb, moistureCond;
float *moistScalars, *moistScalarsFrhs, *moistTauFlds;
int moistureAdvSelectorQi;
float moistureCondTscale;
int moistureCondBasePres;
float moistureMPcallTscale;
int filterSelector;
float filter_6th_coeff;
int dampingLayerSelector;
float dampingLayerDepth;
float temp_grnd, pres_grnd;
float U_g, V_g, z_Ug, z_Vg, Ug_grad, Vg_grad;
int physics_oneRKonly;
int timeMethod, Nt, NtBatch;
float dt;
float simTime;
int simTime_it, simTime_itRestart, numRKstages;

/* host-only parameters (not read by the CUDA layer) */
static int coordHorizHalos, verticalDeformSwitch;
static float verticalDeformFactor, verticalDeformQuadCoeff;
static int stabilityScheme;
static float zStableBottom, stableGradient, zStableBottom2, stableGradient2, zStableBottom3, stableGradient3;
static int thetaPerturbationSwitch;
static float thetaHeight, thetaAmplitude;
static float nu_0;
static char g_topoFile[1024];
static char g_inFile[1024];
static char g_inPath[1024];
static int ioOutputMode, frqOutput;
static char g_msg[512];
static char g_outPath[1024], g_outFileBase[256];
static double *g_topoGlobal; /* Nx*Ny, i-major, set by fe_host_set_topography */

const char *fe_host_last_message(void) { return g_msg[0] ? g_msg : fe_params_last_message(); }

#define Q(rc_, call_) do { int r__ = (call_); if (r__ != FE_PARAM_OK && r__ != FE_PARAM_WARN_DEFAULTED) rc_ = r__; } while (0)

static int query_all(void) {
  int rc = 0;
  const char *s;
  /* Description (FastEddy.c:84) */
  Q(rc, fe_params_query_string("Description", &s, FE_PARAM_MANDATORY));
  /* FEMPI (fempi.c:80-94): this build is single-GPU */
  numProcsX = 1; numProcsY = 1;
  Q(rc, fe_params_query_int("numProcsX", &numProcsX, 1, 1, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("numProcsY", &numProcsY, 1, 1, FE_PARAM_MANDATORY));
  /* IO (io.c:65-77): accepted, output is not part of the hot path */
  ioOutputMode = 0;
  Q(rc, fe_params_query_int("ioOutputMode", &ioOutputMode, 0, 1, FE_PARAM_OPTIONAL));
  g_inPath[0] = 0;
  Q(rc, fe_params_query_string("inPath", &s, FE_PARAM_OPTIONAL));
  if (s) snprintf(g_inPath, sizeof(g_inPath), "%s", s);
  g_inFile[0] = 0;
  Q(rc, fe_params_query_string("inFile", &s, FE_PARAM_OPTIONAL));
  if (s) snprintf(g_inFile, sizeof(g_inFile), "%s", s);
  g_outPath[0] = g_outFileBase[0] = 0;
  Q(rc, fe_params_query_string("outPath", &s, FE_PARAM_MANDATORY));
  if (s) snprintf(g_outPath, sizeof(g_outPath), "%s", s);
  Q(rc, fe_params_query_string("outFileBase", &s, FE_PARAM_MANDATORY));
  if (s) snprintf(g_outFileBase, sizeof(g_outFileBase), "%s", s);
  Q(rc, fe_params_query_int("frqOutput", &frqOutput, 0, INT_MAX, FE_PARAM_MANDATORY));
  /* FECUDA (fecuda.c:35-44) */
  Q(rc, fe_params_query_int("tBx", &tBx, 1, INT_MAX, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("tBy", &tBy, 1, INT_MAX, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("tBz", &tBz, 1, INT_MAX, FE_PARAM_MANDATORY));
  /* GRID (grid.c:68-88) */
  Q(rc, fe_params_query_string("gridFile", &s, FE_PARAM_OPTIONAL));
  g_topoFile[0] = 0;
  Q(rc, fe_params_query_string("topoFile", &s, FE_PARAM_OPTIONAL));
  if (s) snprintf(g_topoFile, sizeof(g_topoFile), "%s", s);
  Q(rc, fe_params_query_int("Nx", &Nx, 1, INT_MAX, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("Ny", &Ny, 1, INT_MAX, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("Nz", &Nz, 1, INT_MAX, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("Nh", &Nh, 0, INT_MAX, FE_PARAM_MANDATORY));
  {
    float dxi = 0, deta = 0, dzeta = 0;
    Q(rc, fe_params_query_float("d_xi", &dxi, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("d_eta", &deta, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("d_zeta", &dzeta, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
    dX = dxi; dY = deta; dZ = dzeta;
  }
  Q(rc, fe_params_query_int("coordHorizHalos", &coordHorizHalos, 0, 1, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_int("verticalDeformSwitch", &verticalDeformSwitch, 0, 1, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_float("verticalDeformFactor", &verticalDeformFactor, 0.0f, 1.0f, FE_PARAM_MANDATORY));
  Q(rc, fe_params_query_float("verticalDeformQuadCoeff", &verticalDeformQuadCoeff, -2.0f, 2.0f, FE_PARAM_MANDATORY));
  /* TIME_INTEGRATION (time_integration.c:51-64) */
  timeMethod = 0;
  Q(rc, fe_params_query_int("timeMethod", &timeMethod, 0, 0, FE_PARAM_MANDATORY));
  Nt = 1000;
  Q(rc, fe_params_query_int("Nt", &Nt, 1, INT_MAX, FE_PARAM_MANDATORY));
  dt = 1.0f;
  Q(rc, fe_params_query_float("dt", &dt, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  NtBatch = 1;
  Q(rc, fe_params_query_int("NtBatch", &NtBatch, 1, Nt, FE_PARAM_MANDATORY));
  /* HYDRO_CORE (hydro_core.c:197-395): same keys, defaults, ranges and status */
  hydroBCs = 0;
  Q(rc, fe_params_query_int("hydroBCs", &hydroBCs, 2, 2, FE_PARAM_MANDATORY));
  hydroForcingWrite = 0;
  Q(rc, fe_params_query_int("hydroForcingWrite", &hydroForcingWrite, 0, 1, FE_PARAM_MANDATORY));
  hydroForcingLog = 0;
  Q(rc, fe_params_query_int("hydroForcingLog", &hydroForcingLog, 0, 1, FE_PARAM_MANDATORY));
  hydroSubGridWrite = 0;
  Q(rc, fe_params_query_int("hydroSubGridWrite", &hydroSubGridWrite, 0, 1, FE_PARAM_MANDATORY));
  pgfSelector = 1;
  Q(rc, fe_params_query_int("pgfSelector", &pgfSelector, 0, 1, FE_PARAM_OPTIONAL));
  buoyancySelector = 1;
  Q(rc, fe_params_query_int("buoyancySelector", &buoyancySelector, 0, 1, FE_PARAM_OPTIONAL));
  coriolisSelector = 0;
  Q(rc, fe_params_query_int("coriolisSelector", &coriolisSelector, 0, 2, FE_PARAM_MANDATORY));
  coriolisLatitude = 54.0f;
  Q(rc, fe_params_query_float("coriolisLatitude", &coriolisLatitude, -90.0f, 90.0f, FE_PARAM_MANDATORY));
  turbulenceSelector = 0;
  Q(rc, fe_params_query_int("turbulenceSelector", &turbulenceSelector, 0, 1, FE_PARAM_MANDATORY));
  TKESelector = 0;
  Q(rc, fe_params_query_int("TKESelector", &TKESelector, 0, 1, FE_PARAM_MANDATORY));
  TKEAdvSelector = 0;
  Q(rc, fe_params_query_int("TKEAdvSelector", &TKEAdvSelector, 0, 6, FE_PARAM_MANDATORY));
  TKEAdvSelector_b_hyb = 0.0f;
  Q(rc, fe_params_query_float("TKEAdvSelector_b_hyb", &TKEAdvSelector_b_hyb, 0.0f, 1.0f, FE_PARAM_MANDATORY));
  c_s = 0.18f;
  Q(rc, fe_params_query_float("c_s", &c_s, 1e-6f, 1e6f, FE_PARAM_MANDATORY));
  c_k = 0.10f;
  Q(rc, fe_params_query_float("c_k", &c_k, 1e-6f, 1e6f, FE_PARAM_MANDATORY));
  advectionSelector = 0;
  Q(rc, fe_params_query_int("advectionSelector", &advectionSelector, 0, 6, FE_PARAM_MANDATORY));
  b_hyb = 0.8f;
  Q(rc, fe_params_query_float("b_hyb", &b_hyb, 0.0f, 1.0f, FE_PARAM_MANDATORY));
  diffusionSelector = 0;
  Q(rc, fe_params_query_int("diffusionSelector", &diffusionSelector, 0, 1, FE_PARAM_MANDATORY));
  nu_0 = 1.0f;
  Q(rc, fe_params_query_float("nu_0", &nu_0, 0.0f, FLT_MAX, FE_PARAM_MANDATORY));
  surflayerSelector = 0;
  Q(rc, fe_params_query_int("surflayerSelector", &surflayerSelector, 0, 2, FE_PARAM_MANDATORY));
  surflayer_z0 = 0.1f;
  Q(rc, fe_params_query_float("surflayer_z0", &surflayer_z0, 1e-6f, 1e+0f, FE_PARAM_MANDATORY));
  surflayer_z0t = 0.1f;
  Q(rc, fe_params_query_float("surflayer_z0t", &surflayer_z0t, 1e-6f, 1e+1f, FE_PARAM_MANDATORY));
  surflayer_tr = 0.0f;
  Q(rc, fe_params_query_float("surflayer_tr", &surflayer_tr, -1e+1f, 1e+1f, FE_PARAM_MANDATORY));
  surflayer_wth = 0.0f;
  Q(rc, fe_params_query_float("surflayer_wth", &surflayer_wth, -5e+0f, 5e+0f, FE_PARAM_MANDATORY));
  surflayer_idealsine = 0;
  Q(rc, fe_params_query_int("surflayer_idealsine", &surflayer_idealsine, 0, 1, FE_PARAM_MANDATORY));
  surflayer_ideal_ts = 0.0f; surflayer_ideal_te = 0.0f; surflayer_ideal_amp = 0.1f;
  if (surflayer_idealsine > 0) {
    Q(rc, fe_params_query_float("surflayer_ideal_ts", &surflayer_ideal_ts, 0, 1e+5f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("surflayer_ideal_te", &surflayer_ideal_te, 0, 1e+5f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("surflayer_ideal_amp", &surflayer_ideal_amp, 0, 1e+3f, FE_PARAM_MANDATORY));
  }
  surflayer_wq = 0.0f; surflayer_qr = 0.0f; surflayer_qskin_input = 0;
  surflayer_ideal_qts = 0.0f; surflayer_ideal_qte = 0.0f; surflayer_ideal_qamp = 0.1f;
  surflayer_stab = 0;
  Q(rc, fe_params_query_int("surflayer_stab", &surflayer_stab, 0, 1, FE_PARAM_OPTIONAL));
  lsfSelector = 0;
  Q(rc, fe_params_query_int("lsfSelector", &lsfSelector, 0, 1, FE_PARAM_MANDATORY));
  /* large-scale forcing: defaults, then the keys read under lsfSelector > 0 (hydro_core.c:267-311) */
  lsf_w_surf = lsf_w_lev1 = lsf_w_lev2 = 0.0f; lsf_w_zlev1 = 100.0f; lsf_w_zlev2 = 200.0f;
  lsf_th_surf = lsf_th_lev1 = lsf_th_lev2 = 0.0f; lsf_th_zlev1 = 100.0f; lsf_th_zlev2 = 200.0f;
  lsf_qv_surf = lsf_qv_lev1 = lsf_qv_lev2 = 0.0f; lsf_qv_zlev1 = 100.0f; lsf_qv_zlev2 = 200.0f;
  lsf_horMnSubTerms = 0;
  lsf_freq = 1.0f;
  if (lsfSelector > 0) {
    Q(rc, fe_params_query_float("lsf_w_surf", &lsf_w_surf, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_w_lev1", &lsf_w_lev1, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_w_lev2", &lsf_w_lev2, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_w_zlev1", &lsf_w_zlev1, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_w_zlev2", &lsf_w_zlev2, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_th_surf", &lsf_th_surf, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_th_lev1", &lsf_th_lev1, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_th_lev2", &lsf_th_lev2, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_th_zlev1", &lsf_th_zlev1, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_th_zlev2", &lsf_th_zlev2, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_qv_surf", &lsf_qv_surf, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_qv_lev1", &lsf_qv_lev1, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_qv_lev2", &lsf_qv_lev2, -1e+4f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_qv_zlev1", &lsf_qv_zlev1, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_qv_zlev2", &lsf_qv_zlev2, 0.0f, 1e+4f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("lsf_horMnSubTerms", &lsf_horMnSubTerms, 0, 1, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("lsf_freq", &lsf_freq, 1e-3f, 1e+3f, FE_PARAM_MANDATORY));
  }
  moistureSelector = 0;
  Q(rc, fe_params_query_int("moistureSelector", &moistureSelector, 0, 1, FE_PARAM_MANDATORY));
  moistureNvars = 0; moistureAdvSelectorQv = 0; moistureAdvSelectorQv_b = 0.0f;
  moistureAdvSelectorQi = 0; moistureSGSturb = 0; moistureCond = 1;
  moistureCondTscale = 1.0f; moistureCondBasePres = 0; moistureMPcallTscale = 1.0f;
  if (moistureSelector > 0) {
    Q(rc, fe_params_query_int("moistureNvars", &moistureNvars, 0, 2, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("moistureAdvSelectorQv", &moistureAdvSelectorQv, 0, 6, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("moistureAdvSelectorQv_b", &moistureAdvSelectorQv_b, 0.0f, 1.0f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("moistureAdvSelectorQi", &moistureAdvSelectorQi, 0, 2, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("moistureSGSturb", &moistureSGSturb, 0, 1, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("moistureCond", &moistureCond, 1, 3, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("moistureCondTscale", &moistureCondTscale, 1e-4f, 1000.0f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("moistureCondBasePres", &moistureCondBasePres, 0, 1, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("moistureMPcallTscale", &moistureMPcallTscale, 1e-4f, 1000.0f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("surflayer_wq", &surflayer_wq, -5e+0f, 5e+0f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_float("surflayer_qr", &surflayer_qr, -1e+1f, 1e+1f, FE_PARAM_MANDATORY));
    Q(rc, fe_params_query_int("surflayer_qskin_input", &surflayer_qskin_input, 0, 1, FE_PARAM_OPTIONAL));
    if (surflayer_idealsine > 0) {
      Q(rc, fe_params_query_float("surflayer_ideal_qts", &surflayer_ideal_qts, 0, 1e+5f, FE_PARAM_MANDATORY));
      Q(rc, fe_params_query_float("surflayer_ideal_qte", &surflayer_ideal_qte, 0, 1e+5f, FE_PARAM_MANDATORY));
      Q(rc, fe_params_query_float("surflayer_ideal_qamp", &surflayer_ideal_qamp, 0, 1e+3f, FE_PARAM_MANDATORY));
    }
  }
  filterSelector = 0;
  Q(rc, fe_params_query_int("filterSelector", &filterSelector, 0, 1, FE_PARAM_MANDATORY));
  filter_6th_coeff = 0.12f;
  Q(rc, fe_params_query_float("filter_6th_coeff", &filter_6th_coeff, 0.0f, 1.0f, FE_PARAM_MANDATORY));
  dampingLayerSelector = 0;
  Q(rc, fe_params_query_int("dampingLayerSelector", &dampingLayerSelector, 0, 1, FE_PARAM_MANDATORY));
  dampingLayerDepth = 100.0f;
  Q(rc, fe_params_query_float("dampingLayerDepth", &dampingLayerDepth, 0.0f, FLT_MAX, FE_PARAM_MANDATORY));
  stabilityScheme = 0;
  Q(rc, fe_params_query_int("stabilityScheme", &stabilityScheme, 0, 2, FE_PARAM_MANDATORY));
  temp_grnd = 300.0f;
  Q(rc, fe_params_query_float("temp_grnd", &temp_grnd, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  pres_grnd = 1.0e5f;
  Q(rc, fe_params_query_float("pres_grnd", &pres_grnd, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  zStableBottom = 1000.0f;
  Q(rc, fe_params_query_float("zStableBottom", &zStableBottom, 0, FLT_MAX, FE_PARAM_MANDATORY));
  stableGradient = 0.1f;
  Q(rc, fe_params_query_float("stableGradient", &stableGradient, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  zStableBottom2 = 1100.0f;
  Q(rc, fe_params_query_float("zStableBottom2", &zStableBottom2, 0, FLT_MAX, FE_PARAM_MANDATORY));
  stableGradient2 = 0.03f;
  Q(rc, fe_params_query_float("stableGradient2", &stableGradient2, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  zStableBottom3 = 1500.0f;
  Q(rc, fe_params_query_float("zStableBottom3", &zStableBottom3, 0, FLT_MAX, FE_PARAM_MANDATORY));
  stableGradient3 = 0.03f;
  Q(rc, fe_params_query_float("stableGradient3", &stableGradient3, FLT_MIN, FLT_MAX, FE_PARAM_MANDATORY));
  U_g = 0.0f;
  Q(rc, fe_params_query_float("U_g", &U_g, -FLT_MAX, FLT_MAX, FE_PARAM_MANDATORY));
  V_g = 0.0f;
  Q(rc, fe_params_query_float("V_g", &V_g, -FLT_MAX, FLT_MAX, FE_PARAM_MANDATORY));
  z_Ug = 10000.0f;
  Q(rc, fe_params_query_float("z_Ug", &z_Ug, 0.0f, FLT_MAX, FE_PARAM_MANDATORY));
  z_Vg = 10000.0f;
  Q(rc, fe_params_query_float("z_Vg", &z_Vg, 0.0f, FLT_MAX, FE_PARAM_MANDATORY));
  Ug_grad = 0.0f;
  Q(rc, fe_params_query_float("Ug_grad", &Ug_grad, -1e2f, 1e2f, FE_PARAM_MANDATORY));
  Vg_grad = 0.0f;
  Q(rc, fe_params_query_float("Vg_grad", &Vg_grad, -1e2f, 1e2f, FE_PARAM_MANDATORY));
  thetaPerturbationSwitch = 0;
  Q(rc, fe_params_query_int("thetaPerturbationSwitch", &thetaPerturbationSwitch, 0, 1, FE_PARAM_MANDATORY));
  thetaHeight = 0.0f;
  Q(rc, fe_params_query_float("thetaHeight", &thetaHeight, 0.0f, FLT_MAX, FE_PARAM_MANDATORY));
  thetaAmplitude = 0.0f;
  Q(rc, fe_params_query_float("thetaAmplitude", &thetaAmplitude, 0.0f, 2.0f, FE_PARAM_MANDATORY));
  physics_oneRKonly = 1;
  Q(rc, fe_params_query_int("physics_oneRKonly", &physics_oneRKonly, 0, 1, FE_PARAM_OPTIONAL));
  /* keys the reference reads only under lsfSelector>0 or for other subsystems are
   * accepted silently so an unmodified tutorial file parses */
  {
    static const char *accepted[] = {"lsf_horMnSubTerms", "lsf_freq", "lsf_w_surf", "lsf_w_lev1", "lsf_w_lev2",
      "lsf_w_zlev1", "lsf_w_zlev2", "lsf_th_surf", "lsf_th_lev1", "lsf_th_lev2", "lsf_th_zlev1", "lsf_th_zlev2",
      "lsf_qv_surf", "lsf_qv_lev1", "lsf_qv_lev2", "lsf_qv_zlev1", "lsf_qv_zlev2", "surflayer_ideal_ts",
      "surflayer_ideal_te", "surflayer_ideal_amp", "surflayer_ideal_qts", "surflayer_ideal_qte",
      "surflayer_ideal_qamp", "surflayer_wq", "surflayer_qr", "moistureNvars", "moistureAdvSelectorQv",
      "moistureAdvSelectorQv_b", "moistureAdvSelectorQi", "moistureSGSturb", "moistureCond",
      "moistureCondTscale", "moistureCondBasePres", "moistureMPcallTscale", NULL};
    int a;
    for (a = 0; accepted[a]; a++) (void)fe_params_query_string(accepted[a], &s, FE_PARAM_NOT_REQUIRED);
  }
  return rc;
}

static void derive_constants(void) {
  double pi = acos(-1.0);
  /* constants as hydro_core.c:941-952 and :836 */
  kappa = 0.4f;
  accel_g = 9.81f;
  R_gas = 287.04f;
  R_vapor = 461.60f;
  cv_gas = 718.0f;
  cp_gas = R_gas + cv_gas;
  L_v = 2.5e6f;
  R_cp = R_gas / cp_gas;
  cp_R = cp_gas / R_gas;
  cp_cv = cp_gas / cv_gas;
  refPressure = 1.0e5f;
  Rv_Rg = R_vapor / R_gas;
  /* Coriolis factors (hydro_core.c:955-967): 1.45842e-4 = 2*Omega_earth */
  if (coriolisSelector > 0) {
    corioConstHorz = (float)(1.45842e-4 * sin(pi / 180.0 * coriolisLatitude));
    corioConstVert = coriolisSelector > 1 ? (float)(1.45842e-4 * cos(pi / 180.0 * coriolisLatitude)) : 0.0f;
    corioLS_fact = 1.0f;
  } else {
    corioConstHorz = 0.0f;
    corioConstVert = 0.0f;
    corioLS_fact = 0.0f;
  }
}

int fe_host_load_params_file(const char *path) {
  int rc;
  free(g_topoGlobal);
  g_topoGlobal = NULL;
  fe_params_reset();
  g_msg[0] = 0;
  rc = fe_params_read_file(path);
  if (rc == FE_PARAM_ERR_FILE) return -1;
  query_all();
  derive_constants();
  return fe_params_error_count();
}

int fe_host_load_params_text(const char *text) {
  free(g_topoGlobal);
  g_topoGlobal = NULL;
  fe_params_reset();
  g_msg[0] = 0;
  fe_params_read_text(text);
  query_all();
  derive_constants();
  return fe_params_error_count();
}

int fe_host_unused_params(char *buf, int buflen) { return fe_params_report_unused(buf, buflen); }

/* ------------------------------------------------------------------ allocation */
static float *alloc_f(size_t n) {
  float *p = (float *)calloc(n ? n : 1, sizeof(float));
  return p;
}

#define FREE(p) do { free(p); (p) = NULL; } while (0)

void fe_host_cleanup(void) {
  FREE(xPos); FREE(yPos); FREE(zPos); FREE(topoPos);
  FREE(J31); FREE(J32); FREE(J33); FREE(D_Jac); FREE(invD_Jac);
  FREE(hydroFlds); FREE(hydroFldsFrhs); FREE(hydroBaseStateFlds); FREE(hydroPres); FREE(hydroBaseStatePres);
  FREE(hydroTauFlds); FREE(sgstkeScalars); FREE(sgstkeScalarsFrhs);
  FREE(moistScalars); FREE(moistScalarsFrhs); FREE(moistTauFlds);
  FREE(fricVel); FREE(htFlux); FREE(tskin); FREE(invOblen); FREE(z0m); FREE(z0t); FREE(qFlux); FREE(qskin);
}

size_t fe_host_field_elems(void) { return (size_t)(Nxp + 2 * Nh) * (size_t)(Nyp + 2 * Nh) * (size_t)(Nzp + 2 * Nh); }
size_t fe_host_plane_elems(void) { return (size_t)(Nxp + 2 * Nh) * (size_t)(Nyp + 2 * Nh); }

#define IJK(i, j, k) ((size_t)(i) * (size_t)(Nyp + 2 * Nh) * (size_t)(Nzp + 2 * Nh) + (size_t)(j) * (size_t)(Nzp + 2 * Nh) + (size_t)(k))
#define IJ(i, j) ((size_t)(i) * (size_t)(Nyp + 2 * Nh) + (size_t)(j))

/* ------------------------------------------------------------------ topography */
int fe_host_set_topography(const float *topo_ij, int nx, int ny) {
  int i, j;
  if (nx != Nx || ny != Ny) {
    snprintf(g_msg, sizeof(g_msg), "topography extents (%d,%d) != (Nx,Ny) = (%d,%d)", nx, ny, Nx, Ny);
    return -1;
  }
  free(g_topoGlobal);
  g_topoGlobal = (double *)malloc(sizeof(double) * (size_t)Nx * (size_t)Ny);
  if (!g_topoGlobal) return -1;
  for (i = 0; i < Nx; i++)
    for (j = 0; j < Ny; j++) g_topoGlobal[(size_t)i * Ny + j] = topo_ij[(size_t)i * Ny + j];
  return 0;
}

/* Gaussian hill h(r) = height * 2^(-(r/halfwidth)^2), centred in the domain; r from cell centres. */
int fe_host_gaussian_hill(float height, float halfwidth) {
  int i, j;
  float *t = alloc_f((size_t)Nx * Ny);
  double xc = 0.5 * Nx * dX, yc = 0.5 * Ny * dY;
  if (!t) return -1;
  for (i = 0; i < Nx; i++)
    for (j = 0; j < Ny; j++) {
      double x = (i + 0.5) * dX - xc, y = (j + 0.5) * dY - yc;
      double r = sqrt(x * x + y * y) / halfwidth;
      t[(size_t)i * Ny + j] = (float)(height * pow(2.0, -r * r));
    }
  i = fe_host_set_topography(t, Nx, Ny);
  free(t);
  return i;
}

/* topoFile format of the reference (grid.c:313-326): int Nx, int Ny, float[Ny][Nx]. */
int fe_host_write_topofile(const char *path) {
  FILE *f;
  int i, j;
  if (!g_topoGlobal) return -1;
  f = fopen(path, "wb");
  if (!f) return -1;
  fwrite(&Nx, sizeof(int), 1, f);
  fwrite(&Ny, sizeof(int), 1, f);
  for (j = 0; j < Ny; j++)
    for (i = 0; i < Nx; i++) {
      float v = (float)g_topoGlobal[(size_t)i * Ny + j];
      fwrite(&v, sizeof(float), 1, f);
    }
  fclose(f);
  return 0;
}

static int read_topofile(const char *path) {
  FILE *f = fopen(path, "rb");
  int tnx = 0, tny = 0, i, j, ok = 1;
  float *buf, *t;
  if (!f) {
    snprintf(g_msg, sizeof(g_msg), "cannot open topoFile %s", path);
    return -1;
  }
  if (fread(&tnx, sizeof(int), 1, f) != 1 || fread(&tny, sizeof(int), 1, f) != 1 || tnx != Nx || tny != Ny) {
    fclose(f);
    snprintf(g_msg, sizeof(g_msg), "topoFile extents (%d,%d) != (Nx,Ny)", tnx, tny);
    return -1;
  }
  buf = alloc_f((size_t)Nx * Ny);
  t = alloc_f((size_t)Nx * Ny);
  if (!buf || !t || fread(buf, sizeof(float), (size_t)Nx * Ny, f) != (size_t)Nx * Ny) ok = 0;
  fclose(f);
  if (ok) {
    for (i = 0; i < Nx; i++)
      for (j = 0; j < Ny; j++) t[(size_t)i * Ny + j] = buf[(size_t)j * Nx + i]; /* transpose as grid.c:329-333 */
    ok = fe_host_set_topography(t, Nx, Ny) == 0;
  }
  free(buf);
  free(t);
  return ok ? 0 : -1;
}

/* ------------------------------------------------------------------ grid */
/* Non-uniform vertical coordinate (grid.c:880-892), evaluated in double. */
static double z_deform(double zRect, double zGround, double zCeiling) {
  double c1 = verticalDeformFactor;
  double c2 = verticalDeformQuadCoeff * (1.0 - c1) / zCeiling;
  double c3 = (1.0 - c2 * zCeiling - c1) / (zCeiling * zCeiling);
  return (c3 * zRect * zRect * zRect + c2 * zRect * zRect + c1 * zRect) * (zCeiling - zGround) / zCeiling + zGround;
}

static void build_grid(void) {
  int i, j, k;
  double ztop = (double)Nz * dZ - 0.5 * dZ;
  /* topography with halos clamped to the domain edge (grid.c:350-375) */
  for (i = iMin - Nh; i < iMax + Nh; i++)
    for (j = jMin - Nh; j < jMax + Nh; j++) {
      int ig = i - Nh, jg = j - Nh;
      if (ig < 0) ig = 0;
      if (ig > Nx - 1) ig = Nx - 1;
      if (jg < 0) jg = 0;
      if (jg > Ny - 1) jg = Ny - 1;
      topoPos[IJ(i, j)] = g_topoGlobal ? (float)g_topoGlobal[(size_t)ig * Ny + jg] : 0.0f;
    }
  /* interior cell centres, terrain-following compression (grid.c:386-410), in the reference's
   * float arithmetic (float products, the 0.5*d literals promoting the sum to double, the
   * compression in float) so the coordinates equal the reference's bit for bit */
  {
    const float ztopf = (float)((double)((float)Nz * dZ) - 0.5 * (double)dZ);
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++) {
        const float h = topoPos[IJ(i, j)];
        for (k = kMin; k < kMax; k++) {
          float z = (float)((double)(((float)k - (float)Nh) * dZ) + 0.5 * (double)dZ);
          if (verticalDeformSwitch == 1) z = (float)z_deform(z, 0.0, ztop);
          xPos[IJK(i, j, k)] = (float)((double)((float)(i - Nh) * dX) + 0.5 * (double)dX);
          yPos[IJK(i, j, k)] = (float)((double)((float)(j - Nh) * dY) + 0.5 * (double)dY);
          zPos[IJK(i, j, k)] = z * ((ztopf - h) / ztopf) + h;
        }
      }
  }
  /* horizontal coordinate halos: x/y continue linearly, z copies the edge column
   * (single-rank result of grid.c:459-541 after the boundary-rank overrides) */
  for (i = iMin - Nh; i < iMin; i++)
    for (j = jMin; j < jMax; j++)
      for (k = kMin; k < kMax; k++) {
        xPos[IJK(i, j, k)] = xPos[IJK(iMin, j, k)] - (float)(Nh - i) * dX;
        yPos[IJK(i, j, k)] = yPos[IJK(iMin, j, k)];
        zPos[IJK(i, j, k)] = zPos[IJK(iMin, j, k)];
      }
  for (i = iMax; i < iMax + Nh; i++)
    for (j = jMin; j < jMax; j++)
      for (k = kMin; k < kMax; k++) {
        xPos[IJK(i, j, k)] = xPos[IJK(iMax - 1, j, k)] + (float)(i - iMax + 1) * dX;
        yPos[IJK(i, j, k)] = yPos[IJK(iMax - 1, j, k)];
        zPos[IJK(i, j, k)] = zPos[IJK(iMax - 1, j, k)];
      }
  for (i = iMin - Nh; i < iMax + Nh; i++)
    for (k = kMin; k < kMax; k++) {
      for (j = jMin - Nh; j < jMin; j++) {
        yPos[IJK(i, j, k)] = yPos[IJK(i, jMin, k)] - (float)(Nh - j) * dY;
        xPos[IJK(i, j, k)] = xPos[IJK(i, jMin, k)];
        zPos[IJK(i, j, k)] = zPos[IJK(i, jMin, k)];
      }
      for (j = jMax; j < jMax + Nh; j++) {
        yPos[IJK(i, j, k)] = yPos[IJK(i, jMax - 1, k)] + (float)(j - jMax + 1) * dY;
        xPos[IJK(i, j, k)] = xPos[IJK(i, jMax - 1, k)];
        zPos[IJK(i, j, k)] = zPos[IJK(i, jMax - 1, k)];
      }
    }
  /* vertical halos: linear continuation of the first/last interior spacing in float (grid.c:547-573) */
  for (i = iMin - Nh; i < iMax + Nh; i++)
    for (j = jMin - Nh; j < jMax + Nh; j++) {
      const float dzb = zPos[IJK(i, j, kMin + 1)] - zPos[IJK(i, j, kMin)];
      const float dzt = zPos[IJK(i, j, kMax - 1)] - zPos[IJK(i, j, kMax - 2 >= kMin ? kMax - 2 : kMin)];
      for (k = kMin - Nh; k < kMin; k++) {
        zPos[IJK(i, j, k)] = zPos[IJK(i, j, kMin)] - (float)(Nh - k) * dzb;
        xPos[IJK(i, j, k)] = xPos[IJK(i, j, kMin)];
        yPos[IJK(i, j, k)] = yPos[IJK(i, j, kMin)];
      }
      for (k = kMax; k < kMax + Nh; k++) {
        zPos[IJK(i, j, k)] = zPos[IJK(i, j, kMax - 1)] + (float)(k - kMax + 1) * dzt;
        xPos[IJK(i, j, k)] = xPos[IJK(i, j, kMax - 1)];
        yPos[IJK(i, j, k)] = yPos[IJK(i, j, kMax - 1)];
      }
    }
}

/* Metric terms by centred differences of the coordinates (grid.c:584-655), in the reference's
 * float arithmetic (float metric tensor and determinant, the inverse determinant divided in
 * double), so the metrics equal the reference's bit for bit. The inverse-metric entries use the
 * reference's cofactor choice. Halos copy the nearest interior value (grid.c:663-742). */
static void build_metrics(void) {
  int i, j, k, b;
  const float i2x = (float)(1.0 / (2.0 * (double)dX)), i2y = (float)(1.0 / (2.0 * (double)dY));
  const float i2z = (float)(1.0 / (2.0 * (double)dZ));
  for (i = iMin; i < iMax; i++)
    for (j = jMin; j < jMax; j++)
      for (k = kMin; k < kMax; k++) {
        const float T00 = (xPos[IJK(i + 1, j, k)] - xPos[IJK(i - 1, j, k)]) * i2x;
        const float T01 = (yPos[IJK(i + 1, j, k)] - yPos[IJK(i - 1, j, k)]) * i2x;
        const float T02 = (zPos[IJK(i + 1, j, k)] - zPos[IJK(i - 1, j, k)]) * i2x;
        const float T10 = (xPos[IJK(i, j + 1, k)] - xPos[IJK(i, j - 1, k)]) * i2y;
        const float T11 = (yPos[IJK(i, j + 1, k)] - yPos[IJK(i, j - 1, k)]) * i2y;
        const float T12 = (zPos[IJK(i, j + 1, k)] - zPos[IJK(i, j - 1, k)]) * i2y;
        const float T20 = (xPos[IJK(i, j, k + 1)] - xPos[IJK(i, j, k - 1)]) * i2z;
        const float T21 = (yPos[IJK(i, j, k + 1)] - yPos[IJK(i, j, k - 1)]) * i2z;
        const float T22 = (zPos[IJK(i, j, k + 1)] - zPos[IJK(i, j, k - 1)]) * i2z;
        float detf = (T11 * T22 - T12 * T21) * T00 - (T01 * T22 - T02 * T21) * T10 + (T01 * T12 - T02 * T11) * T20;
        float invf;
        if (fabsf(detf) < 1e-6f) detf = 1e-6f;
        invf = (float)(1.0 / (double)detf);
        D_Jac[IJK(i, j, k)] = detf;
        invD_Jac[IJK(i, j, k)] = invf;
        J31[IJK(i, j, k)] = (T10 * T21 - T11 * T20) * invf;
        J32[IJK(i, j, k)] = -(T00 * T21 - T01 * T20) * invf;
        J33[IJK(i, j, k)] = (T00 * T11 - T01 * T10) * invf;
      }
  for (b = 0; b < 6; b++) {
    int ilo = iMin - Nh, ihi = iMax + Nh, jlo = jMin - Nh, jhi = jMax + Nh, klo = kMin - Nh, khi = kMax + Nh;
    switch (b) {
      case 0: ihi = iMin; break;
      case 1: ilo = iMax; break;
      case 2: jhi = jMin; break;
      case 3: jlo = jMax; break;
      case 4: khi = kMin; break;
      default: klo = kMax; break;
    }
    for (i = ilo; i < ihi; i++)
      for (j = jlo; j < jhi; j++)
        for (k = klo; k < khi; k++) {
          int it = i, jt = j, kt = k;
          size_t d, s;
          switch (b) {
            case 0: it = iMin; break;
            case 1: it = iMax - 1; break;
            case 2: jt = jMin; break;
            case 3: jt = jMax - 1; break;
            case 4: kt = kMin; break;
            default: kt = kMax - 1; break;
          }
          d = IJK(i, j, k);
          s = IJK(it, jt, kt);
          D_Jac[d] = D_Jac[s];
          invD_Jac[d] = invD_Jac[s];
          J31[d] = J31[s];
          J32[d] = J32[s];
          J33[d] = J33[s];
        }
  }
}

/* ------------------------------------------------------------------ base state, FP64 */
/* Hydrostatic base state at height z for stabilityScheme 0/1/2 (hydro_core.c:1053-1190),
 * analytic integral of dp/dz = -g p/(R T) with theta(z) piecewise linear, all in double.
 * Returns rho, rho*theta. */
static void base_state_at(double z, double *rho, double *rhotheta) {
  double Rg = R_gas, cp = cp_gas, g = accel_g, p0 = refPressure, Rcp = (double)R_gas / cp_gas;
  double pg = pres_grnd, Tg = temp_grnd;
  double theta_g = Tg * pow(pg / p0, -Rcp);
  double th, pr, T, r, a0 = pow(pg / p0, Rcp);
  if (stabilityScheme == 0) {
    r = pg / (Rg * Tg);
    *rho = r;
    *rhotheta = r * theta_g;
    return;
  }
  if (z <= zStableBottom) {
    th = theta_g;
    pr = p0 * pow((-g / cp) * (z / theta_g) + a0, cp / Rg);
  } else if (stabilityScheme == 1 || z <= zStableBottom2) {
    th = theta_g + stableGradient * (z - zStableBottom);
    pr = p0 * pow((-g / cp) * (zStableBottom / theta_g + (1.0 / stableGradient) *
                                 log(1.0 + stableGradient * (z - zStableBottom) / theta_g)) + a0, cp / Rg);
  } else {
    double th2 = theta_g + stableGradient * ((double)zStableBottom2 - zStableBottom);
    double sum = zStableBottom / theta_g +
                 (1.0 / stableGradient) * log(1.0 + stableGradient * ((double)zStableBottom2 - zStableBottom) / theta_g);
    if (z <= zStableBottom3) {
      th = th2 + stableGradient2 * (z - zStableBottom2);
      sum += (1.0 / stableGradient2) * log(1.0 + stableGradient2 * (z - zStableBottom2) / th2);
    } else {
      double th3 = th2 + stableGradient2 * ((double)zStableBottom3 - zStableBottom2);
      sum += (1.0 / stableGradient2) * log(1.0 + stableGradient2 * ((double)zStableBottom3 - zStableBottom2) / th2);
      th = th3 + stableGradient3 * (z - zStableBottom3);
      sum += (1.0 / stableGradient3) * log(1.0 + stableGradient3 * (z - zStableBottom3) / th3);
    }
    pr = p0 * pow((-g / cp) * sum + a0, cp / Rg);
  }
  T = th * pow(pr / p0, Rcp);
  r = pr / (T * Rg);
  *rho = r;
  *rhotheta = th * r;
}

/* splitmix64: seeded, platform-independent stream for the initial perturbations */
static uint64_t g_rng;
static double rng_uniform(void) {
  uint64_t z = (g_rng += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void build_base_state_and_ics(unsigned long long seed) {
  size_t n = fe_host_field_elems();
  float *rhoBS = hydroBaseStateFlds, *thBS = hydroBaseStateFlds + n;
  float *rho = hydroFlds, *u = hydroFlds + n, *v = hydroFlds + 2 * n, *w = hydroFlds + 3 * n, *th = hydroFlds + 4 * n;
  double c1 = (double)R_gas / pow((double)refPressure, (double)R_gas / cp_gas);
  int i, j, k;
  for (i = iMin - Nh; i < iMax + Nh; i++)
    for (j = jMin - Nh; j < jMax + Nh; j++)
      for (k = kMin - Nh; k < kMax + Nh; k++) {
        size_t ijk = IJK(i, j, k);
        double r, rt;
        base_state_at(zPos[ijk], &r, &rt);
        rhoBS[ijk] = (float)r;
        thBS[ijk] = (float)rt;
        hydroBaseStatePres[ijk] = (float)pow(rt * c1, (double)cp_gas / cv_gas);
      }
  /* geostrophic momentum, w = 0 (hydro_core.c:1193-1214: k from kMin) */
  for (i = iMin - Nh; i < iMax + Nh; i++)
    for (j = jMin - Nh; j < jMax + Nh; j++)
      for (k = kMin; k < kMax + Nh; k++) {
        size_t ijk = IJK(i, j, k);
        double z = zPos[ijk];
        u[ijk] = (float)((z < z_Ug ? (double)U_g : U_g + (double)Ug_grad * (z - z_Ug)) * rhoBS[ijk]);
        v[ijk] = (float)((z < z_Vg ? (double)V_g : V_g + (double)Vg_grad * (z - z_Vg)) * rhoBS[ijk]);
        w[ijk] = 0.0f;
      }
  for (i = 0; i < (int)n; i++) {
    rho[i] = rhoBS[i];
    th[i] = thBS[i];
  }
  /* theta perturbations over interior cells below thetaHeight, i-j-k order (hydro_core.c:1237-1250) */
  if (thetaPerturbationSwitch == 1) {
    g_rng = seed;
    for (i = iMin; i < iMax; i++)
      for (j = jMin; j < jMax; j++)
        for (k = kMin; k < kMax; k++) {
          size_t ijk = IJK(i, j, k);
          if (zPos[ijk] <= thetaHeight) {
            double pert = 2.0 * thetaAmplitude * (rng_uniform() - 0.5);
            th[ijk] = (float)(((double)th[ijk] / rho[ijk] + pert) * rho[ijk]);
          }
        }
  }
}

/* Surface-layer 2-D inputs (hydro_core.c:835-860). cd/ch are not inputs of the device
 * path: the device initialises them from the log law on the first step. */
static void build_surface(void) {
  size_t n2 = fe_host_plane_elems(), ij;
  for (ij = 0; ij < n2; ij++) {
    z0m[ij] = surflayer_z0;
    z0t[ij] = surflayer_z0t;
    if (surflayerSelector == 1) {
      htFlux[ij] = surflayer_wth;
      if (moistureSelector > 0) qFlux[ij] = surflayer_wq;
    }
    tskin[ij] = (float)(temp_grnd / pow((double)refPressure / pres_grnd, (double)R_cp));
    if (moistureSelector > 0) qskin[ij] = 0.0f;
  }
}

static int restart_topography(const char *path);
static int restart_state(const char *path);

int fe_host_init(unsigned long long seed) {
  size_t n, n2;
  char inName[2100];
  if (fe_params_error_count() != 0) {
    snprintf(g_msg, sizeof(g_msg), "parameter errors present: %s", fe_params_last_message());
    return -1;
  }
  if (Nh != 3) {
    snprintf(g_msg, sizeof(g_msg), "Nh must be 3 (5th-order advection stencil)");
    return -1;
  }
  fe_host_cleanup();
  Nxp = Nx; Nyp = Ny; Nzp = Nz;
  iMin = Nh; iMax = Nxp + Nh; jMin = Nh; jMax = Nyp + Nh; kMin = Nh; kMax = Nzp + Nh;
  dXi = 1.0f / dX; dYi = 1.0f / dY; dZi = 1.0f / dZ;
  n = fe_host_field_elems();
  n2 = fe_host_plane_elems();
  xPos = alloc_f(n); yPos = alloc_f(n); zPos = alloc_f(n); topoPos = alloc_f(n2);
  J31 = alloc_f(n); J32 = alloc_f(n); J33 = alloc_f(n); D_Jac = alloc_f(n); invD_Jac = alloc_f(n);
  hydroFlds = alloc_f(n * 5); hydroFldsFrhs = alloc_f(n * 5);
  hydroBaseStateFlds = alloc_f(n * 2); hydroPres = alloc_f(n); hydroBaseStatePres = alloc_f(n);
  hydroTauFlds = alloc_f(n * 9);
  sgstkeScalars = alloc_f(n * (TKESelector > 0 ? TKESelector : 1));
  sgstkeScalarsFrhs = alloc_f(n * (TKESelector > 0 ? TKESelector : 1));
  moistScalars = alloc_f(n * (moistureNvars > 0 ? moistureNvars : 1));
  moistScalarsFrhs = alloc_f(n * (moistureNvars > 0 ? moistureNvars : 1));
  moistTauFlds = alloc_f(n * 3 * (moistureNvars > 0 ? moistureNvars : 1));
  fricVel = alloc_f(n2); htFlux = alloc_f(n2); tskin = alloc_f(n2); invOblen = alloc_f(n2);
  z0m = alloc_f(n2); z0t = alloc_f(n2); qFlux = alloc_f(n2); qskin = alloc_f(n2);
  if (!xPos || !yPos || !zPos || !topoPos || !J31 || !J32 || !J33 || !D_Jac || !invD_Jac || !hydroFlds ||
      !hydroFldsFrhs || !hydroBaseStateFlds || !hydroPres || !hydroBaseStatePres || !hydroTauFlds ||
      !sgstkeScalars || !sgstkeScalarsFrhs || !moistScalars || !moistScalarsFrhs || !moistTauFlds || !fricVel ||
      !htFlux || !tskin || !invOblen || !z0m || !z0t || !qFlux || !qskin) {
    snprintf(g_msg, sizeof(g_msg), "host allocation failed");
    fe_host_cleanup();
    return -1;
  }
  if (g_topoFile[0] && !g_topoGlobal) {
    if (read_topofile(g_topoFile) != 0) return -1;
  }
  snprintf(inName, sizeof(inName), "%s%s", g_inPath, g_inFile);  /* io_netcdf.c:112 */
  if (g_inFile[0] && !g_topoFile[0] && restart_topography(inName) != 0) return -1;
  build_grid();
  build_metrics();
  build_base_state_and_ics(seed);
  if (surflayerSelector > 0) build_surface();
  /* time (time_integration.c:95-105): a restart continues at the step after the first '.' of inFile */
  simTime = 0.0f;
  simTime_it = 0;
  simTime_itRestart = 0;
  numRKstages = 2;
  if (g_inFile[0]) {
    const char *dot = strchr(g_inFile, '.');
    if (!dot || sscanf(dot + 1, "%d", &simTime_itRestart) != 1) {
      snprintf(g_msg, sizeof(g_msg), "inFile %s has no .<step> suffix", g_inFile);
      return -1;
    }
    simTime_it = simTime_itRestart;
    simTime = dt * (float)simTime_it;
    if (restart_state(inName) != 0) return -1;
  }
  return 0;
}

/* Water-vapour initial condition: rho*qv [g/kg * kg/m^3] with qv falling linearly from
 * q_sfc at z = 0 to q_top at z_top (constant above), evaluated at zPos; q_l = 0. */
int fe_host_set_qv_profile(float q_sfc, float q_top, float z_top) {
  size_t n = fe_host_field_elems(), ijk;
  if (moistureSelector <= 0 || moistureNvars <= 0 || !moistScalars) return -1;
  for (ijk = 0; ijk < n; ijk++) {
    double z = zPos[ijk], q;
    if (z <= 0.0) q = q_sfc;
    else if (z >= z_top) q = q_top;
    else q = q_sfc + ((double)q_top - q_sfc) * z / z_top;
    moistScalars[ijk] = (float)(q * hydroFlds[ijk]);
    if (moistureNvars > 1) moistScalars[n + ijk] = 0.0f;
  }
  return 0;
}

const char *fe_host_topofile(void) { return g_topoFile; }


/* ------------------------------------------------------------------ binary output */
/* The reference's raw binary output (io_binary.c:19-132): one file per rank and output step,
 * <outPath><outFileBase>_rank_<rank>.<step>, holding every variable registered for output in
 * registration order. A record is the name length (int), the name bytes, the number of
 * dimensions (int, 3 or 2) and the halo-inclusive extents (int each), then the float values in
 * the halo-inclusive layout. u, v, w, theta, TKE and moisture are written divided by rho (the
 * reference divides its host arrays in place; this writer divides into a scratch buffer and leaves
 * the host state as it is). */
static int put_record(FILE *f, const char *name, int nd, const float *v, const float *rho, float *tmp) {
  static const char *divided[] = {"u", "v", "w", "theta", "TKE_0", "TKE_1", "qv", "ql", "qr", NULL};
  int len = (int)strlen(name), ext[3] = {Nxp + 2 * Nh, Nyp + 2 * Nh, Nzp + 2 * Nh};
  size_t n = (size_t)ext[0] * ext[1] * (nd == 3 ? (size_t)ext[2] : 1), m;
  int a, div = 0;
  if (nd == 3)
    for (a = 0; divided[a]; a++) div |= !strcmp(name, divided[a]);
  if (div) {
    for (m = 0; m < n; m++) tmp[m] = v[m] / rho[m];
    v = tmp;
  }
  if (fwrite(&len, sizeof(int), 1, f) != 1 || fwrite(name, 1, (size_t)len, f) != (size_t)len ||
      fwrite(&nd, sizeof(int), 1, f) != 1 || fwrite(ext, sizeof(int), (size_t)nd, f) != (size_t)nd ||
      fwrite(v, sizeof(float), n, f) != n)
    return -1;
  return 0;
}

/* Registration order and conditions of the reference's output list (grid.c:229-232,
 * hydro_core.c:632-930) without its DEBUG and BASE_STATE_IO_DUMP builds. */
int fe_host_write_binary(const char *path, int tstep) {
  char name[1100], fn[64];
  size_t n = fe_host_field_elems();
  const float *rho = hydroFlds;
  float *tmp;
  FILE *f;
  int rc = 0, q;
  static const char *hydroNames[5] = {"rho", "u", "v", "w", "theta"};
  static const char *tauNames[9] = {"Tau11", "Tau21", "Tau31", "Tau32", "Tau22", "Tau33", "TauTH1", "TauTH2", "TauTH3"};
  static const char *moistNames[2] = {"qv", "ql"};
  if (!hydroFlds) {
    snprintf(g_msg, sizeof(g_msg), "fe_host_write_binary: no host state (call fe_host_init first)");
    return -1;
  }
  if (!path || !path[0]) {
    snprintf(name, sizeof(name), "%s%s_rank_%d.%d", g_outPath, g_outFileBase, 0, tstep);
    path = name;
  }
  f = fopen(path, "wb");
  if (!f) {
    snprintf(g_msg, sizeof(g_msg), "fe_host_write_binary: cannot open %s", path);
    return -1;
  }
  tmp = (float *)malloc(n * sizeof(float));
  if (!tmp) {
    fclose(f);
    return -1;
  }
#define PUT(nm, nd, v) rc |= put_record(f, (nm), (nd), (v), rho, tmp)
  PUT("xPos", 3, xPos); PUT("yPos", 3, yPos); PUT("zPos", 3, zPos); PUT("topoPos", 2, topoPos);
  for (q = 0; q < 5; q++) PUT(hydroNames[q], 3, hydroFlds + q * n);
  PUT("pressure", 3, hydroPres);
  if (hydroForcingWrite == 1)
    for (q = 0; q < 5; q++) {
      snprintf(fn, sizeof(fn), "F_%s", hydroNames[q]);
      PUT(fn, 3, hydroFldsFrhs + q * n);
    }
  if (TKESelector > 0) {
    for (q = 0; q < TKESelector; q++) {
      snprintf(fn, sizeof(fn), "TKE_%d", q);
      PUT(fn, 3, sgstkeScalars + q * n);
    }
    if (hydroForcingWrite == 1)
      for (q = 0; q < TKESelector; q++) {
        snprintf(fn, sizeof(fn), "F_TKE%d", q);
        PUT(fn, 3, sgstkeScalarsFrhs + q * n);
      }
  }
  if (hydroSubGridWrite == 1 && turbulenceSelector > 0)
    for (q = 0; q < 9; q++) PUT(tauNames[q], 3, hydroTauFlds + q * n);
  if (surflayerSelector > 0) {
    PUT("tskin", 2, tskin); PUT("fricVel", 2, fricVel); PUT("htFlux", 2, htFlux); PUT("invOblen", 2, invOblen);
    if (moistureSelector > 0) { PUT("qskin", 2, qskin); PUT("qFlux", 2, qFlux); }
    PUT("z0m", 2, z0m); PUT("z0t", 2, z0t);
  }
  if (moistureSelector > 0) {
    for (q = 0; q < moistureNvars && q < 2; q++) PUT(moistNames[q], 3, moistScalars + q * n);
    if (hydroForcingWrite == 1)
      for (q = 0; q < moistureNvars && q < 2; q++) {
        snprintf(fn, sizeof(fn), "F_%s", moistNames[q]);
        PUT(fn, 3, moistScalarsFrhs + q * n);
      }
    if (hydroSubGridWrite == 1 && moistureSGSturb > 0)
      for (q = 0; q < moistureNvars && q < 2; q++) {
        int d;
        for (d = 0; d < 3; d++) {
          snprintf(fn, sizeof(fn), "TauQ%c%d", q == 0 ? 'v' : 'l', d + 1);
          PUT(fn, 3, moistTauFlds + (size_t)(q * 3 + d) * n);
        }
      }
  }
#undef PUT
  free(tmp);
  if (fclose(f) != 0) rc = -1;
  if (rc) snprintf(g_msg, sizeof(g_msg), "fe_host_write_binary: write to %s failed", path);
  return rc;
}


/* ------------------------------------------------------------------ netCDF output */
/* The reference writes its output as netCDF (io_netcdf.c:392-717): dimensions time (unlimited,
 * one record), zIndex, yIndex, xIndex (interior extents); int coordinate variables zIndex,
 * yIndex, xIndex holding 0..N-1; then every variable registered for output, in registration
 * order, as float (time, zIndex, yIndex, xIndex) or (time, yIndex, xIndex) with the interior cells
 * only, x fastest, u, v, w, theta, TKE and moisture divided by rho (its NORHO build,
 * io_netcdf.c:340). The reference asks the netCDF library for its NETCDF4 (HDF5) container; this
 * writer has no library to call and writes the same dimensions, variables and values in the
 * classic 64-bit-offset container (CDF-2), which the netCDF library and its Python readers open
 * the same way. No attributes are written (the reference writes none). */
typedef struct {
  const char *name;
  int nd;           /* 3: (time, z, y, x), 2: (time, y, x) */
  const float *v;   /* halo-inclusive host array */
} nc_rec;

static void be32(unsigned char *p, uint32_t x) { p[0] = x >> 24; p[1] = x >> 16; p[2] = x >> 8; p[3] = x; }
static int put_be32(FILE *f, uint32_t x) { unsigned char b[4]; be32(b, x); return fwrite(b, 1, 4, f) == 4 ? 0 : -1; }
static int put_be64(FILE *f, uint64_t x) {
  int rc = put_be32(f, (uint32_t)(x >> 32));
  rc |= put_be32(f, (uint32_t)x);
  return rc;
}
static int put_name(FILE *f, const char *s) {
  static const unsigned char zero[4] = {0, 0, 0, 0};
  size_t n = strlen(s);
  int rc = put_be32(f, (uint32_t)n);
  if (fwrite(s, 1, n, f) != n) return -1;
  /* (name bytes follow their length, zero-padded to 4 bytes) */
  if (n % 4) rc |= fwrite(zero, 1, 4 - n % 4, f) == 4 - n % 4 ? 0 : -1;
  return rc;
}
static size_t name_bytes(const char *s) { size_t n = strlen(s); return 4 + (n + 3) / 4 * 4; }

/* The same registration order and conditions as fe_host_write_binary. Returns the count. */
static int output_registry(nc_rec *r, char names[][16]) {
  size_t n = fe_host_field_elems();
  int c = 0, q, d;
  static const char *hydroNames[5] = {"rho", "u", "v", "w", "theta"};
  static const char *tauNames[9] = {"Tau11", "Tau21", "Tau31", "Tau32", "Tau22", "Tau33", "TauTH1", "TauTH2", "TauTH3"};
  static const char *moistNames[2] = {"qv", "ql"};
#define REG(nm, dims, arr) do { snprintf(names[c], 16, "%s", (nm)); r[c].name = names[c]; r[c].nd = (dims); r[c].v = (arr); c++; } while (0)
  REG("xPos", 3, xPos); REG("yPos", 3, yPos); REG("zPos", 3, zPos); REG("topoPos", 2, topoPos);
  for (q = 0; q < 5; q++) REG(hydroNames[q], 3, hydroFlds + q * n);
  REG("pressure", 3, hydroPres);
  if (hydroForcingWrite == 1)
    for (q = 0; q < 5; q++) { char t[16]; snprintf(t, sizeof(t), "F_%s", hydroNames[q]); REG(t, 3, hydroFldsFrhs + q * n); }
  if (TKESelector > 0) {
    for (q = 0; q < TKESelector; q++) { char t[16]; snprintf(t, sizeof(t), "TKE_%d", q); REG(t, 3, sgstkeScalars + q * n); }
    if (hydroForcingWrite == 1)
      for (q = 0; q < TKESelector; q++) { char t[16]; snprintf(t, sizeof(t), "F_TKE%d", q); REG(t, 3, sgstkeScalarsFrhs + q * n); }
  }
  if (hydroSubGridWrite == 1 && turbulenceSelector > 0)
    for (q = 0; q < 9; q++) REG(tauNames[q], 3, hydroTauFlds + q * n);
  if (surflayerSelector > 0) {
    REG("tskin", 2, tskin); REG("fricVel", 2, fricVel); REG("htFlux", 2, htFlux); REG("invOblen", 2, invOblen);
    if (moistureSelector > 0) { REG("qskin", 2, qskin); REG("qFlux", 2, qFlux); }
    REG("z0m", 2, z0m); REG("z0t", 2, z0t);
  }
  if (moistureSelector > 0) {
    for (q = 0; q < moistureNvars && q < 2; q++) REG(moistNames[q], 3, moistScalars + q * n);
    if (hydroForcingWrite == 1)
      for (q = 0; q < moistureNvars && q < 2; q++) { char t[16]; snprintf(t, sizeof(t), "F_%s", moistNames[q]); REG(t, 3, moistScalarsFrhs + q * n); }
    if (hydroSubGridWrite == 1 && moistureSGSturb > 0)
      for (q = 0; q < moistureNvars && q < 2; q++)
        for (d = 0; d < 3; d++) { char t[16]; snprintf(t, sizeof(t), "TauQ%c%d", q == 0 ? 'v' : 'l', d + 1); REG(t, 3, moistTauFlds + (size_t)(q * 3 + d) * n); }
  }
#undef REG
  return c;
}

int fe_host_write_netcdf(const char *path, int tstep) {
  static const char *dimNames[4] = {"time", "zIndex", "yIndex", "xIndex"};
  static const char *divided[] = {"u", "v", "w", "theta", "TKE_0", "TKE_1", "qv", "ql", "qr", NULL};
  nc_rec reg[64];
  char names[64][16], fname[1100];
  const int Nx = Nxp, Ny = Nyp, Nz = Nzp, Nyh = Nyp + 2 * Nh, Nzh = Nzp + 2 * Nh;
  const uint32_t dimLen[4] = {0, (uint32_t)Nz, (uint32_t)Ny, (uint32_t)Nx};
  int nreg, v, rc = 0, i, j, k, a;
  uint64_t hdr, off;
  size_t n3 = (size_t)Nx * Ny * Nz;
  float *buf;
  unsigned char *out;
  FILE *f;
  if (!hydroFlds) {
    snprintf(g_msg, sizeof(g_msg), "fe_host_write_netcdf: no host state (call fe_host_init first)");
    return -1;
  }
  nreg = output_registry(reg, names);
  /* the classic container records each variable's size in 32 bits */
  if (4 * (uint64_t)Nx * Ny * Nz > 0xFFFFFFFCull) {
    snprintf(g_msg, sizeof(g_msg), "fe_host_write_netcdf: a %dx%dx%d field exceeds the classic container's 4 GiB "
             "variable size; use fe_host_write_binary", Nx, Ny, Nz);
    return -1;
  }
  if (!path || !path[0]) {
    snprintf(fname, sizeof(fname), "%s%s.%d", g_outPath, g_outFileBase, tstep);
    path = fname;
  }
  /* header size: magic, numrecs, dim list, empty attribute list, variable list */
  hdr = 4 + 4 + 8;
  for (a = 0; a < 4; a++) hdr += name_bytes(dimNames[a]) + 4;
  hdr += 8 + 8;
  for (a = 1; a < 4; a++) hdr += name_bytes(dimNames[a]) + 4 + 4 + 8 + 4 + 4 + 8;
  for (v = 0; v < nreg; v++) hdr += name_bytes(reg[v].name) + 4 + 4 * (reg[v].nd == 3 ? 4 : 3) + 8 + 4 + 4 + 8;
  f = fopen(path, "wb");
  if (!f) {
    snprintf(g_msg, sizeof(g_msg), "fe_host_write_netcdf: cannot open %s", path);
    return -1;
  }
  /* every write below is its own statement: the file order is the statement order */
#define W(x) rc |= (x)
  W(fwrite("CDF\x02", 1, 4, f) == 4 ? 0 : -1);
  W(put_be32(f, 1));                         /* numrecs */
  W(put_be32(f, 0x0A)); W(put_be32(f, 4));   /* NC_DIMENSION, 4 dimensions */
  for (a = 0; a < 4; a++) { W(put_name(f, dimNames[a])); W(put_be32(f, dimLen[a])); }
  W(put_be32(f, 0)); W(put_be32(f, 0));      /* no global attributes */
  W(put_be32(f, 0x0B)); W(put_be32(f, (uint32_t)(3 + nreg)));  /* NC_VARIABLE */
  off = hdr;
  for (a = 1; a < 4; a++) {  /* coordinate variables zIndex, yIndex, xIndex: NC_INT, non-record */
    W(put_name(f, dimNames[a])); W(put_be32(f, 1)); W(put_be32(f, (uint32_t)a));
    W(put_be32(f, 0)); W(put_be32(f, 0));    /* no attributes */
    W(put_be32(f, 4)); W(put_be32(f, 4 * dimLen[a])); W(put_be64(f, off));
    off += 4 * (uint64_t)dimLen[a];
  }
  for (v = 0; v < nreg; v++) {  /* record variables, NC_FLOAT, in one record */
    uint64_t vsize = 4 * (uint64_t)Nx * Ny * (reg[v].nd == 3 ? (uint64_t)Nz : 1);
    W(put_name(f, reg[v].name)); W(put_be32(f, reg[v].nd == 3 ? 4 : 3)); W(put_be32(f, 0));
    if (reg[v].nd == 3) W(put_be32(f, 1));
    W(put_be32(f, 2)); W(put_be32(f, 3));
    W(put_be32(f, 0)); W(put_be32(f, 0));    /* no attributes */
    W(put_be32(f, 5)); W(put_be32(f, (uint32_t)vsize)); W(put_be64(f, off));
    off += vsize;
  }
#undef W
  buf = (float *)malloc(n3 * sizeof(float));
  out = (unsigned char *)malloc(n3 * 4);
  if (!buf || !out) {
    free(buf); free(out); fclose(f);
    return -1;
  }
  for (a = 1; a < 4; a++) {
    for (i = 0; i < (int)dimLen[a]; i++) be32(out + 4 * i, (uint32_t)i);
    rc |= fwrite(out, 1, 4 * dimLen[a], f) == 4 * dimLen[a] ? 0 : -1;
  }
  for (v = 0; v < nreg; v++) {
    const float *src = reg[v].v;
    size_t m = 0;
    int div = 0;
    for (a = 0; reg[v].nd == 3 && divided[a]; a++) div |= !strcmp(reg[v].name, divided[a]);
    if (reg[v].nd == 3) {
      for (k = 0; k < Nz; k++)
        for (j = 0; j < Ny; j++)
          for (i = 0; i < Nx; i++) {
            size_t c = ((size_t)(i + Nh) * Nyh + (j + Nh)) * Nzh + (k + Nh);
            buf[m++] = div ? src[c] / hydroFlds[c] : src[c];
          }
    } else {
      for (j = 0; j < Ny; j++)
        for (i = 0; i < Nx; i++) buf[m++] = src[(size_t)(i + Nh) * Nyh + (j + Nh)];
    }
    for (i = 0; i < (int)m; i++) {
      uint32_t u;
      memcpy(&u, buf + i, 4);
      be32(out + 4 * (size_t)i, u);
    }
    rc |= fwrite(out, 1, 4 * m, f) == 4 * m ? 0 : -1;
  }
  free(buf);
  free(out);
  if (fclose(f) != 0) rc = -1;
  if (rc) snprintf(g_msg, sizeof(g_msg), "fe_host_write_netcdf: write to %s failed", path);
  return rc;
}


/* ------------------------------------------------------------------ restart input */
/* Reading an initial-condition / restart file (inFile; FastEddy.c:202-243, io_netcdf.c:106-390):
 * every variable registered for output that the file holds is read from its first time record
 * into the interior cells; u, v, w, theta, TKE and moisture are multiplied back by rho (its NORHO
 * build), the Tau fields are skipped, and the surface planes get their periodic halos
 * (hydro_core.c:982-1014). The file must use the classic netCDF container (CDF-1 or CDF-2, as
 * fe_host_write_netcdf writes): this build links no netCDF/HDF5 library. The grid is rebuilt from
 * the file's topoPos (unless a topoFile is given) by the same grid code as a fresh start. */
typedef struct {
  char name[64];
  int ndims, dimids[8], type, isrec;
  uint64_t vsize, begin;
} cdf_var;
typedef struct {
  FILE *f;
  int version, ndims, nvars;
  uint32_t numrecs, dimlen[16];
  char dimname[16][64];
  cdf_var var[256];
  uint64_t recsize;
} cdf_file;

static int get_be32(FILE *f, uint32_t *x) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return -1;
  *x = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
  return 0;
}
static int get_name(FILE *f, char *out, size_t cap) {
  uint32_t n;
  char pad[4];
  if (get_be32(f, &n) || n >= cap || fread(out, 1, n, f) != n) return -1;
  out[n] = 0;
  if (n % 4 && fread(pad, 1, 4 - n % 4, f) != 4 - n % 4) return -1;
  return 0;
}
static int skip_atts(FILE *f) {
  uint32_t tag, n, a, type, cnt;
  char name[256];
  static const int tsize[7] = {0, 1, 1, 2, 4, 4, 8};
  if (get_be32(f, &tag) || get_be32(f, &n)) return -1;
  if (tag == 0) return n == 0 ? 0 : -1;
  if (tag != 0x0C) return -1;
  for (a = 0; a < n; a++) {
    uint64_t bytes;
    if (get_name(f, name, sizeof(name)) || get_be32(f, &type) || get_be32(f, &cnt) || type < 1 || type > 6) return -1;
    bytes = ((uint64_t)cnt * tsize[type] + 3) / 4 * 4;
    if (fseek(f, (long)bytes, SEEK_CUR) != 0) return -1;
  }
  return 0;
}
static int cdf_open(cdf_file *c, const char *path) {
  char magic[4];
  uint32_t tag, n, k, x, hi, lo;
  memset(c, 0, sizeof(*c));
  c->f = fopen(path, "rb");
  if (!c->f) return -1;
  if (fread(magic, 1, 4, c->f) != 4 || memcmp(magic, "CDF", 3) != 0 || (magic[3] != 1 && magic[3] != 2)) return -2;
  c->version = magic[3];
  if (get_be32(c->f, &c->numrecs) || get_be32(c->f, &tag) || get_be32(c->f, &n)) return -2;
  if (tag == 0x0A) {
    if (n > 16) return -2;
    for (k = 0; k < n; k++)
      if (get_name(c->f, c->dimname[k], 64) || get_be32(c->f, &c->dimlen[k])) return -2;
    c->ndims = (int)n;
  } else if (tag != 0 || n != 0) {
    return -2;
  }
  if (skip_atts(c->f)) return -2;
  if (get_be32(c->f, &tag) || get_be32(c->f, &n)) return -2;
  if (tag == 0x0B) {
    if (n > 256) return -2;
    for (k = 0; k < n; k++) {
      cdf_var *v = &c->var[k];
      uint32_t nd, d, type, vs;
      if (get_name(c->f, v->name, sizeof(v->name)) || get_be32(c->f, &nd) || nd > 8) return -2;
      v->ndims = (int)nd;
      for (d = 0; d < nd; d++) {
        if (get_be32(c->f, &x) || x >= (uint32_t)c->ndims) return -2;
        v->dimids[d] = (int)x;
      }
      if (skip_atts(c->f) || get_be32(c->f, &type) || get_be32(c->f, &vs)) return -2;
      v->type = (int)type;
      v->vsize = vs;
      if (c->version == 2) {
        if (get_be32(c->f, &hi) || get_be32(c->f, &lo)) return -2;
        v->begin = ((uint64_t)hi << 32) | lo;
      } else {
        if (get_be32(c->f, &lo)) return -2;
        v->begin = lo;
      }
      v->isrec = nd > 0 && c->dimlen[v->dimids[0]] == 0;
      if (v->isrec) c->recsize += v->vsize;
    }
    c->nvars = (int)n;
  } else if (tag != 0 || n != 0) {
    return -2;
  }
  return 0;
}
static const cdf_var *cdf_find(const cdf_file *c, const char *name) {
  int k;
  for (k = 0; k < c->nvars; k++)
    if (!strcmp(c->var[k].name, name)) return &c->var[k];
  return NULL;
}
static int cdf_dim(const cdf_file *c, const char *name) {
  int k;
  for (k = 0; k < c->ndims; k++)
    if (!strcmp(c->dimname[k], name)) return k;
  return -1;
}
/* First record of a float variable over (time, zIndex, yIndex, xIndex) or (time, yIndex, xIndex)
 * into the interior of a halo-inclusive host array; nd = 3 or 2. Returns 0, 1 (absent), -1. */
static int cdf_read_interior(cdf_file *c, const char *name, int nd, float *dst) {
  const cdf_var *v = cdf_find(c, name);
  const int Nyh = Nyp + 2 * Nh, Nzh = Nzp + 2 * Nh, nk = nd == 3 ? Nzp : 1;
  size_t cnt = (size_t)Nxp * Nyp * nk, m;
  unsigned char *raw;
  int i, j, k;
  if (!v) return 1;
  if (v->type != 5 || v->ndims != nd + 1 || !v->isrec || c->numrecs < 1) return -1;
  /* the dimensions must be (time, zIndex, yIndex, xIndex) or (time, yIndex, xIndex) in this order
   * (io_netcdf.c:392-717): any other order or any other dimensions would be read transposed */
  {
    const char *order[4] = {"time", "zIndex", "yIndex", "xIndex"};
    int d;
    for (d = 0; d <= nd; d++) {
      const char *want = d == 0 ? order[0] : order[nd == 3 ? d : d + 1];
      if (v->dimids[d] != cdf_dim(c, want)) {
        snprintf(g_msg, sizeof(g_msg), "variable %s: dimension %d is not %s", name, d, want);
        return -2;
      }
    }
  }
  raw = (unsigned char *)malloc(cnt * 4);
  if (!raw) return -1;
  if (fseek(c->f, (long)v->begin, SEEK_SET) != 0 || fread(raw, 4, cnt, c->f) != cnt) {
    free(raw);
    return -1;
  }
  m = 0;
  for (k = 0; k < nk; k++)
    for (j = 0; j < Nyp; j++)
      for (i = 0; i < Nxp; i++, m++) {
        uint32_t u = ((uint32_t)raw[4 * m] << 24) | ((uint32_t)raw[4 * m + 1] << 16) | ((uint32_t)raw[4 * m + 2] << 8) |
                     raw[4 * m + 3];
        float val;
        memcpy(&val, &u, 4);
        if (nd == 3) dst[((size_t)(i + Nh) * Nyh + (j + Nh)) * Nzh + (k + Nh)] = val;
        else dst[(size_t)(i + Nh) * Nyh + (j + Nh)] = val;
      }
  free(raw);
  return 0;
}
static int cdf_check_dims(cdf_file *c, const char *path) {
  int z = cdf_dim(c, "zIndex"), y = cdf_dim(c, "yIndex"), x = cdf_dim(c, "xIndex");
  if (cdf_dim(c, "time") < 0 || z < 0 || y < 0 || x < 0) {
    snprintf(g_msg, sizeof(g_msg), "inFile %s lacks the time/zIndex/yIndex/xIndex dimensions", path);
    return -1;
  }
  if ((int)c->dimlen[z] != Nzp || (int)c->dimlen[y] != Nyp || (int)c->dimlen[x] != Nxp) {
    snprintf(g_msg, sizeof(g_msg), "inFile %s is %ux%ux%u, the parameters ask for %dx%dx%d", path, c->dimlen[x],
             c->dimlen[y], c->dimlen[z], Nxp, Nyp, Nzp);
    return -1;
  }
  return 0;
}
static int cdf_open_checked(cdf_file *c, const char *path) {
  int rc = cdf_open(c, path);
  if (rc) {
    snprintf(g_msg, sizeof(g_msg), rc == -1 ? "cannot open inFile %s" : "inFile %s is not a classic netCDF file", path);
    if (c->f) fclose(c->f);
    return -1;
  }
  if (cdf_check_dims(c, path)) {
    fclose(c->f);
    return -1;
  }
  return 0;
}

static int restart_topography(const char *path) {
  cdf_file *c = (cdf_file *)calloc(1, sizeof(cdf_file));
  float *t = alloc_f(fe_host_plane_elems());
  int rc = -1, i, j;
  if (!c || !t) goto done;
  if (cdf_open_checked(c, path)) goto done;
  rc = cdf_read_interior(c, "topoPos", 2, t);
  fclose(c->f);
  if (rc == 1) {  /* no topography in the file: flat, or the parameters' */
    rc = 0;
    goto done;
  }
  if (rc == 0) {
    free(g_topoGlobal);
    g_topoGlobal = (double *)malloc(sizeof(double) * (size_t)Nx * (size_t)Ny);
    if (!g_topoGlobal) { rc = -1; goto done; }
    for (i = 0; i < Nx; i++)
      for (j = 0; j < Ny; j++) g_topoGlobal[(size_t)i * Ny + j] = t[(size_t)(i + Nh) * (Ny + 2 * Nh) + (j + Nh)];
  } else if (rc != -2) {
    snprintf(g_msg, sizeof(g_msg), "inFile %s: cannot read topoPos", path);
  }
done:
  free(t);
  free(c);
  return rc;
}

/* periodic halo of a 2-D host plane (single rank) */
static void plane_halo(float *a) {
  const int Nxh = Nxp + 2 * Nh, Nyh = Nyp + 2 * Nh;
  int i, j;
  for (i = Nh; i < Nxp + Nh; i++)
    for (j = 0; j < Nh; j++) {
      a[(size_t)i * Nyh + j] = a[(size_t)i * Nyh + j + Nyp];
      a[(size_t)i * Nyh + Nyp + Nh + j] = a[(size_t)i * Nyh + Nh + j];
    }
  for (i = 0; i < Nh; i++)
    for (j = 0; j < Nyh; j++) {
      a[(size_t)i * Nyh + j] = a[(size_t)(i + Nxp) * Nyh + j];
      a[(size_t)(Nxp + Nh + i) * Nyh + j] = a[(size_t)(Nh + i) * Nyh + j];
    }
  (void)Nxh;
}

static int restart_state(const char *path) {
  static const char *hydroNames[5] = {"rho", "u", "v", "w", "theta"};
  static const char *moistNames[2] = {"qv", "ql"};
  cdf_file *c = (cdf_file *)calloc(1, sizeof(cdf_file));
  size_t n = fe_host_field_elems();
  const int Nyh = Nyp + 2 * Nh, Nzh = Nzp + 2 * Nh;
  int rc = 0, q, i, j, k;
  if (!c) return -1;
  if (cdf_open_checked(c, path)) { free(c); return -1; }
#define RD(nm, nd, dst) do { int r_ = cdf_read_interior(c, (nm), (nd), (dst)); \
    if (r_ == -2) { char t_[sizeof(g_msg)]; snprintf(t_, sizeof(t_), "%s", g_msg); \
      snprintf(g_msg, sizeof(g_msg), "inFile %s: %s", path, t_); rc = -1; } \
    else if (r_ < 0) { snprintf(g_msg, sizeof(g_msg), "inFile %s: cannot read %s", path, (nm)); rc = -1; } } while (0)
  for (q = 0; q < 5; q++) RD(hydroNames[q], 3, hydroFlds + q * n);
  RD("pressure", 3, hydroPres);
  for (q = 0; q < TKESelector; q++) { char t[16]; snprintf(t, sizeof(t), "TKE_%d", q); RD(t, 3, sgstkeScalars + q * n); }
  if (surflayerSelector > 0) {
    RD("tskin", 2, tskin); RD("fricVel", 2, fricVel); RD("htFlux", 2, htFlux); RD("invOblen", 2, invOblen);
    if (moistureSelector > 0) { RD("qskin", 2, qskin); RD("qFlux", 2, qFlux); }
    RD("z0m", 2, z0m); RD("z0t", 2, z0t);
  }
  for (q = 0; moistureSelector > 0 && q < moistureNvars && q < 2; q++) RD(moistNames[q], 3, moistScalars + q * n);
#undef RD
  fclose(c->f);
  free(c);
  if (rc) return rc;
  /* back to flux form (io_netcdf.c:340-375): interior cells times the file's rho */
  {
    float *flux[2 + 2 + 3] = {hydroFlds + n, hydroFlds + 2 * n, hydroFlds + 3 * n, hydroFlds + 4 * n, NULL, NULL, NULL};
    int nf = 4;
    for (q = 0; q < TKESelector && q < 1; q++) flux[nf++] = sgstkeScalars + q * n;
    for (q = 0; moistureSelector > 0 && q < moistureNvars && q < 2; q++) flux[nf++] = moistScalars + q * n;
    for (q = 0; q < nf; q++)
      for (i = Nh; i < Nxp + Nh; i++)
        for (j = Nh; j < Nyp + Nh; j++)
          for (k = Nh; k < Nzp + Nh; k++) {
            size_t cc = ((size_t)i * Nyh + j) * Nzh + k;
            flux[q][cc] = flux[q][cc] * hydroFlds[cc];
          }
  }
  if (surflayerSelector > 0) {
    plane_halo(z0m); plane_halo(z0t); plane_halo(htFlux); plane_halo(fricVel); plane_halo(tskin);
    if (moistureSelector > 0) { plane_halo(qFlux); plane_halo(qskin); }
  }
  return 0;
}
