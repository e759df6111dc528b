/* fe_refglobals.h -- the global host symbols through which the FastEddy driver hands
 * its inputs to the CUDA layer.
 *
 * The reference CUDA wrappers take no arguments: they read these globals, which the
 * reference's host modules define (SRC/GRID/grid.h:28-57, SRC/FEMPI/fempi.h:25-39,
 * SRC/HYDRO_CORE/hydro_core.h:35-183, SRC/TIME_INTEGRATION/time_integration.h:24-33,
 * SRC/IO/io.h:36). A drop-in replacement of that layer therefore has to read the
 * same names with the same C types; this header declares exactly the subset the
 * replacement reads or writes. In a FastEddy executable they resolve to the
 * reference's definitions; in this repository libfe_host.so defines them.
 */
#ifndef FE_REFGLOBALS_H
#define FE_REFGLOBALS_H

#ifdef __cplusplus
extern "C" {
#endif

/* FEMPI */
extern int mpi_size_world, mpi_rank_world;
extern int numProcsX, numProcsY;
extern int Nxp, Nyp, Nzp;
/* GRID */
extern int Nh;
extern int Nx, Ny, Nz;
extern int iMin, iMax, jMin, jMax, kMin, kMax;
extern float dX, dY, dZ, dXi, dYi, dZi;
extern float *xPos, *yPos, *zPos, *topoPos;
extern float *J31, *J32, *J33, *D_Jac, *invD_Jac;
/* FECUDA */
extern int tBx, tBy, tBz;
/* HYDRO_CORE */
extern int Nhydro, hydroBCs;
extern int hydroForcingWrite, hydroForcingLog, hydroSubGridWrite;
extern float *hydroFlds, *hydroFldsFrhs, *hydroBaseStateFlds, *hydroPres, *hydroBaseStatePres;
extern float *hydroTauFlds;
extern float R_gas, R_vapor, Rv_Rg, cp_gas, cv_gas, accel_g, R_cp, cp_R, cp_cv, refPressure, kappa, L_v;
extern int pgfSelector, buoyancySelector, coriolisSelector;
extern float coriolisLatitude, corioConstHorz, corioConstVert, corioLS_fact;
extern int turbulenceSelector, TKESelector, TKEAdvSelector;
extern float TKEAdvSelector_b_hyb, c_s, c_k;
extern float *sgstkeScalars, *sgstkeScalarsFrhs;
extern int diffusionSelector;
extern int advectionSelector;
extern float b_hyb;
extern int surflayerSelector;
extern float surflayer_z0, surflayer_z0t, surflayer_wth, surflayer_tr, surflayer_wq, surflayer_qr;
extern int surflayer_qskin_input, surflayer_stab;
extern float *fricVel, *htFlux, *tskin, *invOblen, *z0m, *z0t, *qFlux, *qskin;
extern int surflayer_idealsine;
extern float surflayer_ideal_ts, surflayer_ideal_te, surflayer_ideal_amp;
extern float surflayer_ideal_qts, surflayer_ideal_qte, surflayer_ideal_qamp;
extern int lsfSelector;
extern int lsf_horMnSubTerms;
extern float lsf_freq;
extern float lsf_w_surf, lsf_w_lev1, lsf_w_lev2, lsf_w_zlev1, lsf_w_zlev2;
extern float lsf_th_surf, lsf_th_lev1, lsf_th_lev2, lsf_th_zlev1, lsf_th_zlev2;
extern float lsf_qv_surf, lsf_qv_lev1, lsf_qv_lev2, lsf_qv_zlev1, lsf_qv_zlev2;
extern int moistureSelector, moistureNvars, moistureAdvSelectorQv;
extern float moistureAdvSelectorQv_b;
extern int moistureSGSturb, moistureCond;
extern float *moistScalars, *moistScalarsFrhs, *moistTauFlds;
extern int moistureAdvSelectorQi;
extern float moistureCondTscale;
extern int moistureCondBasePres;
extern float moistureMPcallTscale;
extern int filterSelector;
extern float filter_6th_coeff;
extern int dampingLayerSelector;
extern float dampingLayerDepth;
extern float temp_grnd, pres_grnd;
extern float U_g, V_g, z_Ug, z_Vg, Ug_grad, Vg_grad;
extern int physics_oneRKonly;
/* TIME_INTEGRATION */
extern int timeMethod, Nt, NtBatch;
extern float dt;
extern float simTime;
extern int simTime_it, simTime_itRestart, numRKstages;

#ifdef __cplusplus
}
#endif
#endif
