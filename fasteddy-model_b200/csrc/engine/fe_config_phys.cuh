// fe_config_phys.cuh -- the kernels' parameter block (Phys) derived from a configuration.
//
// One derivation for every entry point that launches the kernels (the engine's domains and the
// allocation-free tendency call), so they cannot disagree on a cadence, a scheme or a constant.
// Expects fasteddy_b200.h (fe_config) and fe_device.cuh (Phys) to be included before.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>

namespace fe {

inline void phys_from_config(const fe_config& c, Phys& P) {
  std::memset(&P, 0, sizeof(P));
  P.Nx = c.Nx; P.Ny = c.Ny; P.Nz = c.Nz;
  P.nxh = c.Nx + 6; P.nyh = c.Ny + 6; P.nzh = c.Nz + 6;
  P.sj = P.nzh;
  P.si = P.nyh * P.nzh;
  P.n = (long long)P.nxh * P.nyh * P.nzh;
  P.n2 = (long long)P.nxh * P.nyh;
  P.iMin = 3; P.iMax = c.Nx + 3; P.jMin = 3; P.jMax = c.Ny + 3; P.kMin = 3; P.kMax = c.Nz + 3;
  P.dX = c.dX; P.dY = c.dY; P.dZ = c.dZ;
  P.dXi = 1.0f / c.dX; P.dYi = 1.0f / c.dY; P.dZi = 1.0f / c.dZ;
  P.dt = c.dt;
  P.itRestart = c.simTime_itRestart;
  P.turb = c.turbulenceSelector > 0;
  P.tke = P.turb && c.TKESelector > 0;
  P.ntke = P.tke ? 1 : 0;
  P.moist = c.moistureSelector > 0;
  P.nmoist = P.moist ? c.moistureNvars : 0;
  P.nf = 5 + P.ntke + P.nmoist;
  P.pgf = c.pgfSelector > 0;
  P.buoy = c.buoyancySelector > 0;
  P.cor = c.coriolisSelector > 0;
  P.advSel = c.advectionSelector;
  P.tkeAdvSel = c.TKEAdvSelector;
  P.qvAdvSel = c.moistureAdvSelectorQv;
  P.qiAdvSel = c.moistureAdvSelectorQi;
  P.qlSch = ql_scheme(c.moistureAdvSelectorQi);
  P.bHyb = c.b_hyb; P.tkeBHyb = c.TKEAdvSelector_b_hyb; P.qvB = c.moistureAdvSelectorQv_b;
  P.filt = c.filterSelector > 0;
  P.filtCoef = filter_coef(c.filter_6th_coeff, c.dt);
  P.lsf = c.lsfSelector > 0;
  P.lsfSub = P.lsf && c.lsf_horMnSubTerms == 1;
  P.lsfN = P.lsf ? (int)roundf(c.lsf_freq / c.dt) : 1;  // as the reference rounds it (cuda_hydroCoreDevice.cu:402-404)
  P.lsfFac = (float)P.lsfN;
  {
    const float w[5] = {c.lsf_w_surf, c.lsf_w_lev1, c.lsf_w_lev2, c.lsf_w_zlev1, c.lsf_w_zlev2};
    const float th[5] = {c.lsf_th_surf, c.lsf_th_lev1, c.lsf_th_lev2, c.lsf_th_zlev1, c.lsf_th_zlev2};
    const float qv[5] = {c.lsf_qv_surf, c.lsf_qv_lev1, c.lsf_qv_lev2, c.lsf_qv_zlev1, c.lsf_qv_zlev2};
    for (int m = 0; m < 5; m++) { P.lsfW[m] = w[m]; P.lsfTh[m] = th[m]; P.lsfQv[m] = qv[m]; }
  }
  P.c_s = c.c_s; P.c_k = c.c_k;
  P.surf = c.surflayerSelector;
  P.surfStab = c.surflayer_stab;
  P.idealSine = c.surflayer_idealsine;
  P.qskinInput = c.surflayer_qskin_input;
  P.z0 = c.surflayer_z0; P.z0t = c.surflayer_z0t; P.wth = c.surflayer_wth; P.tr = c.surflayer_tr;
  P.wq = c.surflayer_wq; P.qr = c.surflayer_qr;
  P.idealTs = c.surflayer_ideal_ts; P.idealTe = c.surflayer_ideal_te; P.idealAmp = c.surflayer_ideal_amp;
  P.idealQts = c.surflayer_ideal_qts; P.idealQte = c.surflayer_ideal_qte; P.idealQamp = c.surflayer_ideal_qamp;
  P.moistSGS = c.moistureSGSturb;
  P.moistCond = c.moistureCond;
  P.condBasePres = c.moistureCondBasePres;
  P.condTscale = c.moistureCondTscale;
  // cadences as the reference computes them (cuda_hydroCoreDevice.cu:382, cuda_surfaceLayerDevice.cu:128)
  P.mpFreq = std::max(1, (int)roundf(fmaxf(c.moistureMPcallTscale, c.dt) / c.dt));
  P.tempFreq = std::max(1, (int)roundf((float)(10.0 / c.dt)));
  P.damp = c.dampingLayerSelector > 0;
  P.dampDepth = c.dampingLayerDepth;
  P.U_g = c.U_g; P.V_g = c.V_g; P.z_Ug = c.z_Ug; P.z_Vg = c.z_Vg; P.Ug_grad = c.Ug_grad; P.Vg_grad = c.Vg_grad;
  P.fHorz = c.corioConstHorz; P.fVert = c.corioConstVert; P.fLS = c.corioLS_fact;
  P.oneRK = c.physics_oneRKonly;
  P.tempGrnd = c.temp_grnd; P.presGrnd = c.pres_grnd;
  P.R_gas = c.R_gas; P.R_vapor = c.R_vapor; P.Rv_Rg = c.Rv_Rg; P.cp_gas = c.cp_gas; P.cv_gas = c.cv_gas;
  P.g = c.accel_g; P.R_cp = c.R_cp; P.cp_R = c.cp_R; P.cp_cv = c.cp_cv; P.p0 = c.refPressure; P.kappa = c.kappa;
  P.L_v = c.L_v;
}

}  // namespace fe
