// fe_device.cuh -- device-side data structures and physics routines of the B200 engine.
//
// Layout: every 3-D field is stored exactly as at the C-ABI boundary (reference layout,
// halo width 3, k fastest): c = i*si + j*sj + k, si = (Ny+6)*(Nz+6), sj = Nz+6. Halo
// cells are real memory: the periodic images and the vertical boundary values are
// written by the producer of a state (the RK commit epilogue or the halo-fill kernel),
// so stencils never branch on boundaries. Field f of a state block starts at f*n.
//
// Floating point follows the reference's FP32 expressions operation by operation where
// the result is cancellation-sensitive (perturbation pressure, face velocities), so the
// device path tracks the reference CUDA build to a few ulps.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fe {

// Scalar configuration of one domain, passed by value to every kernel.
struct Phys {
  int Nx, Ny, Nz;
  int nxh, nyh, nzh;
  int si, sj;                // i and j strides of a field
  long long n;               // elements of one halo-inclusive field
  long long n2;              // elements of one halo-inclusive 2-D plane
  int iMin, iMax, jMin, jMax, kMin, kMax;
  float dX, dY, dZ, dXi, dYi, dZi;
  float dt;
  int itRestart;
  int ntke, nmoist, nf;      // prognostic field counts (nf = 5 + ntke + nmoist)
  int pgf, buoy, cor, turb, tke, advSel, tkeAdvSel, qvAdvSel, qiAdvSel;
  float bHyb, tkeBHyb, qvB;
  float c_s, c_k;
  int surf, surfStab, idealSine, qskinInput;
  float z0, z0t, wth, tr, wq, qr, idealTs, idealTe, idealAmp, idealQts, idealQte, idealQamp;
  int moist, moistSGS, moistCond, condBasePres;
  float condTscale;
  int mpFreq;                // steps between microphysics calls
  int tempFreq;              // steps between skin-temperature updates
  int damp;
  float dampDepth;
  float U_g, V_g, z_Ug, z_Vg, Ug_grad, Vg_grad;
  float fHorz, fVert, fLS;
  int oneRK;
  float tempGrnd, presGrnd;
  float R_gas, R_vapor, Rv_Rg, cp_gas, cv_gas, g, R_cp, cp_R, cp_cv, p0, kappa, L_v;
  float c1;                  // R/p0^(R/cp), evaluated on the device (as the reference does)
  float presFac;             // powf(p0/pres_grnd, R_cp), evaluated on the device
};

// Device pointers of one domain.
struct Ptrs {
  const float *zPos, *J31, *J32, *J33, *D, *invD;
  const float *rhoBS, *thBS;   // base state (rho, rho*theta)
  const float *pBS;            // powf(thBS*c1, cp_cv) per cell, device-evaluated
  float *tau;                  // 9 SGS stress/flux fields (order of the reference's hydroTauFlds)
  float *tkeQ;                 // 3 fields: (de/dx_j)*Km*rho, the TKE transport fluxes
  float *ls;                   // SGS length scale
  float *mtau;                 // 3 per moisture species
  float *cd, *ch, *cq, *fricVel, *htFlux, *tskin, *invOblen, *z0m, *z0t, *qFlux, *qskin;
  int *clockIt;                // simTime_it of the step being computed
  float *clockTime;            // simTime of the step being computed
};

__device__ __forceinline__ float sgnf(float x) { return copysignf(1.0f, x); }

// 1/rho with the reference's floor (rhoInv in cuda_hydroCoreDevice.cu:952-957)
__device__ __forceinline__ float rinv(float r) { return 1.0f / fmaxf(r, 1e-6f); }

// ---------------------------------------------------------------- boundary values
// Value of field `f` in the vertical halo cell (column source cell `src` = interior
// column (is,js), level k outside [kMin,kMax)), for hydroBCs = 2:
//   rho, rho*theta : base state at that cell          (cuda_BCsDevice.cu:120-150)
//   rho*u, rho*v   : bottom copy of kMin, top geostrophic * rho_BS(kMax-1) (:152-211)
//   rho*w          : bottom copy, top 0
//   rho*e          : bottom copy, top 0               (cuda_hydroCoreDevice.cu:516-529)
//   moisture       : zero gradient both ends          (cuda_BCsDevice.cu:213-241)
__device__ __forceinline__ float momentum_bs(const Phys& P, int fld, float z, float rho) {
  float zg, vg, gr;
  if (fld == 1) { zg = P.z_Ug; vg = P.U_g; gr = P.Ug_grad; }
  else if (fld == 2) { zg = P.z_Vg; vg = P.V_g; gr = P.Vg_grad; }
  else { zg = 0.0f; vg = 0.0f; gr = 0.0f; }
  if (z < zg) return vg * rho;
  return (vg + gr * (z - zg)) * rho;
}

// ---------------------------------------------------------------- pressure
// Perturbation pressure of cell t (cuda_pressureDevice.cu:53-113). The moist factor is
// evaluated with the same double promotions as the reference expression.
__device__ __forceinline__ float pert_pressure(const Phys& P, const float* __restrict__ st, const float* __restrict__ pBS,
                                               long long t) {
  const float rt = st[4 * P.n + t];
  float rtm = rt;
  if (P.nmoist > 0) {
    const float qv = st[(long long)(5 + P.ntke) * P.n + t];
    const float r = st[t];
    rtm = (float)((double)rt * (1.0 + (double)(P.Rv_Rg * qv / r) * 1e-3));
  }
  return powf(rtm * P.c1, P.cp_cv) - pBS[t];
}

// ---------------------------------------------------------------- advection
// 5th/6th-order hybrid flux across the face between cells s0 (lower) and s1 (upper):
// arguments are the stencil m2,m1,z0,p1,p2,p3 relative to the lower cell
// (cuda_advectionDevice.cu:365-376).
__device__ __forceinline__ float hyb56_flux(float m2, float m1, float z0, float p1, float p2, float p3, float vel,
                                            float bfac) {
  const float sixtieth = 1.0f / 60.0f;
  return sixtieth * (37.0f * (p1 + z0) - 8.0f * (p2 + m1) + (p3 + m2) -
                     bfac * sgnf(vel) * ((p3 - m2) - 5.0f * (p2 - m1) + 10.0f * (p1 - z0)));
}

// WENO5 face value from the upwind side, stencil a..e (cuda_advectionDevice.cu:626-926).
// The squares of the smoothness indicators are products (the reference spells them
// powf(x, 2.0)); the three normalised weights share one reciprocal of their sum.
__device__ __forceinline__ float weno5_face(float a, float b, float c, float d, float e) {
  const float g1 = 1.0f / 10.0f, g2 = 3.0f / 5.0f, g3 = 3.0f / 10.0f, tol = 1e-6f;
  const float f1 = (1.0f / 3.0f) * a - (7.0f / 6.0f) * b + (11.0f / 6.0f) * c;
  const float f2 = -(1.0f / 6.0f) * b + (5.0f / 6.0f) * c + (1.0f / 3.0f) * d;
  const float f3 = (1.0f / 3.0f) * c + (5.0f / 6.0f) * d - (1.0f / 6.0f) * e;
  const float s1 = a - 2.0f * b + c, t1 = a - 4.0f * b + 3.0f * c;
  const float s2 = b - 2.0f * c + d, t2 = b - d;
  const float s3 = c - 2.0f * d + e, t3 = 3.0f * c - 4.0f * d + e;
  const float b1 = (13.0f / 12.0f) * (s1 * s1) + (1.0f / 4.0f) * (t1 * t1);
  const float b2 = (13.0f / 12.0f) * (s2 * s2) + (1.0f / 4.0f) * (t2 * t2);
  const float b3 = (13.0f / 12.0f) * (s3 * s3) + (1.0f / 4.0f) * (t3 * t3);
  const float q1 = tol + b1, q2 = tol + b2, q3 = tol + b3;
  const float w1 = g1 / (q1 * q1);
  const float w2 = g2 / (q2 * q2);
  const float w3 = g3 / (q3 * q3);
  const float inv = 1.0f / (w1 + w2 + w3);
  return (w1 * inv) * f1 + (w2 * inv) * f2 + (w3 * inv) * f3;
}

// The reference blends both one-sided values with weights 0.5(1 +- sign(u)), which are
// exactly 1 and 0; only the upwind value is evaluated here (same result).
__device__ __forceinline__ float weno5_flux(float m2, float m1, float z0, float p1, float p2, float p3, float vel) {
  return sgnf(vel) > 0.0f ? weno5_face(m2, m1, z0, p1, p2) : weno5_face(p3, p2, p1, z0, m1);
}

// Face velocities of a cell: lower/upper faces in x, y, z (cuda_advectionDevice.cu:54-121).
struct FaceVel {
  float um, up, vm, vp, wm, wp;
};

// Contravariant momentum term (D/rho)*(m + w*J) of one cell, as in the reference sum.
__device__ __forceinline__ float contra(float D, float r, float m, float w, float J) { return (D / r) * (m + w * J); }

}  // namespace fe
