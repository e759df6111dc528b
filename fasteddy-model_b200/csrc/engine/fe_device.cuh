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
  int qlSch;                 // q_l's scheme as an ADV_* id (from qiAdvSel: 0 upwind, 1 WENO3, 2 WENO5)
  float bHyb, tkeBHyb, qvB;
  int filt;                  // 6th-order vertical filter of rho w on (filterSelector = 1)
  float filtCoef;            // 0.015625 filter_6th_coeff / dt
  int lsf, lsfSub;           // large-scale forcing; its subsidence terms (lsf_horMnSubTerms)
  int lsfN;                  // steps between applications, roundf(lsf_freq/dt)
  float lsfFac;              // the same as a float factor of the per-hour rates
  float lsfW[5], lsfTh[5], lsfQv[5];  // surface value, values at zlev1 and zlev2, zlev1, zlev2
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
  // halo exchange of a decomposed domain: offsets, in floats, from this domain's state arena to
  // the arena of the domain holding the horizontal neighbour (dx, dy) at [(dx+1)*3 + (dy+1)]
  // (all 0 for an undecomposed domain), and whether the x / y halos come from neighbours
  long long nbr[9];
  int peerX, peerY;
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
  const float* delta;          // grid scale (dx dy dz D)^(1/3) per cell, or nullptr (evaluated inline)
  float* feat;                 // inputs of the learned closure per ring cell (11 fields), or nullptr
  float* sgsF;                 // SGS tendencies for the march kernel's physics stages (7 fields), or nullptr
  float* lsfProf;              // slab means of rho, rho u, rho v, rho theta, rho q_v (nzh levels each), or nullptr
  double* lsfPart;             // per-block FP64 partial sums of the slab means
  int *clockIt;                // simTime_it of the step being computed
  float *clockTime;            // simTime of the step being computed
};

__device__ __forceinline__ float sgnf(float x) { return copysignf(1.0f, x); }

// 1/rho with the reference's floor (rhoInv in cuda_hydroCoreDevice.cu:952-957)
__device__ __forceinline__ float rinv(float r) { return 1.0f / fmaxf(r, 1e-6f); }

// SGS grid scale (dx dy dz D)^(1/3) of cell c (cuda_sgstkeDevice.cu:96-151); constant in time, so
// the engine evaluates it once per grid, with this same expression, into Q.delta.
__device__ __forceinline__ float grid_scale_of(const Phys& P, float D) { return powf(P.dX * P.dY * P.dZ * D, (float)(1.0 / 3.0)); }
__device__ __forceinline__ float grid_scale(const Phys& P, const Ptrs& Q, long long c) {
  return Q.delta ? Q.delta[c] : grid_scale_of(P, Q.D[c]);
}

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

// Perturbation pressure of the bottom halo level (k = 0) of a column after a commit: rho and
// rho theta there are the base state, q_v the bottom copy of the first level (the reference
// recomputes this level every stage, cuda_pressureDevice.cu:53-113; no stencil reads it).
struct Level0 {
  float thBS, rhoBS, pBS;
};
__device__ __forceinline__ Level0 level0_inputs(const Ptrs& Q, long long c0) { return {Q.thBS[c0], Q.rhoBS[c0], Q.pBS[c0]}; }
__device__ __forceinline__ float level0_pressure(const Phys& P, const Level0& b, int nmoist, float qv) {
  float rt = b.thBS;
  if (nmoist > 0) rt = (float)((double)rt * (1.0 + (double)(P.Rv_Rg * qv / b.rhoBS) * 1e-3));
  return powf(rt * P.c1, P.cp_cv) - b.pBS;
}
__device__ __forceinline__ float level0_pressure(const Phys& P, const Ptrs& Q, long long c0, int nmoist, float qv) {
  return level0_pressure(P, level0_inputs(Q, c0), nmoist, qv);
}

// Primitive variables (phi/rho, formed as phi * rinv(rho)) of a cell and its neighbours, read
// straight from the flux-form state. Offsets (di, dj, dk) are relative to cell c. The product is
// rounded on its own (never fused into a following add), as when it is staged in a tile.
struct GlobalPrims {
  const float *rho, *mu, *mv, *mw, *mth, *e, *q;
  long long n, c;
  int si, sj;
  __device__ __forceinline__ long long at(int di, int dj, int dk) const { return c + di * (long long)si + dj * (long long)sj + dk; }
  __device__ __forceinline__ float r(int di, int dj, int dk) const { return rho[at(di, dj, dk)]; }
  __device__ __forceinline__ float u(int di, int dj, int dk) const { const long long x = at(di, dj, dk); return __fmul_rn(mu[x], rinv(rho[x])); }
  __device__ __forceinline__ float v(int di, int dj, int dk) const { const long long x = at(di, dj, dk); return __fmul_rn(mv[x], rinv(rho[x])); }
  __device__ __forceinline__ float w(int di, int dj, int dk) const { const long long x = at(di, dj, dk); return __fmul_rn(mw[x], rinv(rho[x])); }
  __device__ __forceinline__ float th(int di, int dj, int dk) const { const long long x = at(di, dj, dk); return __fmul_rn(mth[x], rinv(rho[x])); }
  __device__ __forceinline__ float ev(int di, int dj, int dk) const { const long long x = at(di, dj, dk); return __fmul_rn(e[x], rinv(rho[x])); }
  __device__ __forceinline__ float qm(int m, int di, int dj, int dk) const {
    const long long x = at(di, dj, dk);
    return __fmul_rn(q[m * n + x], rinv(rho[x]));
  }
};

// ---------------------------------------------------------------- advection
// The flux and velocity helpers spell out every rounding (__fmaf_rn/__fmul_rn/__fadd_rn):
// the same face is evaluated by more than one inlined copy (a marching thread block's first
// plane and its loop), and explicit roundings make every copy produce the same bits, so
// results do not depend on the launch shape.
//
// 5th/6th-order hybrid flux across the face between cells s0 (lower) and s1 (upper):
// arguments are the stencil m2,m1,z0,p1,p2,p3 relative to the lower cell
// (cuda_advectionDevice.cu:365-376): (37(p1+z0) - 8(p2+m1) + (p3+m2)
//  - bfac sgn(vel) ((p3-m2) - 5(p2-m1) + 10(p1-z0))) / 60, bfac = 1 - b_hyb >= 0.
__device__ __forceinline__ float hyb56_flux(float m2, float m1, float z0, float p1, float p2, float p3, float vel,
                                            float bfac) {
  const float sixtieth = 1.0f / 60.0f;
  const float a = __fadd_rn(p1, z0), b = __fadd_rn(p2, m1), c = __fadd_rn(p3, m2);
  const float d = __fsub_rn(p3, m2), e = __fsub_rn(p2, m1), f = __fsub_rn(p1, z0);
  const float cen = __fadd_rn(__fmaf_rn(37.0f, a, __fmul_rn(-8.0f, b)), c);
  const float upw = __fmaf_rn(10.0f, f, __fmaf_rn(-5.0f, e, d));
  const float sb = copysignf(bfac, vel);  // = bfac sgn(vel) exactly (bfac >= 0)
  return __fmul_rn(sixtieth, __fmaf_rn(-sb, upw, cen));
}

// WENO5 face value from the upwind side, stencil a..e (cuda_advectionDevice.cu:626-926).
// The squares of the smoothness indicators are products (the reference spells them
// powf(x, 2.0)). The normalised weights w_k = (g_k/q_k^2) / sum_j (g_j/q_j^2), q = tol + beta,
// are formed with one division: multiplying through by (q1 q2 q3)^2 gives w_k ~ g_k (q_i q_j)^2
// (i, j != k). With q >= tol = 1e-6 the products stay normal, and they stay finite while the
// smoothness indicators are below 1e9 (jumps of the advected field below ~3e4 across a cell).
// FAST: the normalisation by the weight sum uses the fast division (__fdividef, 2 ulp; the sum
// lies in [1e-25, 2e36], well inside its range) instead of the IEEE one.
template <bool FAST = false>
__device__ __forceinline__ float weno5_face(float a, float b, float c, float d, float e) {
  const float g1 = 1.0f / 10.0f, g2 = 3.0f / 5.0f, g3 = 3.0f / 10.0f, tol = 1e-6f;
  const float k13 = 1.0f / 3.0f, k76 = 7.0f / 6.0f, k116 = 11.0f / 6.0f, k16 = 1.0f / 6.0f, k56 = 5.0f / 6.0f;
  const float f1 = __fmaf_rn(k116, c, __fmaf_rn(-k76, b, __fmul_rn(k13, a)));
  const float f2 = __fmaf_rn(k13, d, __fmaf_rn(k56, c, __fmul_rn(-k16, b)));
  const float f3 = __fmaf_rn(-k16, e, __fmaf_rn(k56, d, __fmul_rn(k13, c)));
  const float s1 = __fadd_rn(__fmaf_rn(-2.0f, b, a), c), t1 = __fmaf_rn(3.0f, c, __fmaf_rn(-4.0f, b, a));
  const float s2 = __fadd_rn(__fmaf_rn(-2.0f, c, b), d), t2 = __fsub_rn(b, d);
  const float s3 = __fadd_rn(__fmaf_rn(-2.0f, d, c), e), t3 = __fadd_rn(__fmaf_rn(-4.0f, d, __fmul_rn(3.0f, c)), e);
  const float k1312 = 13.0f / 12.0f, k14 = 1.0f / 4.0f;
  const float b1 = __fmaf_rn(k14, __fmul_rn(t1, t1), __fmul_rn(k1312, __fmul_rn(s1, s1)));
  const float b2 = __fmaf_rn(k14, __fmul_rn(t2, t2), __fmul_rn(k1312, __fmul_rn(s2, s2)));
  const float b3 = __fmaf_rn(k14, __fmul_rn(t3, t3), __fmul_rn(k1312, __fmul_rn(s3, s3)));
  const float q1 = __fadd_rn(tol, b1), q2 = __fadd_rn(tol, b2), q3 = __fadd_rn(tol, b3);
  const float a1 = __fmul_rn(q2, q3), a2 = __fmul_rn(q1, q3), a3 = __fmul_rn(q1, q2);
  const float u1 = __fmul_rn(g1, __fmul_rn(a1, a1));
  const float u2 = __fmul_rn(g2, __fmul_rn(a2, a2));
  const float u3 = __fmul_rn(g3, __fmul_rn(a3, a3));
  const float num = __fmaf_rn(u3, f3, __fmaf_rn(u2, f2, __fmul_rn(u1, f1)));
  const float den = __fadd_rn(__fadd_rn(u1, u2), u3);
  return FAST ? __fdividef(num, den) : __fdiv_rn(num, den);
}

// The reference blends both one-sided values with weights 0.5(1 +- sign(u)), which are
// exactly 1 and 0; only the upwind value is evaluated here (same result). The upwind stencil
// is selected value by value, so lanes of one warp with opposite velocities do not diverge.
template <bool FAST = false>
__device__ __forceinline__ float weno5_flux(float m2, float m1, float z0, float p1, float p2, float p3, float vel) {
  const bool up = sgnf(vel) > 0.0f;
  return weno5_face<FAST>(up ? m2 : p3, up ? m1 : p2, up ? z0 : p1, up ? p1 : z0, up ? p2 : m1);
}

// Advection schemes by the reference's selector value (advectionSelector, TKEAdvSelector,
// moistureAdvSelectorQv; cuda_hydroCoreDevice.cu:635-654). q_l's selector (0 upwind, 1 WENO3,
// 2 WENO5, cuda_hydroCoreDevice.cu:726-736) is mapped onto these ids by the host.
constexpr int ADV_UPWIND = 0, ADV_QUICK = 1, ADV_HYB34 = 2, ADV_HYB56 = 3, ADV_WENO3 = 4, ADV_WENO5 = 5,
              ADV_CEN2 = 6;
// The WENO schemes update the tendency direction by direction (three updates, x then y then
// z); the others subtract the divergence summed over the three directions in one update.
__host__ __device__ constexpr bool adv_split(int sel) { return sel == ADV_WENO3 || sel == ADV_WENO5; }

// WENO3 face value from the upwind side (cuda_advectionDevice.cu:382-623): a = second cell
// upwind, b = upwind cell, c = downwind cell. Candidates -a/2 + 3b/2 and (b + c)/2, smoothness
// (b - a)^2 and (c - b)^2, linear weights 1/3 and 2/3, tol 1e-6. As in weno5_face the two
// normalised weights come from one division: w_k ~ g_k q_j^2 (j != k), q = tol + beta.
template <bool FAST = false>
__device__ __forceinline__ float weno3_face(float a, float b, float c) {
  const float g1 = 1.0f / 3.0f, g2 = 2.0f / 3.0f, tol = 1e-6f;
  const float f1 = __fmaf_rn(1.5f, b, __fmul_rn(-0.5f, a));
  const float f2 = __fmaf_rn(0.5f, b, __fmul_rn(0.5f, c));
  const float d1 = __fsub_rn(b, a), d2 = __fsub_rn(c, b);
  const float q1 = __fadd_rn(tol, __fmul_rn(d1, d1)), q2 = __fadd_rn(tol, __fmul_rn(d2, d2));
  const float u1 = __fmul_rn(g1, __fmul_rn(q2, q2)), u2 = __fmul_rn(g2, __fmul_rn(q1, q1));
  const float num = __fmaf_rn(u2, f2, __fmul_rn(u1, f1));
  const float den = __fadd_rn(u1, u2);
  return FAST ? __fdividef(num, den) : __fdiv_rn(num, den);
}

// Face value of scheme `sel` across the face between cells z0 (lower) and p1 (upper), stencil
// m2..p3 as for hyb56_flux; the flux through the face is vel times this value. bfac = 1 - b
// for the hybrid schemes.
//   upwind  z0 if vel > 0 else p1        (cuda_advectionDevice.cu:126-158, fmaxf/fminf form)
//   QUICK   (6 z0 + 3 p1 - m1)/8 if vel > 0 else (6 p1 + 3 z0 - p2)/8       (:206-254)
//   HYB34   (7(p1+z0) - (p2+m1) + bfac sgn(vel) ((p2-m1) - 3(p1-z0)))/12   (:260-312)
//   centred (z0 + p1)/2                                                    (:162-200)
template <bool FAST = false>
__device__ __forceinline__ float adv_face(int sel, float m2, float m1, float z0, float p1, float p2, float p3,
                                          float vel, float bfac) {
  switch (sel) {
    case ADV_UPWIND:
      return vel > 0.0f ? z0 : p1;
    case ADV_QUICK: {
      const bool up = vel > 0.0f;
      const float a = up ? z0 : p1, b = up ? p1 : z0, c = up ? m1 : p2;
      return __fmul_rn(0.125f, __fsub_rn(__fmaf_rn(6.0f, a, __fmul_rn(3.0f, b)), c));
    }
    case ADV_HYB34: {
      const float twelfth = 1.0f / 12.0f;
      const float cen = __fsub_rn(__fmul_rn(7.0f, __fadd_rn(p1, z0)), __fadd_rn(p2, m1));
      const float upw = __fmaf_rn(-3.0f, __fsub_rn(p1, z0), __fsub_rn(p2, m1));
      return __fmul_rn(twelfth, __fmaf_rn(copysignf(bfac, vel), upw, cen));
    }
    case ADV_HYB56:
      return hyb56_flux(m2, m1, z0, p1, p2, p3, vel, bfac);
    case ADV_WENO3: {
      const bool up = sgnf(vel) > 0.0f;
      return weno3_face<FAST>(up ? m1 : p2, up ? z0 : p1, up ? p1 : z0);
    }
    case ADV_WENO5:
      return weno5_flux<FAST>(m2, m1, z0, p1, p2, p3, vel);
    default:
      return __fmul_rn(0.5f, __fadd_rn(z0, p1));
  }
}

// ---------------------------------------------------------------- two faces at once
// The same face values for two stencils held lane-wise in float2 (the two y faces or the two
// z faces of a cell, or the x faces of two fields), on the packed FP32 pipe of sm_100
// (__ffma2_rn, __fadd2_rn, __fmul2_rn: each lane rounds exactly as the scalar operation). Every
// lane equals adv_face() of its own stencil bit for bit: the same operations in the same order,
// x - y written as x + (-y), which IEEE addition gives exactly. The WENO division stays per lane.
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 f2s(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float2 hyb56_flux2(float2 m2, float2 m1, float2 z0, float2 p1, float2 p2, float2 p3,
                                              float2 vel, float2 bfac) {
  const float2 a = add2(p1, z0), b = add2(p2, m1), c = add2(p3, m2);
  const float2 d = sub2(p3, m2), e = sub2(p2, m1), f = sub2(p1, z0);
  const float2 cen = add2(fma2(f2s(37.0f), a, mul2(f2s(-8.0f), b)), c);
  const float2 upw = fma2(f2s(10.0f), f, fma2(f2s(-5.0f), e, d));
  const float2 msb = f2(-copysignf(bfac.x, vel.x), -copysignf(bfac.y, vel.y));
  return mul2(f2s(1.0f / 60.0f), fma2(msb, upw, cen));
}

template <bool FAST = false>
__device__ __forceinline__ float2 weno5_face2(float2 a, float2 b, float2 c, float2 d, float2 e) {
  const float g1 = 1.0f / 10.0f, g2 = 3.0f / 5.0f, g3 = 3.0f / 10.0f, tol = 1e-6f;
  const float k13 = 1.0f / 3.0f, k76 = 7.0f / 6.0f, k116 = 11.0f / 6.0f, k16 = 1.0f / 6.0f, k56 = 5.0f / 6.0f;
  const float2 f1 = fma2(f2s(k116), c, fma2(f2s(-k76), b, mul2(f2s(k13), a)));
  const float2 fB = fma2(f2s(k13), d, fma2(f2s(k56), c, mul2(f2s(-k16), b)));
  const float2 f3 = fma2(f2s(-k16), e, fma2(f2s(k56), d, mul2(f2s(k13), c)));
  const float2 s1 = add2(fma2(f2s(-2.0f), b, a), c), t1 = fma2(f2s(3.0f), c, fma2(f2s(-4.0f), b, a));
  const float2 s2 = add2(fma2(f2s(-2.0f), c, b), d), t2 = sub2(b, d);
  const float2 s3 = add2(fma2(f2s(-2.0f), d, c), e), t3 = add2(fma2(f2s(-4.0f), d, mul2(f2s(3.0f), c)), e);
  const float k1312 = 13.0f / 12.0f, k14 = 1.0f / 4.0f;
  const float2 b1 = fma2(f2s(k14), mul2(t1, t1), mul2(f2s(k1312), mul2(s1, s1)));
  const float2 b2 = fma2(f2s(k14), mul2(t2, t2), mul2(f2s(k1312), mul2(s2, s2)));
  const float2 b3 = fma2(f2s(k14), mul2(t3, t3), mul2(f2s(k1312), mul2(s3, s3)));
  const float2 q1 = add2(f2s(tol), b1), q2 = add2(f2s(tol), b2), q3 = add2(f2s(tol), b3);
  const float2 a1 = mul2(q2, q3), a2 = mul2(q1, q3), a3 = mul2(q1, q2);
  const float2 u1 = mul2(f2s(g1), mul2(a1, a1));
  const float2 u2 = mul2(f2s(g2), mul2(a2, a2));
  const float2 u3 = mul2(f2s(g3), mul2(a3, a3));
  const float2 num = fma2(u3, f3, fma2(u2, fB, mul2(u1, f1)));
  const float2 den = add2(add2(u1, u2), u3);
  return FAST ? f2(__fdividef(num.x, den.x), __fdividef(num.y, den.y)) : f2(__fdiv_rn(num.x, den.x), __fdiv_rn(num.y, den.y));
}

template <bool FAST = false>
__device__ __forceinline__ float2 weno5_flux2(float2 m2, float2 m1, float2 z0, float2 p1, float2 p2, float2 p3, float2 vel) {
  const bool ux = sgnf(vel.x) > 0.0f, uy = sgnf(vel.y) > 0.0f;
  return weno5_face2<FAST>(f2(ux ? m2.x : p3.x, uy ? m2.y : p3.y), f2(ux ? m1.x : p2.x, uy ? m1.y : p2.y),
                           f2(ux ? z0.x : p1.x, uy ? z0.y : p1.y), f2(ux ? p1.x : z0.x, uy ? p1.y : z0.y),
                           f2(ux ? p2.x : m1.x, uy ? p2.y : m1.y));
}

// adv_face() of two stencils (bfac per lane): HYB56 and WENO5 on the packed pipe, the other
// schemes lane by lane.
template <bool FAST = false>
__device__ __forceinline__ float2 adv_face2(int sel, float2 m2, float2 m1, float2 z0, float2 p1, float2 p2, float2 p3,
                                            float2 vel, float2 bfac) {
  if (sel == ADV_HYB56) return hyb56_flux2(m2, m1, z0, p1, p2, p3, vel, bfac);
  if (sel == ADV_WENO5) return weno5_flux2<FAST>(m2, m1, z0, p1, p2, p3, vel);
  return f2(adv_face<FAST>(sel, m2.x, m1.x, z0.x, p1.x, p2.x, p3.x, vel.x, bfac.x),
            adv_face<FAST>(sel, m2.y, m1.y, z0.y, p1.y, p2.y, p3.y, vel.y, bfac.y));
}

// q_l's selector (moistureAdvSelectorQi) as a scheme id.
__host__ __device__ constexpr int ql_scheme(int qi) { return qi == 0 ? ADV_UPWIND : (qi == 1 ? ADV_WENO3 : ADV_WENO5); }
// The filter's factor as the reference forms it (cuda_filtersDevice.cu:86): the literal
// 0.015625 is double, so the quotient is taken in double and stored as float.
__host__ __device__ inline float filter_coef(float coeff, float dt) { return (float)(0.015625 * (double)coeff / (double)(1.0f * dt)); }

// ---------------------------------------------------------------- large-scale forcing
// Step `it` applies the forcing in its last RK stage and takes the slab means at its start
// (cuda_hydroCoreDevice.cu:401-406, cuda_timeIntDevice.cu:125-127): every lsfN steps after
// the restart step (the forcing also needs lsfN steps since the restart).
__device__ __forceinline__ bool lsf_step(const Phys& P, int it) {
  return P.lsf && it > P.itRestart && (it - P.itRestart) >= P.lsfN && it % P.lsfN == 0;
}
__device__ __forceinline__ bool lsf_means_step(const Phys& P, int it) {
  return P.lsf && P.lsfSub && it > P.itRestart && it % P.lsfN == 0;
}
// Piecewise-linear forcing profile times rho (cuda_largeScaleForcingsDevice.cu:177-212): linear
// from the surface value to lev1 at zlev1, to lev2 at zlev2, constant lev2 above.
__device__ __forceinline__ float lsf_profile(const float (&p)[5], float z, float rho) {
  if (z <= p[3]) return (p[0] + ((p[1] - p[0]) / p[3]) * z) * rho;
  if (z <= p[4]) return (p[1] + ((p[2] - p[1]) / (p[4] - p[3])) * (z - p[3])) * rho;
  return p[2] * rho;
}
// The per-hour rates times the application interval in steps (the double literal 3600.0 makes
// the division double, as in the reference).
__device__ __forceinline__ float lsf_rate(const Phys& P, float f) { return (float)((double)(f * P.lsfFac) / 3600.0); }
// Vertical difference of the slab-mean ratio <rho phi>/<rho> between levels k+1 and k-1.
__device__ __forceinline__ float lsf_dmean(const float* prof, int nzh, int f, int k) {
  return prof[f * nzh + k + 1] / prof[k + 1] - prof[f * nzh + k - 1] / prof[k - 1];
}
// Large-scale forcing of one interior cell (cuda_largeScaleForcingsDevice.cu:155-252): theta and
// q_v tendencies, then the subsidence terms -w_ls rho d<phi>/dz of u, v, theta and q_v from the
// slab means (w_ls already carries rho, so rho enters twice, as in the reference).
// Fu/Fv/Fth/Fqv are the cell's tendencies of rho u, rho v, rho theta, rho q_v.
__device__ __forceinline__ void lsf_tend(const Phys& P, const Ptrs& Q, long long c, int k, float z, float rho,
                                         float& Fu, float& Fv, float& Fth, float& Fqv) {
  Fth = Fth + lsf_rate(P, lsf_profile(P.lsfTh, z, rho));
  if (P.moist) Fqv = Fqv + lsf_rate(P, lsf_profile(P.lsfQv, z, rho));
  if (P.lsfSub) {
    const float fw = lsf_rate(P, lsf_profile(P.lsfW, z, rho));
    const float dz = Q.zPos[c + 1] - Q.zPos[c - 1];
    const float* pr = Q.lsfProf;
    Fu = Fu - fw * rho * lsf_dmean(pr, P.nzh, 1, k) / dz;
    Fv = Fv - fw * rho * lsf_dmean(pr, P.nzh, 2, k) / dz;
    Fth = Fth - fw * rho * lsf_dmean(pr, P.nzh, 3, k) / dz;
    if (P.moist) Fqv = Fqv - fw * rho * lsf_dmean(pr, P.nzh, 4, k) / dz;
  }
}

// 6th-order vertical filter of rho w (cuda_filtersDevice.cu:73-122; Xue 2000, Knievel et al.
// 2007), stencil s[k-3..k+3] as m3..p3: face fluxes 10 d1 - 5 d3 + d5 at k-1/2 and k+1/2, each
// kept only where its product with the face's first difference is not negative (the reference's
// fmaxf(copysign(1, grad), 0): a product of -0 also drops it), scaled by `coef` =
// 0.015625 filter_6th_coeff / dt.
__device__ __forceinline__ float filter6_tend(float m3, float m2, float m1, float z0, float p1, float p2, float p3,
                                              float coef) {
  const float dm = __fsub_rn(z0, m1), dp = __fsub_rn(p1, z0);
  float fm = __fadd_rn(__fmaf_rn(-5.0f, __fsub_rn(p1, m2), __fmul_rn(10.0f, dm)), __fsub_rn(p2, m3));
  float fp = __fadd_rn(__fmaf_rn(-5.0f, __fsub_rn(p2, m1), __fmul_rn(10.0f, dp)), __fsub_rn(p3, m2));
  if (signbit(__fmul_rn(dm, fm))) fm = 0.0f;
  if (signbit(__fmul_rn(dp, fp))) fp = 0.0f;
  return __fmul_rn(coef, __fsub_rn(fp, fm));
}

// Face velocities of a cell: lower/upper faces in x, y, z (cuda_advectionDevice.cu:54-121).
struct FaceVel {
  float um, up, vm, vp, wm, wp;
};

// Contravariant momentum term (D/rho)*(m + w*J) of one cell, as in the reference sum.
__device__ __forceinline__ float contra(float D, float r, float m, float w, float J) {
  return __fmul_rn(__fdiv_rn(D, r), __fmaf_rn(w, J, m));
}
// The same with D/rho already formed (one division shared by the three directions).
__device__ __forceinline__ float contra_dr(float dr, float m, float w, float J) { return __fmul_rn(dr, __fmaf_rn(w, J, m)); }
__device__ __forceinline__ float contra_z_dr(float dr, float w, float J) { return __fmul_rn(dr, __fmul_rn(w, J)); }
// Its vertical form (D/rho)*(w*J33).
__device__ __forceinline__ float contra_z(float D, float r, float w, float J) {
  return __fmul_rn(__fdiv_rn(D, r), __fmul_rn(w, J));
}

}  // namespace fe
