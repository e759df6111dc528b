// fe_kernels.cuh -- CUDA kernels of the hot path (sm_100a).
//
//   k_consts      device-evaluated constants c1 = R/p0^(R/cp) and (p0/p_grnd)^(R/cp)
//   k_pbs         powf(thBS*c1, cp/cv) per cell (the base-state pressure term of p')
//   k_fill        boundary values of every halo cell of a state block (gather form)
//   k_pressure    perturbation pressure of a state block, halo-inclusive
//   k_turb        last-stage SGS physics on the +1 ring: strain, length scale, Km, stresses,
//                 TKE transport fluxes, moisture SGS fluxes, surface layer
//   k_stage       fused tendency + WS2002 RK3 commit of one stage; writes the next state
//                 with its halo images and its perturbation pressure (or, in Frhs mode,
//                 writes the tendency only)
//   k_clock       advance the device simulation clock after the last stage
//   k_nonfinite, k_means   device reductions (NaN/Inf count, FP64 domain means)
//   k_slab_partial, k_slab_final   FP64 slab means of the large-scale subsidence terms
#pragma once
#include "fe_device.cuh"
#include "fe_sgs.cuh"

namespace fe {

constexpr int MODE_COMMIT = 0;
constexpr int MODE_FRHS = 1;

static __global__ void k_consts(float R_gas, float p0, float R_cp, float presGrnd, float* out) {
  out[0] = R_gas / powf(p0, R_cp);
  out[1] = powf((p0 / presGrnd), R_cp);
}

static __global__ void k_delta(Phys P, long long n, const float* __restrict__ D, float* __restrict__ delta) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) delta[t] = grid_scale_of(P, D[t]);
}

static __global__ void k_pbs(long long n, const float* __restrict__ thBS, float c1, float cp_cv, float* __restrict__ pBS) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) pBS[t] = powf(thBS[t] * c1, cp_cv);
}

// Source column of a halo column: its periodic image, or itself in a direction whose halos the
// neighbouring slabs provide.
__device__ __forceinline__ int wrap_i(const Phys& P, int i) {
  return P.peerX ? i : (i < P.iMin ? i + P.Nx : (i >= P.iMax ? i - P.Nx : i));
}
__device__ __forceinline__ int wrap_j(const Phys& P, int j) {
  return P.peerY ? j : (j < P.jMin ? j + P.Ny : (j >= P.jMax ? j - P.Ny : j));
}

// Boundary value of field f at halo cell (i,j,k): the vertical boundary rule applied on
// the periodic source column, i.e. the reference's Commence BCs (cuda_hydroCoreDevice.cu:
// 469-550) with every read of the current stage.
static __global__ void k_fill(Phys P, Ptrs Q, float* st) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n) return;
  const int k = (int)(t % P.nzh);
  const int j = (int)((t / P.nzh) % P.nyh);
  const int i = (int)(t / ((long long)P.nzh * P.nyh));
  const bool inI = i >= P.iMin && i < P.iMax, inJ = j >= P.jMin && j < P.jMax, inK = k >= P.kMin && k < P.kMax;
  if (inI && inJ && inK) return;
  const int is = wrap_i(P, i), js = wrap_j(P, j);
  const long long col = (long long)is * P.si + (long long)js * P.sj;
  const long long src = col + k;
  const long long bot = col + P.kMin, top = col + P.kMax - 1;
  for (int f = 0; f < P.nf; f++) {
    float* F = st + (long long)f * P.n;
    float v;
    if (inK) {
      v = F[src];
    } else {
      const bool below = k < P.kMin;
      if (f == 0) v = Q.rhoBS[src];
      else if (f == 4) v = Q.thBS[src];
      else if (f <= 3) v = below ? F[bot] : momentum_bs(P, f, Q.zPos[top], Q.rhoBS[top]);
      else if (f == 5 && P.ntke) v = below ? F[bot] : 0.0f;
      else v = below ? F[bot] : F[top];
    }
    F[t] = v;
  }
}

// Perturbation pressure over the halo-inclusive block (cuda_pressureDevice.cu:53-113):
// levels 1..kMin-1 use the kMin cell, levels >= kMax use kMax-1, level 0 its own cell.
static __global__ void k_pressure(Phys P, Ptrs Q, const float* __restrict__ st, float* __restrict__ pres) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P.n) return;
  const int k = (int)(t % P.nzh);
  long long src = t;
  if (k > 0 && k < P.kMin) src = t - k + P.kMin;
  else if (k >= P.kMax) src = t - k + P.kMax - 1;
  pres[t] = pert_pressure(P, st, Q.pBS, src);
}

// SGS length scale at cell c + dk (cuda_sgstkeDevice.cu:96-151), from primitives.
// The metric terms and grid scale of one point (the values the SGS helpers below read at c).
struct PointMetrics {
  float J1, J2, J3, delta;
};
__device__ __forceinline__ PointMetrics point_metrics(const Phys& P, const Ptrs& Q, long long c) {
  return {Q.J31[c], Q.J32[c], Q.J33[c], grid_scale(P, Q, c)};
}

template <class A>
__device__ __forceinline__ float length_scale_m(const Phys& P, const A& pr, int dk, const PointMetrics& m) {
  const float dthdz = (float)(0.5 * (double)((m.J1 * P.dXi * (pr.th(1, 0, dk) - pr.th(-1, 0, dk))) +
                                             (m.J2 * P.dYi * (pr.th(0, 1, dk) - pr.th(0, -1, dk))) +
                                             (m.J3 * P.dZi * (pr.th(0, 0, dk + 1) - pr.th(0, 0, dk - 1)))));
  const float N2 = (P.g / pr.th(0, 0, dk)) * dthdz;
  const float len2 = m.delta;
  if (N2 > 0.0f) {
    const float tb = 1.0f / sqrtf(N2);  // N2^(-1/2): two correctly rounded operations
    const float ec = pr.ev(0, 0, dk);
    const float len1 = (float)(0.76 * (double)sqrtf(ec) * (double)tb);
    return fmaxf(fminf(len1, len2), 1e-2f);
  }
  return len2;
}

template <class A>
__device__ __forceinline__ float length_scale_a(const Phys& P, const Ptrs& Q, const A& pr, long long c, int dk) {
  return length_scale_m(P, pr, dk, point_metrics(P, Q, c));
}

__device__ __forceinline__ float length_scale(const Phys& P, const Ptrs& Q, const float* __restrict__ rho,
                                              const float* __restrict__ th, const float* __restrict__ e, long long c) {
  GlobalPrims pr{rho, nullptr, nullptr, nullptr, th, e, nullptr, P.n, c, P.si, P.sj};
  return length_scale_a(P, Q, pr, c, 0);
}

// ------------------------------------------------------------------ surface layer
// Land-surface update and Monin-Obukhov iteration of one column (cuda_surfaceLayerDevice.cu:
// 112-521). Writes tau31, tau32, tauTH3 (and the q_v flux) at kMin.
static __device__ void surface_column(const Phys& P, const Ptrs& Q, const float* __restrict__ st, int i, int j, int stage) {
  const long long c = (long long)i * P.si + (long long)j * P.sj + P.kMin;
  const long long ij = (long long)i * P.nyh + j;
  const bool moist = P.moist > 0 && P.nmoist > 0;
  const float pi = acosf(-1.0f);
  const int it = *Q.clockIt;
  const float simTime = *Q.clockTime;
  const float* rho = st;
  const float r = rho[c], mu = st[P.n + c], mv = st[2 * P.n + c], mth = st[4 * P.n + c];
  const float mq = moist ? st[(long long)(5 + P.ntke) * P.n + c] : 0.0f;
  float z0 = Q.z0m[ij];
  float z1 = 0.5f / (P.dZi * Q.J33[c]);
  float z1oz0 = (z1 + z0) / z0;
  float z0t = Q.z0t[ij];
  float z1ozt0 = (z1 + z0t) / z0t;
  float u1 = mu / r, v1 = mv / r;
  float U1 = sqrtf(powf(u1, 2.0f) + powf(v1, 2.0f));
  float th1 = mth / r;
  float q1 = mq / r;
  float qsk_input = moist ? Q.qskin[ij] : 0.0f;
  // ---- LSM
  if (it == P.itRestart && it == 0) {
    Q.cd[ij] = powf(P.kappa, 2.0f) / powf(logf(z1oz0), 2.0f);
    Q.ch[ij] = powf(P.kappa, 2.0f) / powf(logf(z1ozt0), 2.0f);
    if (moist) Q.cq[ij] = powf(P.kappa, 2.0f) / powf(logf(z1ozt0), 2.0f);
  } else if (it == P.itRestart && it != 0) {
    Q.cd[ij] = powf(Q.fricVel[ij], 2.0f) / (powf(U1, 2.0f));
    float th0 = Q.tskin[ij] * P.presFac;
    Q.ch[ij] = Q.htFlux[ij] / (U1 * (th0 - th1));
    if (moist) Q.cq[ij] = Q.qFlux[ij] / (U1 * (Q.qskin[ij] - q1));
  }
  if (P.surf == 1) {
    if (P.idealSine == 1) {
      if ((simTime > P.idealTs) && (simTime <= P.idealTe))
        Q.htFlux[ij] = (float)(P.wth + P.idealAmp * sin(pi * (simTime - P.idealTs) / (P.idealTe - P.idealTs)));
      else
        Q.htFlux[ij] = P.wth;
      if (moist) {
        if ((simTime > P.idealQts) && (simTime <= P.idealQte))
          Q.qFlux[ij] = (float)(P.idealQamp * sin(pi * (simTime - P.idealQts) / (P.idealQte - P.idealQts)));
        else
          Q.qFlux[ij] = P.wq;
      }
    }
  } else if (P.surf == 2) {
    const float tff = (float)P.tempFreq;
    float tsk_c, qsk_c = 0.0f;
    if ((it % P.tempFreq == 0) && (stage == 2)) {
      if (P.idealSine == 1 && (simTime > P.idealTs) && (simTime < P.idealTe + P.dt * tff)) {
        float prev = fmaxf(simTime - tff * P.dt, P.idealTs);
        float inc = (float)(P.idealAmp * (sin(pi * (simTime - P.idealTs) / (P.idealTe - P.idealTs)) -
                                          sin(pi * (prev - P.idealTs) / (P.idealTe - P.idealTs))));
        tsk_c = Q.tskin[ij] + inc;
        if (moist) {
          float qinc = (float)(P.idealQamp * (sin(pi * (simTime - P.idealQts) / (P.idealQte - P.idealQts)) -
                                              sin(pi * (prev - P.idealQts) / (P.idealQte - P.idealQts))));
          qsk_c = Q.qskin[ij] + qinc;
        }
      } else {
        tsk_c = (float)(Q.tskin[ij] + P.tr * P.dt * tff / 3600.0);
        if (moist) qsk_c = (float)(Q.qskin[ij] + P.qr * P.dt * tff / 3600.0);
      }
      Q.tskin[ij] = tsk_c;
      if (moist) Q.qskin[ij] = qsk_c;
    } else {
      tsk_c = Q.tskin[ij];
      if (moist) qsk_c = Q.qskin[ij];
    }
    float th0 = tsk_c * P.presFac;
    Q.htFlux[ij] = Q.ch[ij] * U1 * (th0 - th1);
    if (moist) {
      Q.qFlux[ij] = Q.cq[ij] * U1 * (qsk_c - q1);
      if (P.qskinInput == 1) Q.qskin[ij] = qsk_input;
    }
  }
  // ---- MOST
  {
    const float beta = 5.0f, ol_lim = 1.0f;
    const int it_max = P.surfStab == 0 ? 5 : 1;
    int it_n = 0;
    float th0 = Q.tskin[ij] * P.presFac;
    float q0 = moist ? Q.qskin[ij] : 0.0f;
    float cd0 = Q.cd[ij], cd_i = 0.0f, ch_i = 0.0f, cq_i = 0.0f;
    float fv = Q.fricVel[ij], iol = Q.invOblen[ij], hf = Q.htFlux[ij], qf = moist ? Q.qFlux[ij] : 0.0f;
    do {
      float tauxz = -cd0 * U1 * u1;
      float tauyz = -cd0 * U1 * v1;
      fv = powf(powf(tauxz, 2.0f) + powf(tauyz, 2.0f), 0.25f);
      it_n = it_n + 1;
      if (P.surfStab == 0) {
        if (fv > 0.0f) {
          iol = -(P.kappa * P.g * hf) / (powf(fv, 3.0f) * th1);
          iol = fmaxf(fminf(iol, ol_lim), -ol_lim);
        } else {
          iol = -ol_lim;
        }
      } else {
        iol = 0.0f;
      }
      float zol = iol * (z1 + z0);
      float psi_m, psi_h;
      if (zol < 0.0f) {
        float xi = powf(1.0f - 16.0f * zol, 0.25f);
        psi_m = (float)(logf(0.5f * (1.0f + powf(xi, 2.0f)) * powf(0.5f * (1.0f + xi), 2.0f)) - 2.0f * atanf(xi) + 0.5f * pi);
        psi_h = 2.0f * logf(0.5f * (1.0f + powf(xi, 2.0f)));
      } else {
        psi_m = -beta * zol;
        psi_h = -beta * zol;
      }
      cd_i = powf(P.kappa, 2.0f) / powf(logf(z1oz0) - psi_m, 2.0f);
      ch_i = powf(P.kappa, 2.0f) / ((logf(z1ozt0) - psi_m) * (logf(z1ozt0) - psi_h));
      cq_i = powf(P.kappa, 2.0f) / ((logf(z1ozt0) - psi_m) * (logf(z1ozt0) - psi_h));
      if (P.surf > 1) {
        hf = ch_i * U1 * (th0 - th1);
        if (moist) qf = cq_i * U1 * (q0 - q1);
      }
      cd0 = cd_i;
    } while (it_n <= it_max);
    Q.cd[ij] = cd_i;
    Q.ch[ij] = ch_i;
    if (moist) Q.cq[ij] = cq_i;
    float tauxz = -cd_i * sqrtf(powf(mu / r, 2.0f) + powf(mv / r, 2.0f)) * mu;
    float tauyz = -cd_i * sqrtf(powf(mu / r, 2.0f) + powf(mv / r, 2.0f)) * mv;
    Q.tau[2 * P.n + c] = tauxz;
    Q.tau[3 * P.n + c] = tauyz;
    fv = powf(powf(tauxz, 2.0f) + powf(tauyz, 2.0f), 0.25f);
    Q.tau[8 * P.n + c] = hf * r;
    if (moist && P.moistSGS > 0) Q.mtau[2 * P.n + c] = qf * r;
    iol = -(P.kappa * P.g * hf) / (powf(fv, 3.0f) * th1);
    Q.fricVel[ij] = fv;
    Q.invOblen[ij] = iol;
    Q.htFlux[ij] = hf;
    if (moist) Q.qFlux[ij] = qf;
  }
}

// ------------------------------------------------------------------ last-stage SGS physics
// The SGS physics of one ring point: the 9 stresses and heat fluxes (hydroTauFlds order), the
// TKE transport fluxes (de/dx_j) Km rho, the moisture SGS fluxes (3 per species) and the length
// scale. Computed at every level by turb_point(); the stresses and the stress-like moisture
// fluxes are the closure's only at k >= kMin (at lower levels: stresses untouched = 0, moisture
// fluxes the raw gradients, tke fluxes 0, as the reference's kernels leave them).
struct TurbOut {
  float tau[9];
  float tkeQ[3];
  float mtau[6];
  float ls;
};

// SGS physics of ring point c = (i,j,k), given the length scale of the cell (lsc) and of the level
// below (lsm) and sqrt(e/rho) of the level below (sem) and of the cell (sec; < 0: computed here),
// all 0 without prognostic TKE; the neighbours' primitive variables come from accessor `pr` (state
// or a shared-memory tile).
template <class A>
__device__ __forceinline__ void turb_point_m(const Phys& P, const A& pr, int k, float lsc, float lsm, float sem,
                                             float sec, const PointMetrics& mt, TurbOut& o);
template <class A>
__device__ __forceinline__ void turb_point(const Phys& P, const Ptrs& Q, const A& pr, long long c, int k, float lsc,
                                           float lsm, float sem, float sec, TurbOut& o) {
  turb_point_m(P, pr, k, lsc, lsm, sem, sec, point_metrics(P, Q, c), o);
}
// turb_point() with the point's metric terms and grid scale given.
template <class A>
__device__ __forceinline__ void turb_point_m(const Phys& P, const A& pr, int k, float lsc, float lsm, float sem,
                                             float sec, const PointMetrics& mt, TurbOut& o) {
#pragma unroll
  for (int t = 0; t < 9; t++) o.tau[t] = 0.0f;
#pragma unroll
  for (int t = 0; t < 3; t++) o.tkeQ[t] = 0.0f;
#pragma unroll
  for (int t = 0; t < 6; t++) o.mtau[t] = 0.0f;
  o.ls = lsc;
  float Km = 0.0f;
  const float delta = mt.delta;
  if (k >= P.kMin) {
    const float J1 = mt.J1, J2 = mt.J2, J3 = mt.J3;
    const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
    // c, a = i-1, b = j-1, d = k-1 and their combinations
    const float uc = pr.u(0, 0, 0), ua = pr.u(-1, 0, 0), ub = pr.u(0, -1, 0), ud = pr.u(0, 0, -1);
    const float uab = pr.u(-1, -1, 0), uad = pr.u(-1, 0, -1), ubd = pr.u(0, -1, -1), uabd = pr.u(-1, -1, -1);
    const float vc = pr.v(0, 0, 0), va = pr.v(-1, 0, 0), vb = pr.v(0, -1, 0), vd = pr.v(0, 0, -1);
    const float vab = pr.v(-1, -1, 0), vad = pr.v(-1, 0, -1), vbd = pr.v(0, -1, -1), vabd = pr.v(-1, -1, -1);
    const float wc = pr.w(0, 0, 0), wa = pr.w(-1, 0, 0), wb = pr.w(0, -1, 0), wd = pr.w(0, 0, -1);
    const float wad = pr.w(-1, 0, -1), wbd = pr.w(0, -1, -1);
    const float thc = pr.th(0, 0, 0), tha = pr.th(-1, 0, 0), thb = pr.th(0, -1, 0), thd = pr.th(0, 0, -1);
    float S11 = dXi * (uc - ua);
    float S22 = dYi * (vc - vb);
    float S33 = J1 * dXi * (wc - wa) + J2 * dYi * (wc - wb) + J3 * dZi * (wc - wd);
    float S21 = 0.5f * (0.5f * (dXi * (vc - va) + dXi * (vb - vab)) + 0.5f * (dYi * (uc - ub) + dYi * (ua - uab)));
    float S31 = 0.5f * (0.5f * (dXi * (wc - wa) + dXi * (wd - wad)) + 0.5f * (J1 * dXi * (uc - ua) + J1 * dXi * (ud - uad)) +
                        0.25f * (J2 * dYi * (uc - ub) + J2 * dYi * (ua - uab) + J2 * dYi * (ud - ubd) + J2 * dYi * (uad - uabd)) +
                        0.5f * (J3 * dZi * (uc - ud) + J3 * dZi * (ua - uad)));
    float S32 = 0.5f * (0.5f * (dYi * (wc - wb) + dYi * (wd - wbd)) +
                        0.25f * (J1 * dXi * (vc - va) + J1 * dXi * (vb - vab) + J1 * dXi * (vd - vad) + J1 * dXi * (vbd - vabd)) +
                        0.5f * (J2 * dYi * (vc - vb) + J2 * dYi * (vd - vbd)) + 0.5f * (J3 * dZi * (vc - vd) + J3 * dZi * (vb - vbd)));
    float ST1 = dXi * (thc - tha);
    float ST2 = dYi * (thc - thb);
    float ST3 = (J1 * dXi * (thc - tha)) + (J2 * dYi * (thc - thb)) + (J3 * dZi * (thc - thd));
    const float r = pr.r(0, 0, 0);
    if (P.tke) {
      const float e0 = pr.ev(0, 0, 0);
      const float se0 = sec >= 0.0f ? sec : sqrtf(e0);  // sqrt(e/rho) of this cell (given by the tiled form)
      Km = (float)((double)P.c_k * 0.5 * (double)(lsc * se0 + lsm * sem));
      const float invPr = 1.0f + 2.0f * lsc / delta;
      const float dev = (float)((2.0 / 3.0) * (double)r *
                                (double)(Km * (dXi * (uc - ua) + dYi * (vc - vb) + J1 * dXi * (wc - wa) +
                                               J2 * dYi * (wc - wb) + J3 * dZi * (wc - wd)) +
                                         e0));
      o.tau[0] = -2.0f * r * Km * S11 + dev;
      o.tau[1] = -2.0f * r * Km * S21;
      o.tau[4] = -2.0f * r * Km * S22 + dev;
      o.tau[5] = -2.0f * r * Km * S33 + dev;
      o.tau[6] = -r * Km * invPr * ST1;
      o.tau[7] = -r * Km * invPr * ST2;
      o.tau[2] = -2.0f * r * Km * S31;
      o.tau[3] = -2.0f * r * Km * S32;
      o.tau[8] = -r * Km * invPr * ST3;
    } else {
      const float t1 = 0.5f * (S11 * S11 + S22 * S22 + S33 * S33) + S21 * S21 + S31 * S31 + S32 * S32;
      const float N2 = P.g / thc * ST3;
      const float t2 = N2 * 3.0f;
      Km = (P.c_s * delta) * (P.c_s * delta) * sqrtf(fmaxf(0.0f, t1 - fmaxf(0.0f, t2)));
      const float invPr = 1.0f + 2.0f * delta / delta;
      o.tau[0] = -2.0f * r * Km * S11;
      o.tau[1] = -2.0f * r * Km * S21;
      o.tau[4] = -2.0f * r * Km * S22;
      o.tau[5] = -2.0f * r * Km * S33;
      o.tau[6] = -r * Km * invPr * ST1;
      o.tau[7] = -r * Km * invPr * ST2;
      o.tau[2] = -2.0f * r * Km * S31;
      o.tau[3] = -2.0f * r * Km * S32;
      o.tau[8] = -r * Km * invPr * ST3;
    }
  }
  if (P.tke) {
    // TKE transport fluxes (de/dx_j)*Km*rho (cuda_sgstkeDevice.cu:309-397), Km = 0 below kMin
    const float ex = pr.ev(1, 0, 0) - pr.ev(-1, 0, 0);
    const float ey = pr.ev(0, 1, 0) - pr.ev(0, -1, 0);
    const float ez = pr.ev(0, 0, 1) - pr.ev(0, 0, -1);
    const float dedx = 0.5f * (P.dXi * ex);
    const float dedy = 0.5f * (P.dYi * ey);
    const float dedz = 0.5f * (mt.J1 * P.dXi * ex + mt.J2 * P.dYi * ey + mt.J3 * P.dZi * ez);
    const float rc = pr.r(0, 0, 0);
    o.tkeQ[0] = dedx * Km * rc;
    o.tkeQ[1] = dedy * Km * rc;
    o.tkeQ[2] = dedz * Km * rc;
  }
  if (P.moist && P.moistSGS > 0) {
    const float invPr = 1.0f + 2.0f * (P.tke ? lsc : delta) / delta;
    const float rc = pr.r(0, 0, 0);
    for (int m = 0; m < P.nmoist && m < 2; m++) {
      const float qc = pr.qm(m, 0, 0, 0), qa = pr.qm(m, -1, 0, 0);
      const float qb = pr.qm(m, 0, -1, 0), qd = pr.qm(m, 0, 0, -1);
      float g1 = P.dXi * (qc - qa);
      float g2 = P.dYi * (qc - qb);
      float g3 = mt.J1 * P.dXi * (qc - qa) + mt.J2 * P.dYi * (qc - qb) + mt.J3 * P.dZi * (qc - qd);
      if (k >= P.kMin) {
        g1 = -rc * Km * invPr * g1;
        g2 = -rc * Km * invPr * g2;
        g3 = -rc * Km * invPr * g3;
      }
      o.mtau[3 * m + 0] = g1;
      o.mtau[3 * m + 1] = g2;
      o.mtau[3 * m + 2] = g3;
    }
  }
}

// SGS physics of ring cell (i,j,k) stored to the scratch fields (turb_point), plus the learned
// closure's inputs when a network is set and, with SURF, the surface layer of a first-level cell.
// Without SURF (the surface layer in its own kernel) the first-level tau31, tau32, tauTH3 and q_v
// flux of the surface columns are that kernel's: this cell leaves them alone.
template <class A, bool SURF = true>
__device__ __forceinline__ void turb_cell_a(const Phys& P, const Ptrs& Q, const A& pr, const float* __restrict__ st, int i,
                                            int j, int k, float lsc, float lsm, float sem, float sec, int stage) {
  const long long n = P.n;
  const long long c = (long long)i * P.si + (long long)j * P.sj + k;
  const bool surfCell = !SURF && P.surf > 0 && k == P.kMin && i >= P.iMin && j >= P.jMin;
  if (P.turb) {
    TurbOut o;
    turb_point(P, Q, pr, c, k, lsc, lsm, sem, sec, o);
    float* T = Q.tau;
    if (k >= P.kMin) {
      T[c] = o.tau[0];
      T[n + c] = o.tau[1];
      T[4 * n + c] = o.tau[4];
      T[5 * n + c] = o.tau[5];
      T[6 * n + c] = o.tau[6];
      T[7 * n + c] = o.tau[7];
      if (!surfCell) {
        T[2 * n + c] = o.tau[2];
        T[3 * n + c] = o.tau[3];
        T[8 * n + c] = o.tau[8];
      }
    }
    if (Q.feat && k >= P.kMin) {
      // inputs of the learned closure at this stress point, for its time-step kernel
      float x[SGS_NIN];
      sgs_inputs_a(P, Q, pr, c, x);
#pragma unroll
      for (int q = 0; q < SGS_NIN; q++) Q.feat[q * n + c] = x[q];
    }
    if (P.tke) {
      Q.ls[c] = lsc;
      Q.tkeQ[c] = o.tkeQ[0];
      Q.tkeQ[n + c] = o.tkeQ[1];
      Q.tkeQ[2 * n + c] = o.tkeQ[2];
    }
    if (P.moist && P.moistSGS > 0) {
      for (int m = 0; m < P.nmoist && m < 2; m++) {
        Q.mtau[(3 * m + 0) * n + c] = o.mtau[3 * m + 0];
        Q.mtau[(3 * m + 1) * n + c] = o.mtau[3 * m + 1];
        if (!(surfCell && m == 0)) Q.mtau[(3 * m + 2) * n + c] = o.mtau[3 * m + 2];
      }
    }
  }
  if (SURF && P.surf > 0 && k == P.kMin && i >= P.iMin && j >= P.jMin) surface_column(P, Q, st, i, j, stage);
}

__device__ __forceinline__ void turb_cell(const Phys& P, const Ptrs& Q, const float* __restrict__ st, int i, int j, int k,
                                          float lsc, float lsm, float sem, int stage) {
  const long long n = P.n;
  GlobalPrims pr{st, st + n, st + 2 * n, st + 3 * n, st + 4 * n, P.ntke ? st + 5 * n : nullptr,
                 P.nmoist ? st + (5 + P.ntke) * n : nullptr, n, (long long)i * P.si + (long long)j * P.sj + k, P.si, P.sj};
  turb_cell_a(P, Q, pr, st, i, j, k, lsc, lsm, sem, -1.0f, stage);
}

// One thread per cell of the ring i in [iMin-1,iMax], j in [jMin-1,jMax], k in [kMin-1,kMax]
// (the reference's ring minus the i=iMax+1/j=jMax+1 cells, which nothing reads). The length
// scale of the level below is recomputed by the same thread (no race on it).
static __global__ void __launch_bounds__(256) k_turb(Phys P, Ptrs Q, const float* __restrict__ st, int stage) {
  const int k = P.kMin - 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = P.jMin - 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = P.iMin - 1 + blockIdx.z * blockDim.z + threadIdx.z;
  if (k > P.kMax || j > P.jMax || i > P.iMax) return;
  float lsc = 0.0f, lsm = 0.0f, sem = 0.0f;
  if (P.turb && P.tke) {
    const long long c = (long long)i * P.si + (long long)j * P.sj + k;
    const float *rho = st, *mth = st + 4 * P.n, *e = st + 5 * P.n;
    lsc = length_scale(P, Q, rho, mth, e, c);
    if (k >= P.kMin) {
      lsm = length_scale(P, Q, rho, mth, e, c - 1);
      sem = sqrtf(e[c - 1] * rinv(rho[c - 1]));
    }
  }
  turb_cell(P, Q, st, i, j, k, lsc, lsm, sem, stage);
}

// The same ring in tiles of 32 levels x 4 rows x 2 planes per block of 256 threads, over the
// interior levels [kMin, kMax) (so a warp's 32 lanes are 32 levels of one column and columns of
// 32k levels fill every lane); the ring level kMax goes to k_turb_ring. The block
// first forms the primitive variables (phi * rinv(rho), the same expression the per-cell form
// evaluates) of the tile and its stencil halo once into shared memory, then the length scale and
// sqrt(e/rho) of every tile column including the level below the tile, then each thread runs
// the SGS physics of its cell on the shared copies. Results equal the per-cell form's bit for bit.
constexpr int TT_K = 32, TT_J = 4, TT_I = 2;
constexpr int TP_K = TT_K + 3, TP_J = TT_J + 2, TP_I = TT_I + 2;  // points k0-2..k0+32, j0-1..j0+4, i0-1..i0+2
constexpr int TP_N = TP_I * TP_J * TP_K;
constexpr int TP_F = 8;  // rho, u, v, w, theta, e/rho, qv/rho, ql/rho

struct TilePrims {
  const float* t;
  int o;  // own point
  __device__ __forceinline__ float at(int f, int di, int dj, int dk) const { return t[f * TP_N + o + di * (TP_J * TP_K) + dj * TP_K + dk]; }
  __device__ __forceinline__ float r(int di, int dj, int dk) const { return at(0, di, dj, dk); }
  __device__ __forceinline__ float u(int di, int dj, int dk) const { return at(1, di, dj, dk); }
  __device__ __forceinline__ float v(int di, int dj, int dk) const { return at(2, di, dj, dk); }
  __device__ __forceinline__ float w(int di, int dj, int dk) const { return at(3, di, dj, dk); }
  __device__ __forceinline__ float th(int di, int dj, int dk) const { return at(4, di, dj, dk); }
  __device__ __forceinline__ float ev(int di, int dj, int dk) const { return at(5, di, dj, dk); }
  __device__ __forceinline__ float qm(int m, int di, int dj, int dk) const { return at(6 + m, di, dj, dk); }
};

static __global__ void __launch_bounds__(256) k_turb_t(Phys P, Ptrs Q, const float* __restrict__ st, int stage) {
  __shared__ float tile[TP_F * TP_N];
  __shared__ float lsT[TT_I][TT_J][TT_K + 1];  // length scale, levels k0-1..k0+31
  __shared__ float seT[TT_I][TT_J][TT_K + 1];  // sqrt(e/rho), same levels
  const int tx = threadIdx.x, ty = threadIdx.y, tz = threadIdx.z;
  const int tid = (tz * TT_J + ty) * TT_K + tx;
  const int k0 = P.kMin + blockIdx.x * TT_K, j0 = P.jMin - 1 + blockIdx.y * TT_J, i0 = P.iMin - 1 + blockIdx.z * TT_I;
  const long long n = P.n;
  for (int p = tid; p < TP_N; p += TT_K * TT_J * TT_I) {
    const int pk = p % TP_K, pj = (p / TP_K) % TP_J, pi = p / (TP_K * TP_J);
    const int i = i0 - 1 + pi, j = j0 - 1 + pj, k = k0 - 2 + pk;  // >= 1, >= 1, >= 1
    float v[TP_F] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (i < P.nxh && j < P.nyh && k < P.nzh) {
      const long long c = (long long)i * P.si + (long long)j * P.sj + k;
      const float rr = st[c];
      const float ri = rinv(rr);
      v[0] = rr;
      v[1] = st[n + c] * ri;
      v[2] = st[2 * n + c] * ri;
      v[3] = st[3 * n + c] * ri;
      v[4] = st[4 * n + c] * ri;
      if (P.ntke) v[5] = st[5 * n + c] * ri;
      if (P.nmoist > 0) v[6] = st[(long long)(5 + P.ntke) * n + c] * ri;
      if (P.nmoist > 1) v[7] = st[(long long)(6 + P.ntke) * n + c] * ri;
    }
#pragma unroll
    for (int f = 0; f < TP_F; f++) tile[f * TP_N + p] = v[f];
  }
  __syncthreads();
  const bool tke = P.turb && P.tke;
  if (tke) {
    for (int q = tid; q < TT_I * TT_J * (TT_K + 1); q += TT_K * TT_J * TT_I) {
      const int lk = q % (TT_K + 1), lj = (q / (TT_K + 1)) % TT_J, li = q / ((TT_K + 1) * TT_J);
      const int i = i0 + li, j = j0 + lj, k = k0 - 1 + lk;
      float ls = 0.0f, se = 0.0f;
      if (i <= P.iMax && j <= P.jMax && k >= 1 && k <= P.kMax) {
        const long long c = (long long)i * P.si + (long long)j * P.sj + k;
        const TilePrims pr{tile, (li + 1) * (TP_J * TP_K) + (lj + 1) * TP_K + (lk + 1)};
        ls = length_scale_a(P, Q, pr, c, 0);
        se = sqrtf(pr.ev(0, 0, 0));
      }
      lsT[li][lj][lk] = ls;
      seT[li][lj][lk] = se;
    }
    __syncthreads();
  }
  const int i = i0 + tz, j = j0 + ty, k = k0 + tx;
  if (i > P.iMax || j > P.jMax || k >= P.kMax) return;
  const TilePrims pr{tile, (tz + 1) * (TP_J * TP_K) + (ty + 1) * TP_K + (tx + 2)};
  const bool below = tke && k >= P.kMin;
  turb_cell_a<TilePrims, false>(P, Q, pr, st, i, j, k, tke ? lsT[tz][ty][tx + 1] : 0.0f, below ? lsT[tz][ty][tx] : 0.0f,
              below ? seT[tz][ty][tx] : 0.0f, tke ? seT[tz][ty][tx + 1] : -1.0f, stage);
}

// The ring level above k_turb_t's columns, k = kMax, one thread per cell on the per-cell path
// (global primitives, the length scale of the cell and of the level below recomputed; the same
// arithmetic as the tiled form). The ring level below, k = kMin - 1, is not computed: there the
// eddy viscosity is zero by construction, so of its outputs only the vertical TKE flux is ever
// read (by the transport term of the first level) and it is zero, which the zero-initialised
// scratch already holds; its moisture gradients and length scale have no reader.
static __global__ void __launch_bounds__(256) k_turb_ring(Phys P, Ptrs Q, const float* __restrict__ st, int stage) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nj = P.Ny + 2;
  if (t >= (long long)nj * (P.Nx + 2)) return;
  const int j = P.jMin - 1 + (int)(t % nj);
  const int i = P.iMin - 1 + (int)(t / nj);
  const int k = P.kMax;
  const long long n = P.n;
  const long long c = (long long)i * P.si + (long long)j * P.sj + k;
  float lsc = 0.0f, lsm = 0.0f, sem = 0.0f;
  if (P.turb && P.tke) {
    const float *rho = st, *mth = st + 4 * n, *e = st + 5 * n;
    lsc = length_scale(P, Q, rho, mth, e, c);
    if (k >= P.kMin) {
      lsm = length_scale(P, Q, rho, mth, e, c - 1);
      sem = sqrtf(e[c - 1] * rinv(rho[c - 1]));
    }
  }
  const GlobalPrims pr{st, st + n, st + 2 * n, st + 3 * n, st + 4 * n, P.ntke ? st + 5 * n : nullptr,
                       P.nmoist ? st + (5 + P.ntke) * n : nullptr, n, c, P.si, P.sj};
  turb_cell_a<GlobalPrims, false>(P, Q, pr, st, i, j, k, lsc, lsm, sem, -1.0f, stage);
}

// The surface layer of the columns the tiled SGS kernel covers (i in [iMin, iMax], j in
// [jMin, jMax]), one thread per column, launched right after it. In the tiled kernel the
// Monin-Obukhov iteration would run on one lane of every warp holding the first level while the
// other 31 lanes wait; here every lane works. It overwrites the same first-level components
// (tau31, tau32, tauTH3, the q_v flux) the per-cell form's in-kernel call does.
static __global__ void __launch_bounds__(128) k_surface(Phys P, Ptrs Q, const float* __restrict__ st, int stage) {
  const int j = P.jMin + blockIdx.x * blockDim.x + threadIdx.x;
  const int i = P.iMin + blockIdx.y;
  if (j > P.jMax || i > P.iMax) return;
  surface_column(P, Q, st, i, j, stage);
}

// Write value v of one field at interior cell (i,j,k) and at its periodic images; `nbot`
// cells below kMin get the same value (bottom copy rule) and, if `top`, the 3 cells above
// kMax-1 too (zero-gradient rule). Image columns exist for i within 3 of either x edge and
// j within 3 of either y edge (both sides when the domain is narrower than 6).
__device__ __forceinline__ void store_column(float* __restrict__ F, long long cb, float v, int nbot, bool top) {
  F[cb] = v;
  for (int h = 1; h <= nbot; h++) F[cb - h] = v;
  if (top)
    for (int h = 1; h <= 3; h++) F[cb + h] = v;
}

// The image of a cell near the low x edge is a cell of the high x halo of the domain that holds
// the neighbour at dx = -1 (and so on): P.nbr[(dx+1)*3 + (dy+1)] is the offset, in floats, from
// this domain's state arena to that domain's. A domain that spans its periodic direction is its
// own neighbour there (offset 0); a slab of a decomposed domain writes the images straight into
// its neighbours' halos, on this device or a peer's (the halo exchange of fecuda_Utils.cu:205-418,
// fused into the commit).
__device__ __forceinline__ void store_images(const Phys& P, float* __restrict__ F, int i, int j, int k, float v, int nbot,
                                             bool top) {
  const long long c = (long long)i * P.si + (long long)j * P.sj + k;
  const long long dI = (long long)P.Nx * P.si, dJ = (long long)P.Ny * P.sj;
  const bool ilo = i < P.iMin + 3, ihi = i >= P.iMax - 3, jlo = j < P.jMin + 3, jhi = j >= P.jMax - 3;
  store_column(F, c, v, nbot, top);
  if (jlo) store_column(F + P.nbr[3], c + dJ, v, nbot, top);
  if (jhi) store_column(F + P.nbr[5], c - dJ, v, nbot, top);
  if (ilo) {
    store_column(F + P.nbr[1], c + dI, v, nbot, top);
    if (jlo) store_column(F + P.nbr[0], c + dI + dJ, v, nbot, top);
    if (jhi) store_column(F + P.nbr[2], c + dI - dJ, v, nbot, top);
  }
  if (ihi) {
    store_column(F + P.nbr[7], c - dI, v, nbot, top);
    if (jlo) store_column(F + P.nbr[6], c - dI + dJ, v, nbot, top);
    if (jhi) store_column(F + P.nbr[8], c - dI - dJ, v, nbot, top);
  }
}

// ------------------------------------------------------------------ fused stage
template <int STAGE, int MODE>
static __global__ void __launch_bounds__(256) k_stage(Phys P, Ptrs Q, const float* __restrict__ cur, const float* __restrict__ base,
                                               float* __restrict__ nxt, const float* __restrict__ pcur,
                                               float* __restrict__ pnxt, float* __restrict__ frhs) {
  const int k = P.kMin + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = P.jMin + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = P.iMin + blockIdx.z * blockDim.z + threadIdx.z;
  if (k >= P.kMax || j >= P.jMax || i >= P.iMax) return;
  const long long n = P.n;
  const int si = P.si, sj = P.sj;
  const long long c = (long long)i * si + (long long)j * sj + k;
  const float *rho = cur, *mu = cur + n, *mv = cur + 2 * n, *mw = cur + 3 * n, *mth = cur + 4 * n;
  const float* me = P.ntke ? cur + 5 * n : nullptr;
  const float* mq0 = P.nmoist > 0 ? cur + (5 + P.ntke) * n : nullptr;
  const float* mq1 = P.nmoist > 1 ? mq0 + n : nullptr;
  const bool phys = (P.oneRK == 0) || (STAGE == 2);
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
  const float J1 = Q.J31[c], J2 = Q.J32[c], J3 = Q.J33[c];
  float F0 = 0.0f, F1 = 0.0f, F2 = 0.0f, F3 = 0.0f, F4 = 0.0f, Fe = 0.0f, Fq0 = 0.0f, Fq1 = 0.0f;

  // pressure-gradient force (cuda_pressureDevice.cu:118-194)
  if (P.pgf) {
    const float dpx = pcur[c + si] - pcur[c - si];
    const float dpy = pcur[c + sj] - pcur[c - sj];
    const float dpz = pcur[c + 1] - pcur[c - 1];
    if (P.nmoist > 0) {
      float rmd = 1.0f;
      rmd = (float)((double)rmd + (double)(mq0[c] / rho[c]) * 1e-3);
      if (P.nmoist > 1) rmd = (float)((double)rmd + (double)(mq1[c] / rho[c]) * 1e-3);
      const float rdm = 1.0f / rmd;
      F1 = (float)((double)F1 - (double)rdm * 0.5 * (double)dXi * (double)dpx);
      F2 = (float)((double)F2 - (double)rdm * 0.5 * (double)dYi * (double)dpy);
      F3 = (float)((double)F3 - (double)rdm * 0.5 * (double)(dXi * J1 * dpx + dYi * J2 * dpy + dZi * J3 * dpz));
    } else {
      F1 = F1 - (0.5f * dXi) * dpx;
      F2 = F2 - (0.5f * dYi) * dpy;
      F3 = F3 - 0.5f * (dXi * J1 * dpx + dYi * J2 * dpy + dZi * J3 * dpz);
    }
  }

  // face velocities of this cell (cuda_advectionDevice.cu:89-106)
  FaceVel fv;
  {
    const float* D = Q.D;
    const long long im = c - si, ip = c + si, jm = c - sj, jp = c + sj, km = c - 1, kp = c + 1;
    const float cxc = contra(D[c], rho[c], mu[c], mw[c], J1);
    const float cxm = contra(D[im], rho[im], mu[im], mw[im], Q.J31[im]);
    const float cxp = contra(D[ip], rho[ip], mu[ip], mw[ip], Q.J31[ip]);
    fv.um = (0.5f * dXi) * (cxc + cxm);
    fv.up = (0.5f * dXi) * (cxp + cxc);
    const float cyc = contra(D[c], rho[c], mv[c], mw[c], J2);
    const float cym = contra(D[jm], rho[jm], mv[jm], mw[jm], Q.J32[jm]);
    const float cyp = contra(D[jp], rho[jp], mv[jp], mw[jp], Q.J32[jp]);
    fv.vm = (0.5f * dYi) * (cyc + cym);
    fv.vp = (0.5f * dYi) * (cyp + cyc);
    const float czc = contra_z(D[c], rho[c], mw[c], J3);
    const float czm = contra_z(D[km], rho[km], mw[km], Q.J33[km]);
    const float czp = contra_z(D[kp], rho[kp], mw[kp], Q.J33[kp]);
    fv.wm = (k == P.kMin) ? 0.0f : (0.5f * dZi) * (czc + czm);
    fv.wp = (k + 1 >= P.kMax) ? 0.0f : (0.5f * dZi) * (czp + czc);
  }
  const float invD = Q.invD[c];

  // Summed schemes: F -= invD (Dx + Dy + Dz) in one update; D = u+ f+ - u- f- per direction.
  auto advSum = [&](const float* __restrict__ s, int sel, float b) -> float {
    const float bf = 1.0f - b;
    float fxp, fxm, fyp, fym, fzp, fzm;
    {
      const float m3 = s[c - 3 * si], m2 = s[c - 2 * si], m1 = s[c - si], z0 = s[c], p1 = s[c + si], p2 = s[c + 2 * si],
                  p3 = s[c + 3 * si];
      fxp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.up, bf);
      fxm = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.um, bf);
    }
    {
      const float m3 = s[c - 3 * sj], m2 = s[c - 2 * sj], m1 = s[c - sj], z0 = s[c], p1 = s[c + sj], p2 = s[c + 2 * sj],
                  p3 = s[c + 3 * sj];
      fyp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.vp, bf);
      fym = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.vm, bf);
    }
    {
      const float m3 = s[c - 3], m2 = s[c - 2], m1 = s[c - 1], z0 = s[c], p1 = s[c + 1], p2 = s[c + 2], p3 = s[c + 3];
      fzp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.wp, bf);
      fzm = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.wm, bf);
    }
    const float Dx = fv.up * fxp - fv.um * fxm;
    const float Dy = fv.vp * fyp - fv.vm * fym;
    const float Dz = fv.wp * fzp - fv.wm * fzm;
    return invD * (Dx + Dy + Dz);
  };
  // WENO3/WENO5 apply x, y, z as three separate updates (cuda_hydroCoreDevice.cu:641-648)
  auto advSplit = [&](float Facc, const float* __restrict__ s, int sel) -> float {
    {
      const float m3 = s[c - 3 * si], m2 = s[c - 2 * si], m1 = s[c - si], z0 = s[c], p1 = s[c + si], p2 = s[c + 2 * si],
                  p3 = s[c + 3 * si];
      const float fp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.up, 1.0f);
      const float fm = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.um, 1.0f);
      Facc = Facc - invD * (fv.up * fp - fv.um * fm);
    }
    {
      const float m3 = s[c - 3 * sj], m2 = s[c - 2 * sj], m1 = s[c - sj], z0 = s[c], p1 = s[c + sj], p2 = s[c + 2 * sj],
                  p3 = s[c + 3 * sj];
      const float fp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.vp, 1.0f);
      const float fm = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.vm, 1.0f);
      Facc = Facc - invD * (fv.vp * fp - fv.vm * fm);
    }
    {
      const float m3 = s[c - 3], m2 = s[c - 2], m1 = s[c - 1], z0 = s[c], p1 = s[c + 1], p2 = s[c + 2], p3 = s[c + 3];
      const float fp = adv_face(sel, m2, m1, z0, p1, p2, p3, fv.wp, 1.0f);
      const float fm = adv_face(sel, m3, m2, m1, z0, p1, p2, fv.wm, 1.0f);
      Facc = Facc - invD * (fv.wp * fp - fv.wm * fm);
    }
    return Facc;
  };
  auto advect = [&](float Facc, const float* __restrict__ s, int sel, float b) -> float {
    if (adv_split(sel)) return advSplit(Facc, s, sel);
    return Facc - advSum(s, sel, b);
  };

  // advection of the hydro fields, Rayleigh damping and buoyancy on w (cuda_hydroCoreDevice.cu:631-672)
  F0 = advect(F0, rho, P.advSel, P.bHyb);
  F1 = advect(F1, mu, P.advSel, P.bHyb);
  F2 = advect(F2, mv, P.advSel, P.bHyb);
  F3 = advect(F3, mw, P.advSel, P.bHyb);
  if (P.damp) {
    const long long ctop = c - k + (P.kMax - 1);
    const float z = Q.zPos[c], zt = Q.zPos[ctop];
    if (z >= (zt - P.dampDepth)) {
      const float wbs = momentum_bs(P, 3, z, Q.rhoBS[c]);
      const float pio2 = 1.5707963267948966f;
      const double s = (double)sinf((float)((double)pio2 * (1.0 - (double)((zt - z) / P.dampDepth))));
      F3 = (float)((double)F3 - 0.2 * (double)rho[c] * (s * s) * (double)(mw[c] / rho[c] - wbs / Q.rhoBS[c]));
    }
  }
  if (P.buoy) {
    const float r = rho[c], rbs = Q.rhoBS[c];
    if (P.nmoist > 0) {
      // Klemp (2007) moist buoyancy; the excess density (cancellation-sensitive) in FP64
      double rm = (double)r + (double)mq0[c] * 1e-3;
      if (P.nmoist == 2) rm += (double)mq1[c] * 1e-3;
      const float ratio = r / (float)rm;
      F3 = (float)((double)F3 - (double)(ratio * P.g) * (rm - (double)rbs));
    } else {
      F3 = F3 - P.g * (r - rbs);
    }
  }
  F4 = advect(F4, mth, P.advSel, P.bHyb);
  if (P.ntke) Fe = advect(Fe, me, P.tkeAdvSel, P.tkeBHyb);
  if (P.nmoist > 0) Fq0 = advect(Fq0, mq0, P.qvAdvSel, P.qvB);
  if (P.nmoist > 1) Fq1 = advect(Fq1, mq1, P.qlSch, 0.0f);

  // Coriolis (cuda_coriolisDevice.cu:50-58)
  if (P.cor) {
    const float z = Q.zPos[c], rbs = Q.rhoBS[c], r = rho[c];
    const float ubs = momentum_bs(P, 1, z, rbs), vbs = momentum_bs(P, 2, z, rbs), wbs = momentum_bs(P, 3, z, rbs);
    F1 = F1 + (P.fHorz * (mv[c] / r - P.fLS * vbs / rbs) - P.fVert * (mw[c] / r - P.fLS * wbs / rbs));
    F2 = F2 - (P.fHorz * (mu[c] / r - P.fLS * ubs / rbs));
    F3 = F3 + (P.fVert * (mu[c] / r - P.fLS * ubs / rbs));
  }

  if (phys && P.turb) {
    // divergence of the SGS stresses (cuda_sgsTurbDevice.cu:447-547)
    const float* T = Q.tau;
    const long long ip = c + si, jp = c + sj, kp = c + 1;
#define TT(m, x) T[(m) * n + (x)]
    F1 = F1 - (dXi * (TT(0, ip) - TT(0, c)) + dYi * (TT(1, jp) - TT(1, c)) + J1 * dXi * (TT(2, ip) - TT(2, c)) +
               J2 * dYi * (TT(2, jp) - TT(2, c)) + J3 * dZi * (TT(2, kp) - TT(2, c)));
    F2 = F2 - (dXi * (TT(1, ip) - TT(1, c)) + dYi * (TT(4, jp) - TT(4, c)) + J1 * dXi * (TT(3, ip) - TT(3, c)) +
               J2 * dYi * (TT(3, jp) - TT(3, c)) + J3 * dZi * (TT(3, kp) - TT(3, c)));
    F3 = F3 - (dXi * (TT(2, ip) - TT(2, c)) + dYi * (TT(3, jp) - TT(3, c)) + J1 * dXi * (TT(5, ip) - TT(5, c)) +
               J2 * dYi * (TT(5, jp) - TT(5, c)) + J3 * dZi * (TT(5, kp) - TT(5, c)));
    F4 = F4 - (dXi * (TT(6, ip) - TT(6, c)) + dYi * (TT(7, jp) - TT(7, c)) + J1 * dXi * (TT(8, ip) - TT(8, c)) +
               J2 * dYi * (TT(8, jp) - TT(8, c)) + J3 * dZi * (TT(8, kp) - TT(8, c)));
    if (P.nmoist > 0 && P.moistSGS > 0) {
      const float* M = Q.mtau;
      Fq0 = Fq0 - (dXi * (M[ip] - M[c]) + dYi * (M[n + jp] - M[n + c]) +
                   J1 * dXi * (M[2 * n + ip] - M[2 * n + c]) + J2 * dYi * (M[2 * n + jp] - M[2 * n + c]) +
                   J3 * dZi * (M[2 * n + kp] - M[2 * n + c]));
      if (P.nmoist > 1) {
        const float* M1 = M + 3 * n;
        Fq1 = Fq1 - (dXi * (M1[ip] - M1[c]) + dYi * (M1[n + jp] - M1[n + c]) + J1 * dXi * (M1[2 * n + ip] - M1[2 * n + c]) +
                     J2 * dYi * (M1[2 * n + jp] - M1[2 * n + c]) + J3 * dZi * (M1[2 * n + kp] - M1[2 * n + c]));
      }
    }
    // SGS TKE budget (cuda_sgstkeDevice.cu:155-397)
    if (P.tke) {
      const float ri = rinv(rho[c]);
      const float delta = grid_scale(P, Q, c);
      const float lsc = Q.ls[c];
      Fe = Fe + P.g / (mth[c] * ri) * TT(8, c);
      const float ce = (float)(1.9 * (double)P.c_k + (0.93 - 1.9 * (double)P.c_k) * (double)lsc / (double)delta);
      const float ec = me[c] * ri;
      Fe = Fe + (-ce * me[c] * sqrtf(ec) / lsc);
      const long long im = c - si, jm = c - sj, km = c - 1;
#define G_(q, x) (q[x] * rinv(rho[x]))
      const float dux = 0.5f * (dXi * (G_(mu, ip) - G_(mu, im)));
      const float duy = 0.5f * (dYi * (G_(mu, jp) - G_(mu, jm)));
      const float duz = 0.5f * (J1 * dXi * (G_(mu, ip) - G_(mu, im)) + J2 * dYi * (G_(mu, jp) - G_(mu, jm)) +
                                J3 * dZi * (G_(mu, kp) - G_(mu, km)));
      const float dvx = 0.5f * (dXi * (G_(mv, ip) - G_(mv, im)));
      const float dvy = 0.5f * (dYi * (G_(mv, jp) - G_(mv, jm)));
      const float dvz = 0.5f * (J1 * dXi * (G_(mv, ip) - G_(mv, im)) + J2 * dYi * (G_(mv, jp) - G_(mv, jm)) +
                                J3 * dZi * (G_(mv, kp) - G_(mv, km)));
      const float dwx = 0.5f * (dXi * (G_(mw, ip) - G_(mw, im)));
      const float dwy = 0.5f * (dYi * (G_(mw, jp) - G_(mw, jm)));
      const float dwz = 0.5f * (J1 * dXi * (G_(mw, ip) - G_(mw, im)) + J2 * dYi * (G_(mw, jp) - G_(mw, jm)) +
                                J3 * dZi * (G_(mw, kp) - G_(mw, km)));
#undef G_
      const float shear = (-TT(0, c) * dux) + (-TT(1, c) * duy) + (-TT(2, c) * duz) + (-TT(1, c) * dvx) +
                          (-TT(4, c) * dvy) + (-TT(3, c) * dvz) + (-TT(2, c) * dwx) + (-TT(3, c) * dwy) + (-TT(5, c) * dwz);
      Fe = Fe + shear;
      const float* G = Q.tkeQ;
      const float tx = -(dXi * (G[ip] - G[im]));
      const float ty = -(dYi * (G[n + jp] - G[n + jm]));
      const float tz = -(J1 * dXi * (G[2 * n + ip] - G[2 * n + im]) + J2 * dYi * (G[2 * n + jp] - G[2 * n + jm]) +
                         J3 * dZi * (G[2 * n + kp] - G[2 * n + km]));
      Fe = Fe + (-(tx + ty + tz));
    }
#undef TT
  }

  // saturation adjustment (cuda_moistureDevice.cu:80-247)
  if (phys && P.nmoist > 1 && P.moist && P.moistCond > 0) {
    if ((*Q.clockIt) % P.mpFreq == 0) {
      const float ri = rinv(rho[c]);
      const float thd = mth[c] * ri;
      const float prd = P.condBasePres == 1 ? powf(Q.thBS[c] * P.c1, P.cp_cv) : powf(mth[c] * P.c1, P.cp_cv);
      const float Td = thd * powf(prd / P.p0, P.R_cp);
      float pvs;
      const float Tc = fmaxf(-80.0f, (Td - 273.16f));
      if (Td >= 273.15f) {
        pvs = (6.11239921f + Tc * (0.443987641f + Tc * (0.142986287e-1f + Tc * (0.264847430e-3f + Tc * (0.302950461e-5f +
              Tc * (0.206739458e-7f + Tc * (0.640689451e-10f + Tc * (-0.952447341e-13f + -0.976195544e-15f * Tc)))))))) * 100.0f;
      } else {
        pvs = (6.11147274f + Tc * (0.503160820f + Tc * (0.188439774e-1f + Tc * (0.420895665e-3f + Tc * (0.615021634e-5f +
              Tc * (0.602588177e-7f + Tc * (0.385852041e-9f + Tc * (0.146898966e-11f + 0.252751365e-14f * Tc)))))))) * 100.0f;
      }
      pvs = fminf((0.99f * prd), pvs);
      float ffor = 0.0f;
      const float flim = mq1[c] * 1e-3f;
      if (P.moistCond == 1) {
        ffor = mq0[c] * 1e-3f - (pvs / (P.R_vapor * Td));
      } else if (P.moistCond == 2) {
        const float rv = mq0[c] * 1e-3f, rvs = pvs / (P.R_vapor * Td);
        ffor = (rv - rvs) / (1.0f + (powf(P.L_v, 2.0f) * rvs * ri / (P.cp_gas * P.R_vapor * powf(Td, 2.0f))));
      } else {
        const float rv = mq0[c] * 1e-3f;
        float rvs = pvs / (prd - pvs) / P.Rv_Rg;
        rvs = rvs / ri;
        ffor = (rv - rvs) / (1.0f + (powf(P.L_v, 2.0f) * rvs * ri / (P.cp_gas * P.R_vapor * powf(Td, 2.0f))));
      }
      float fc = fmaxf(ffor, 0.0f) - fmaxf(fminf(flim, -ffor), 0.0f);
      fc = fc / P.condTscale;
      Fq0 = Fq0 - fc * 1e3f;
      Fq1 = Fq1 + fc * 1e3f;
      const float prd2 = powf(mth[c] * P.c1, P.cp_cv);
      const float Td2 = thd * powf(prd2 / P.p0, P.R_cp);
      F4 = F4 + ((thd * P.L_v) / (Td2 * P.cp_gas)) * fc;
    }
  }

  // large-scale forcing in the last stage (cuda_hydroCoreDevice.cu:401-406)
  if (STAGE == 2 && lsf_step(P, *Q.clockIt)) lsf_tend(P, Q, c, k, Q.zPos[c], rho[c], F1, F2, F4, Fq0);
  // explicit filter of rho w, every stage, after all other terms (cuda_hydroCoreDevice.cu:414-416)
  if (P.filt)
    F3 = __fadd_rn(F3, filter6_tend(mw[c - 3], mw[c - 2], mw[c - 1], mw[c], mw[c + 1], mw[c + 2], mw[c + 3], P.filtCoef));

  if (MODE == MODE_FRHS || (STAGE == 2 && frhs)) {
    // tendencies only, or the last stage's tendencies kept beside its commit
    frhs[c] = F0;
    frhs[n + c] = F1;
    frhs[2 * n + c] = F2;
    frhs[3 * n + c] = F3;
    frhs[4 * n + c] = F4;
    if (P.ntke) frhs[5 * n + c] = Fe;
    if (P.nmoist > 0) frhs[(5 + P.ntke) * n + c] = Fq0;
    if (P.nmoist > 1) frhs[(6 + P.ntke) * n + c] = Fq1;
    if (MODE == MODE_FRHS) return;
  }

  // WS2002 RK3 commit (cuda_RKschemes.cu:113-157) with the reference's rounding:
  // stages 1-2 in double ((1/3)dt, 0.5 dt literals), stage 3 in float.
  auto rk = [&](float phi0, float F) -> float {
    if (STAGE == 0) return (float)fma((1.0 / 3.0) * (double)P.dt, (double)F, (double)phi0);
    if (STAGE == 1) return (float)fma(0.5 * (double)P.dt, (double)F, (double)phi0);
    return __fmaf_rn(P.dt, F, phi0);
  };
  const float* b0 = base;
  const float n0 = rk(b0[c], F0);
  const float n1 = rk(b0[n + c], F1);
  const float n2 = rk(b0[2 * n + c], F2);
  const float n3 = rk(b0[3 * n + c], F3);
  const float n4 = rk(b0[4 * n + c], F4);
  const bool atBot = (k == P.kMin), atTop = (k == P.kMax - 1);
  store_images(P, nxt, i, j, k, n0, 0, false);
  store_images(P, nxt + n, i, j, k, n1, atBot ? 3 : 0, false);
  store_images(P, nxt + 2 * n, i, j, k, n2, atBot ? 3 : 0, false);
  store_images(P, nxt + 3 * n, i, j, k, n3, atBot ? 3 : 0, false);
  store_images(P, nxt + 4 * n, i, j, k, n4, 0, false);
  float nq0 = 0.0f;
  if (P.ntke) {
    const float ne = fmaxf(rk(b0[5 * n + c], Fe), 1e-10f);
    store_images(P, nxt + 5 * n, i, j, k, ne, atBot ? 3 : 0, false);
  }
  if (P.nmoist > 0) {
    const long long o = (5 + P.ntke) * n;
    nq0 = fmaxf(rk(b0[o + c], Fq0), 0.0f);
    store_images(P, nxt + o, i, j, k, nq0, atBot ? 3 : 0, atTop);
    if (P.nmoist > 1) {
      const float nq1 = fmaxf(rk(b0[o + n + c], Fq1), 0.0f);
      store_images(P, nxt + o + n, i, j, k, nq1, atBot ? 3 : 0, atTop);
    }
  }
  // perturbation pressure of the new state (levels 1..kMin-1 and kMax.. copy this cell)
  float pn;
  {
    float rtm = n4;
    if (P.nmoist > 0) rtm = (float)((double)n4 * (1.0 + (double)(P.Rv_Rg * nq0 / n0) * 1e-3));
    pn = powf(rtm * P.c1, P.cp_cv) - Q.pBS[c];
  }
  store_images(P, pnxt, i, j, k, pn, atBot ? 2 : 0, atTop);
  if (atBot) store_images(P, pnxt, i, j, 0, level0_pressure(P, Q, c - k, P.nmoist, nq0), 0, false);
}

static __global__ void k_clock(Ptrs Q, float dt) {
  *Q.clockIt = *Q.clockIt + 1;
  *Q.clockTime = *Q.clockTime + dt;
}

// One member of a batched surface-layer launch: blocks first .. first + gj*(Nx+1) - 1, gj blocks
// of 128 columns along j per i.
struct SurfMember {
  Phys P;
  Ptrs Q;
  const float* st;
  int gj, first;
};

// k_surface of several domains in one launch.
static __global__ void __launch_bounds__(128) k_surface_list(const SurfMember* __restrict__ mem, const int* __restrict__ bmap,
                                                             int stage) {
  __shared__ SurfMember sm_m;
  __shared__ int sm_idx;
  if (threadIdx.x == 0) sm_idx = bmap[blockIdx.x];
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(mem + sm_idx);
    int* dst = reinterpret_cast<int*>(&sm_m);
    for (int q = threadIdx.x; q < (int)(sizeof(SurfMember) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
  }
  __syncthreads();
  const SurfMember& m = sm_m;
  const int local = (int)blockIdx.x - m.first;
  const int j = m.P.jMin + (local % m.gj) * 128 + threadIdx.x;
  const int i = m.P.iMin + local / m.gj;
  if (j > m.P.jMax || i > m.P.iMax) return;
  surface_column(m.P, m.Q, m.st, i, j, stage);
}

// The device clocks of several domains (one thread each).
struct ClockMember {
  int* it;
  float* time;
  float dt;
};
static __global__ void k_clock_list(const ClockMember* __restrict__ mem, int nmem) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nmem) return;
  *mem[t].it = *mem[t].it + 1;
  *mem[t].time = *mem[t].time + mem[t].dt;
}

static __global__ void k_nonfinite(Phys P, const float* __restrict__ st, unsigned long long* out) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned int cnt = 0;
  if (t < P.n) {
    const int k = (int)(t % P.nzh);
    const int j = (int)((t / P.nzh) % P.nyh);
    const int i = (int)(t / ((long long)P.nzh * P.nyh));
    if (i >= P.iMin && i < P.iMax && j >= P.jMin && j < P.jMax && k >= P.kMin && k < P.kMax)
      for (int f = 0; f < P.nf; f++) cnt += isfinite(st[(long long)f * P.n + t]) ? 0u : 1u;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, (unsigned long long)cnt);
}

// Slab means for the large-scale subsidence terms (cuda_largeScaleForcingsDevice.cu:96-138 with
// fecuda_PlugIns.cu:25-45): the mean over every column of the halo-inclusive plane (weight
// 1/(nxh nyh)) of rho, rho u, rho v, rho theta and rho q_v at every level. The reference's RK
// commit writes interior cells only, so when it takes the means at the start of a step its halo
// cells still hold the boundary values of the previous step's last-stage input phi**: interior
// cells are read from `cur` (phi^n) and halo cells from `halo` (the buffer holding phi** with its
// boundary images). Sums are FP64: each block accumulates its columns (thread = level) into
// lsfPart[block][field][level]; k_slab_final adds the blocks in a fixed order.
static __global__ void k_slab_partial(Phys P, Ptrs Q, const float* __restrict__ cur, const float* __restrict__ halo,
                               int force) {
  if (!force && !lsf_means_step(P, *Q.clockIt)) return;
  const long long cols = (long long)P.nxh * P.nyh;
  const long long qv = (long long)(5 + P.ntke) * P.n;
  for (int k = threadIdx.x; k < P.nzh; k += blockDim.x) {
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const bool kin = k >= P.kMin && k < P.kMax;
    for (long long col = blockIdx.x; col < cols; col += gridDim.x) {
      const int i = (int)(col / P.nyh), j = (int)(col % P.nyh);
      const bool in = kin && i >= P.iMin && i < P.iMax && j >= P.jMin && j < P.jMax;
      const float* src = in ? cur : halo;
      const long long c = col * P.nzh + k;
      acc[0] += (double)src[c];
      acc[1] += (double)src[P.n + c];
      acc[2] += (double)src[2 * P.n + c];
      acc[3] += (double)src[4 * P.n + c];
      if (P.moist) acc[4] += (double)src[qv + c];
    }
    double* out = Q.lsfPart + (long long)blockIdx.x * 5 * P.nzh;
#pragma unroll
    for (int f = 0; f < 5; f++) out[f * P.nzh + k] = acc[f];
  }
}

static __global__ void k_slab_final(Phys P, Ptrs Q, int nblocks, int force) {
  if (!force && !lsf_means_step(P, *Q.clockIt)) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 5 * P.nzh) return;
  double sum = 0.0;
  for (int b = 0; b < nblocks; b++) sum += Q.lsfPart[(long long)b * 5 * P.nzh + t];
  Q.lsfProf[t] = (float)(sum / ((double)P.nxh * (double)P.nyh));
}

// FP64 sums of the interior fields: warp shuffle, then one atomic per warp and field.
static __global__ void k_means(Phys P, const float* __restrict__ st, double* out) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool in = false;
  if (t < P.n) {
    const int k = (int)(t % P.nzh);
    const int j = (int)((t / P.nzh) % P.nyh);
    const int i = (int)(t / ((long long)P.nzh * P.nyh));
    in = i >= P.iMin && i < P.iMax && j >= P.jMin && j < P.jMax && k >= P.kMin && k < P.kMax;
  }
  for (int f = 0; f < P.nf; f++) {
    double v = in ? (double)st[(long long)f * P.n + t] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&out[f], v);
  }
}

}  // namespace fe
