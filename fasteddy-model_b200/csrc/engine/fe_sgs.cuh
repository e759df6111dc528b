// fe_sgs.cuh -- inputs of the learned SGS closure, evaluated exactly where and as the TKE
// closure evaluates its strain rates (cuda_sgsTurbDevice.cu:60-197, cuda_sgstkeDevice.cu:96-151).
//
// The 9 velocity-gradient components are the separate halves of the reference's staggered
// strain-rate elements: S11 = g11, S22 = g22, S33 = g33, S21 = (g21 + g12)/2,
// S31 = (g31 + g13)/2, S32 = (g32 + g23)/2, each half in the reference's own arithmetic, so
// the components sit at the stress point the closure writes (index c, lower faces/edges).
// N^2 is the length-scale buoyancy frequency and the grid scale is (dx dy dz D)^(1/3).
#pragma once
#include "fe_device.cuh"

namespace fe {

constexpr int SGS_NIN = 11;   // g11 g12 g13 g21 g22 g23 g31 g32 g33 N^2 Delta
constexpr int SGS_NOUT = 9;   // tau11 tau21 tau31 tau32 tau22 tau33 tauTH1 tauTH2 tauTH3 (hydroTauFlds order)

__device__ __forceinline__ void sgs_inputs(const Phys& P, const Ptrs& Q, const float* __restrict__ st, long long c,
                                           float* x) {
  const long long n = P.n;
  const int si = P.si, sj = P.sj;
  const float *rho = st, *mu = st + n, *mv = st + 2 * n, *mw = st + 3 * n, *mth = st + 4 * n;
  const long long a = c - si, b = c - sj, d = c - 1, ab = a - sj, ad = a - 1, bd = b - 1, abd = ab - 1;
  const float J1 = Q.J31[c], J2 = Q.J32[c], J3 = Q.J33[c];
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
#define U_(x) (mu[x] * rinv(rho[x]))
#define V_(x) (mv[x] * rinv(rho[x]))
#define W_(x) (mw[x] * rinv(rho[x]))
  x[0] = dXi * (U_(c) - U_(a));
  x[1] = 0.5f * (dYi * (U_(c) - U_(b)) + dYi * (U_(a) - U_(ab)));
  x[2] = 0.5f * (J1 * dXi * (U_(c) - U_(a)) + J1 * dXi * (U_(d) - U_(ad))) +
         0.25f * (J2 * dYi * (U_(c) - U_(b)) + J2 * dYi * (U_(a) - U_(ab)) + J2 * dYi * (U_(d) - U_(bd)) +
                  J2 * dYi * (U_(ad) - U_(abd))) +
         0.5f * (J3 * dZi * (U_(c) - U_(d)) + J3 * dZi * (U_(a) - U_(ad)));
  x[3] = 0.5f * (dXi * (V_(c) - V_(a)) + dXi * (V_(b) - V_(ab)));
  x[4] = dYi * (V_(c) - V_(b));
  x[5] = 0.25f * (J1 * dXi * (V_(c) - V_(a)) + J1 * dXi * (V_(b) - V_(ab)) + J1 * dXi * (V_(d) - V_(ad)) +
                  J1 * dXi * (V_(bd) - V_(abd))) +
         0.5f * (J2 * dYi * (V_(c) - V_(b)) + J2 * dYi * (V_(d) - V_(bd))) +
         0.5f * (J3 * dZi * (V_(c) - V_(d)) + J3 * dZi * (V_(b) - V_(bd)));
  x[6] = 0.5f * (dXi * (W_(c) - W_(a)) + dXi * (W_(d) - W_(ad)));
  x[7] = 0.5f * (dYi * (W_(c) - W_(b)) + dYi * (W_(d) - W_(bd)));
  x[8] = J1 * dXi * (W_(c) - W_(a)) + J2 * dYi * (W_(c) - W_(b)) + J3 * dZi * (W_(c) - W_(d));
#undef U_
#undef V_
#undef W_
#define THr(q) (mth[q] * rinv(rho[q]))
  const float dthdz = (float)(0.5 * (double)((J1 * dXi * (THr(c + si) - THr(c - si))) +
                                             (J2 * dYi * (THr(c + sj) - THr(c - sj))) +
                                             (J3 * dZi * (THr(c + 1) - THr(c - 1)))));
  x[9] = (P.g / THr(c)) * dthdz;
#undef THr
  x[10] = grid_scale(P, Q, c);
}

}  // namespace fe
