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

// Every rounding is spelled out (__fmul_rn/__fadd_rn/__fsub_rn, no fused multiply-add): the
// last-stage SGS kernel (primitives from a shared-memory tile) and the sampling kernel (primitives
// from the state) inline separate copies, and the network rounds its standardised inputs to BF16,
// where a one-ulp difference can move a value across a rounding boundary. Both copies therefore
// have to produce the same bits.
template <class A>
__device__ __forceinline__ void sgs_inputs_a(const Phys& P, const Ptrs& Q, const A& pr, long long c, float* x) {
  const float J1 = Q.J31[c], J2 = Q.J32[c], J3 = Q.J33[c];
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
  const float uc = pr.u(0, 0, 0), ua = pr.u(-1, 0, 0), ub = pr.u(0, -1, 0), ud = pr.u(0, 0, -1);
  const float uab = pr.u(-1, -1, 0), uad = pr.u(-1, 0, -1), ubd = pr.u(0, -1, -1), uabd = pr.u(-1, -1, -1);
  const float vc = pr.v(0, 0, 0), va = pr.v(-1, 0, 0), vb = pr.v(0, -1, 0), vd = pr.v(0, 0, -1);
  const float vab = pr.v(-1, -1, 0), vad = pr.v(-1, 0, -1), vbd = pr.v(0, -1, -1), vabd = pr.v(-1, -1, -1);
  const float wc = pr.w(0, 0, 0), wa = pr.w(-1, 0, 0), wb = pr.w(0, -1, 0), wd = pr.w(0, 0, -1);
  const float wad = pr.w(-1, 0, -1), wbd = pr.w(0, -1, -1);
  // scaled differences: s * (p - q), and J * s * (p - q) evaluated as (J * s) * (p - q)
  auto d1 = [](float sc, float p, float q) { return __fmul_rn(sc, __fsub_rn(p, q)); };
  auto d2 = [](float J, float sc, float p, float q) { return __fmul_rn(__fmul_rn(J, sc), __fsub_rn(p, q)); };
  auto add = [](float p, float q) { return __fadd_rn(p, q); };
  x[0] = d1(dXi, uc, ua);
  x[1] = __fmul_rn(0.5f, add(d1(dYi, uc, ub), d1(dYi, ua, uab)));
  x[2] = add(add(__fmul_rn(0.5f, add(d2(J1, dXi, uc, ua), d2(J1, dXi, ud, uad))),
                 __fmul_rn(0.25f, add(add(add(d2(J2, dYi, uc, ub), d2(J2, dYi, ua, uab)), d2(J2, dYi, ud, ubd)),
                                      d2(J2, dYi, uad, uabd)))),
             __fmul_rn(0.5f, add(d2(J3, dZi, uc, ud), d2(J3, dZi, ua, uad))));
  x[3] = __fmul_rn(0.5f, add(d1(dXi, vc, va), d1(dXi, vb, vab)));
  x[4] = d1(dYi, vc, vb);
  x[5] = add(add(__fmul_rn(0.25f, add(add(add(d2(J1, dXi, vc, va), d2(J1, dXi, vb, vab)), d2(J1, dXi, vd, vad)),
                                      d2(J1, dXi, vbd, vabd))),
                 __fmul_rn(0.5f, add(d2(J2, dYi, vc, vb), d2(J2, dYi, vd, vbd)))),
             __fmul_rn(0.5f, add(d2(J3, dZi, vc, vd), d2(J3, dZi, vb, vbd))));
  x[6] = __fmul_rn(0.5f, add(d1(dXi, wc, wa), d1(dXi, wd, wad)));
  x[7] = __fmul_rn(0.5f, add(d1(dYi, wc, wb), d1(dYi, wd, wbd)));
  x[8] = add(add(d2(J1, dXi, wc, wa), d2(J2, dYi, wc, wb)), d2(J3, dZi, wc, wd));
  const float gx = d2(J1, dXi, pr.th(1, 0, 0), pr.th(-1, 0, 0));
  const float gy = d2(J2, dYi, pr.th(0, 1, 0), pr.th(0, -1, 0));
  const float gz = d2(J3, dZi, pr.th(0, 0, 1), pr.th(0, 0, -1));
  const float dthdz = (float)(0.5 * (double)add(add(gx, gy), gz));
  x[9] = __fmul_rn(__fdiv_rn(P.g, pr.th(0, 0, 0)), dthdz);
  x[10] = grid_scale(P, Q, c);
}

// The inputs of cell c straight from the flux-form state.
__device__ __forceinline__ void sgs_inputs(const Phys& P, const Ptrs& Q, const float* __restrict__ st, long long c,
                                           float* x) {
  const long long n = P.n;
  const GlobalPrims pr{st, st + n, st + 2 * n, st + 3 * n, st + 4 * n, nullptr, nullptr, n, c, P.si, P.sj};
  sgs_inputs_a(P, Q, pr, c, x);
}

}  // namespace fe
