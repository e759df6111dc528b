// fe_march.cuh -- the fused stage kernel in i-marching form (sm_100a).
//
// A thread block owns a tile of 32 levels (k, one warp wide, so every row of the tile is one
// 128-byte line) by TJ rows (j) and marches along i over a chunk of `ni` planes:
//
//   x direction   s(i..i+3) of every advected field live in registers (plus the prefetched
//                 plane i+4), s(i-1) and s(i-2) are the thread's own cells of the two other
//                 plane buffers; the x-face flux times the face velocity of the previous plane
//                 is carried, so every x face is evaluated once.
//   y, z          read a shared-memory copy of the (j,k) plane with a 3-cell ring. Three plane
//                 buffers rotate: the thread's own value comes from its register window, the
//                 ring of plane i+1 arrives by cp.async while plane i is computed, and one
//                 __syncthreads per plane separates the two.
//   face velocities  the contravariant velocities (D/rho)(m + w J) of plane i+1 are produced
//                 one plane ahead into the same buffers (own cell plus a one-cell ring), so a
//                 y or z face velocity costs one shared load.
//   own-column inputs  s(i+4) of every field, p'(i+2), the metrics of plane i+2 and 1/D of
//                 plane i+1 are copied by cp.async into a per-thread table one plane ahead, and
//                 the carried x fluxes live in shared memory too: the registers hold only the
//                 x window, so the 8-field flavour stays within 128 registers per thread.
//
// Everything else -- PGF, Rayleigh damping, buoyancy, Coriolis, SGS divergence and TKE budget,
// saturation adjustment, the WS2002 commit with its halo images and the perturbation pressure
// of the new state -- is the cell kernel's arithmetic (fe_kernels.cuh), term by term and in the
// same order, evaluated on the register/shared copies.
#pragma once
#include "fe_kernels.cuh"
#include "fe_march_launch.cuh"

namespace fe {

constexpr int MK = 32;                      // levels per tile
constexpr int MSLOTS = 9;                   // rho, rho u, rho v, rho w, rho theta, rho e, rho qv, rho ql, p'
constexpr int SL_E = 5, SL_QV = 6, SL_QL = 7, SL_P = 8;

template <int TJ>
struct MarchTile {
  static constexpr int PJ = TJ + 6, PK = MK + 6;   // staged plane with a 3-cell ring
  static constexpr int PLANE = PJ * PK;
  static constexpr int CYN = (TJ + 2) * MK;        // contravariant y velocity, rows j = -1..TJ
  static constexpr int CZK = MK + 2;               // contravariant z velocity, columns k = -1..MK
  static constexpr int CZN = TJ * CZK;
  static constexpr int BUF = MSLOTS * PLANE + CYN + CZN;
  static constexpr int NT = MK * TJ;
  static constexpr int RING = PLANE - TJ * MK;
  static constexpr int RPT = (RING + NT - 1) / NT;  // ring cells per thread
  static constexpr int CYT = 2 * MK, CZT = 2 * TJ;   // ring tasks of the velocity planes
  static constexpr int NBUF = 3;
  // per-thread tables: the inputs of the next plane (cp.async, double-buffered) and the
  // carried x-face flux times velocity of every field
  static constexpr int NAUX = 14;
  static constexpr int AUX = 2 * NAUX * NT;
  static constexpr int XC = 8 * NT;
  static constexpr int SMEM_BYTES = (NBUF * BUF + AUX + XC) * 4;
};

// Ring cell r of a staged plane: the 3 rows above and below the tile (full width), then the
// 3 columns left and right of every tile row.
template <int TJ>
__device__ __forceinline__ void march_ring_cell(int r, int& row, int& col) {
  constexpr int PK = MK + 6;
  if (r < 6 * PK) {
    row = r / PK;
    col = r - row * PK;
    if (row >= 3) row += TJ;
  } else {
    const int q = r - 6 * PK;
    row = 3 + q / 6;
    const int cc = q - (q / 6) * 6;
    col = cc < 3 ? cc : MK + cc;
  }
}

__device__ __forceinline__ void cp_async4(float* sdst, const float* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// Pull the line holding p into L2 (no register, no wait). Only ever given addresses of cells
// that exist in the array.
__device__ __forceinline__ void prefetch_l2(const float* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ bool slot_on(const Phys& P, int s) {
  if (s < 5) return true;
  if (s == SL_E) return P.ntke > 0;
  if (s == SL_QV) return P.nmoist > 0;
  if (s == SL_QL) return P.nmoist > 1;
  return P.pgf != 0;
}
__device__ __forceinline__ const float* slot_src(const Phys& P, const float* cur, const float* pcur, int s) {
  if (s < 5) return cur + (long long)s * P.n;
  if (s == SL_E) return cur + 5LL * P.n;
  if (s == SL_QV) return cur + (long long)(5 + P.ntke) * P.n;
  if (s == SL_QL) return cur + (long long)(6 + P.ntke) * P.n;
  return pcur;
}
// advection scheme of a slot as an ADV_* id (q_l's from moistureAdvSelectorQi)
__device__ __forceinline__ int slot_sel(const Phys& P, int s) {
  if (s < 5) return P.advSel;
  if (s == SL_E) return P.tkeAdvSel;
  if (s == SL_QV) return P.qvAdvSel;
  return P.qlSch;
}
__device__ __forceinline__ float slot_b(const Phys& P, int s) {
  if (s < 5) return P.bHyb;
  if (s == SL_E) return P.tkeBHyb;
  if (s == SL_QV) return P.qvB;
  return 0.0f;
}

// Compile-time configurations ("flavours") of the march kernel: fe_march_launch.cuh.
template <int FL>
__device__ __forceinline__ bool f_on(const Phys& P, int s) {
  if constexpr (FL == FL_DRY) return s <= SL_E || s == SL_P;
  else if constexpr (FL == FL_MOIST || FL == FL_MOIST34) return true;
  else return slot_on(P, s);
}
template <int FL>
__device__ __forceinline__ int f_sel(const Phys& P, int s) {
  if constexpr (FL == FL_MOIST34) return s == SL_QL ? 5 : (s == SL_QV ? 2 : 3);
  else if constexpr (FL != FL_ANY) return s == SL_QL ? 5 : 3;
  else return slot_sel(P, s);
}
// Fields s and s + 1 (s even) evaluate their x faces as one lane pair: both present and on the
// same scheme of the packed path, known at compile time. The moist flavours only: in the dry
// flavour the pairs cost more registers than the 128 the launch shape allows (spills).
template <int FL>
__host__ __device__ constexpr bool x_paired(int s) {
  if constexpr (FL == FL_ANY || FL == FL_DRY) {
    return false;
  } else {
    if (s % 2 != 0 || s + 1 > SL_QL) return false;
    const int a = FL == FL_MOIST34 ? (s == SL_QL ? 5 : (s == SL_QV ? 2 : 3)) : (s == SL_QL ? 5 : 3);
    const int b = FL == FL_MOIST34 ? (s + 1 == SL_QL ? 5 : (s + 1 == SL_QV ? 2 : 3)) : (s + 1 == SL_QL ? 5 : 3);
    return a == b && (a == ADV_HYB56 || a == ADV_WENO5);
  }
}
template <int FL>
__device__ __forceinline__ const float* f_src(const Phys& P, const float* cur, const float* pcur, int s) {
  if constexpr (FL != FL_ANY) {
    if (s == SL_P) return pcur;
    return cur + (long long)s * P.n;  // slots 0..7 are fields 0..7 when TKE is prognostic
  } else {
    return slot_src(P, cur, pcur, s);
  }
}

// SGS tendencies of the last-stage physics for the march kernel, one thread per interior cell
// (levels along x of the block): with the SGS stresses and fluxes written by the SGS kernel (and
// the learned closure, when set), seven fields of Q.sgsF at the cell's index:
//   0..3  divergence of the stresses on rho u, rho v, rho w and of the heat flux on rho theta
//         (cuda_sgsTurbDevice.cu:447-547), subtracted from the tendency
//   4     the TKE budget: buoyancy, dissipation, shear production and transport
//         (cuda_sgstkeDevice.cu:155-397), added
//   5, 6  divergence of the q_v and q_l SGS fluxes, subtracted
// Each expression is the per-cell stage kernel's; the TKE terms are summed here and added to the
// tendency once. `st` is the stage's input state; the shear production's velocity gradients use
// central differences of phi/rho at the six neighbours. TKE (prognostic TKE) and NQ (moisture
// species with SGS fluxes) are compile-time so that every load of a cell issues as one batch.
//
// On a large-scale forcing step (last stage) the forcing's tendencies of rho u, rho v, rho theta
// and rho q_v are folded into fields 0, 1, 3 and 5 (subtracted, as those fields are), so the march
// kernel carries no forcing code of its own; with moisture but no moisture SGS fluxes, field 5
// then holds only the forcing (zero on other steps).
template <bool TKE, int NQ>
__global__ void __launch_bounds__(256, 4) k_sgs_tend(Phys P, Ptrs Q, const float* __restrict__ st, int stage) {
  const int k = P.kMin + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = P.jMin + blockIdx.y * blockDim.y + threadIdx.y;
  const int i = P.iMin + blockIdx.z;
  if (k >= P.kMax || j >= P.jMax) return;
  const long long n = P.n;
  const int si = P.si, sj = P.sj;
  const long long c = (long long)i * si + (long long)j * sj + k;
  const long long ip = c + si, jp = c + sj, kp = c + 1;
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
  const float J1 = Q.J31[c], J2 = Q.J32[c], J3 = Q.J33[c];
  const float* Tt = Q.tau;
#define TT(m, x) Tt[(m) * n + (x)]
  // all loads before the first store: the compiler cannot tell the output from the inputs
  const float s0 = dXi * (TT(0, ip) - TT(0, c)) + dYi * (TT(1, jp) - TT(1, c)) + J1 * dXi * (TT(2, ip) - TT(2, c)) +
                   J2 * dYi * (TT(2, jp) - TT(2, c)) + J3 * dZi * (TT(2, kp) - TT(2, c));
  const float s1 = dXi * (TT(1, ip) - TT(1, c)) + dYi * (TT(4, jp) - TT(4, c)) + J1 * dXi * (TT(3, ip) - TT(3, c)) +
                   J2 * dYi * (TT(3, jp) - TT(3, c)) + J3 * dZi * (TT(3, kp) - TT(3, c));
  const float s2 = dXi * (TT(2, ip) - TT(2, c)) + dYi * (TT(3, jp) - TT(3, c)) + J1 * dXi * (TT(5, ip) - TT(5, c)) +
                   J2 * dYi * (TT(5, jp) - TT(5, c)) + J3 * dZi * (TT(5, kp) - TT(5, c));
  const float s3 = dXi * (TT(6, ip) - TT(6, c)) + dYi * (TT(7, jp) - TT(7, c)) + J1 * dXi * (TT(8, ip) - TT(8, c)) +
                   J2 * dYi * (TT(8, jp) - TT(8, c)) + J3 * dZi * (TT(8, kp) - TT(8, c));
  float sq[2] = {0.0f, 0.0f};
#pragma unroll
  for (int m = 0; m < NQ; m++) {
    const float* M = Q.mtau + 3 * m * n;
    sq[m] = dXi * (M[ip] - M[c]) + dYi * (M[n + jp] - M[n + c]) + J1 * dXi * (M[2 * n + ip] - M[2 * n + c]) +
            J2 * dYi * (M[2 * n + jp] - M[2 * n + c]) + J3 * dZi * (M[2 * n + kp] - M[2 * n + c]);
  }
  float se = 0.0f;
  if (TKE) {
    const float r0 = st[c];
    const float ri = rinv(r0);
    const float delta = grid_scale(P, Q, c);
    const float lsc = Q.ls[c];
    const float mec = st[5 * n + c];
    float Se = P.g / (st[4 * n + c] * ri) * TT(8, c);
    const float ce = (float)(1.9 * (double)P.c_k + (0.93 - 1.9 * (double)P.c_k) * (double)lsc / (double)delta);
    const float ec = mec * ri;
    Se = Se + (-ce * mec * sqrtf(ec) / lsc);
    // (rho phi)/rho of field f at the neighbour c + o, rounded on its own (as the fused SGS kernel's
    // shared-memory primitives are), so the differences below are not contracted into FMAs
    auto G = [&](int f, long long o) -> float { return __fmul_rn(st[f * n + c + o], rinv(st[c + o])); };
    const float ux = G(1, si) - G(1, -si), uy = G(1, sj) - G(1, -sj), uz = G(1, 1) - G(1, -1);
    const float vx = G(2, si) - G(2, -si), vy = G(2, sj) - G(2, -sj), vz = G(2, 1) - G(2, -1);
    const float wx = G(3, si) - G(3, -si), wy = G(3, sj) - G(3, -sj), wz = G(3, 1) - G(3, -1);
    const float dux = 0.5f * (dXi * ux), duy = 0.5f * (dYi * uy);
    const float duz = 0.5f * (J1 * dXi * ux + J2 * dYi * uy + J3 * dZi * uz);
    const float dvx = 0.5f * (dXi * vx), dvy = 0.5f * (dYi * vy);
    const float dvz = 0.5f * (J1 * dXi * vx + J2 * dYi * vy + J3 * dZi * vz);
    const float dwx = 0.5f * (dXi * wx), dwy = 0.5f * (dYi * wy);
    const float dwz = 0.5f * (J1 * dXi * wx + J2 * dYi * wy + J3 * dZi * wz);
    const float shear = (-TT(0, c) * dux) + (-TT(1, c) * duy) + (-TT(2, c) * duz) + (-TT(1, c) * dvx) +
                        (-TT(4, c) * dvy) + (-TT(3, c) * dvz) + (-TT(2, c) * dwx) + (-TT(3, c) * dwy) + (-TT(5, c) * dwz);
    Se = Se + shear;
    const float* Gq = Q.tkeQ;
    const long long im = c - si, jm = c - sj, km = c - 1;
    const float tx_ = -(dXi * (Gq[ip] - Gq[im]));
    const float ty_ = -(dYi * (Gq[n + jp] - Gq[n + jm]));
    const float tz_ = -(J1 * dXi * (Gq[2 * n + ip] - Gq[2 * n + im]) + J2 * dYi * (Gq[2 * n + jp] - Gq[2 * n + jm]) +
                        J3 * dZi * (Gq[2 * n + kp] - Gq[2 * n + km]));
    Se = Se + (-(tx_ + ty_ + tz_));
    se = Se;
  }
#undef TT
  // large-scale forcing of the last stage (cuda_hydroCoreDevice.cu:401-406)
  float lu = 0.0f, lv = 0.0f, lth = 0.0f, lqv = 0.0f;
  if (stage == 2 && lsf_step(P, *Q.clockIt)) lsf_tend(P, Q, c, k, Q.zPos[c], st[c], lu, lv, lth, lqv);
  float* S = Q.sgsF + c;
  S[0] = s0 - lu;
  S[n] = s1 - lv;
  S[2 * n] = s2;
  S[3 * n] = s3 - lth;
  if (TKE) S[4 * n] = se;
  if (NQ > 0) S[5 * n] = sq[0] - lqv;
  else if (P.lsf && P.moist) S[5 * n] = -lqv;
#pragma unroll
  for (int m = 1; m < NQ; m++) S[(5 + m) * n] = sq[m];
}

// MP: the saturation adjustment of the last stage. -1 decides per step from the device clock;
// 0 and 1 are the two halves of a pair launched back to back, each returning at once unless the
// step is its kind (0: no adjustment this step, compiled without the adjustment; 1: adjustment).
// The body of one thread block: tile (bx, by, bz) of the domain P / Q (k tile, j tile, i chunk).
template <int STAGE, int MODE, int TJ, int FL, int MP>
__device__ __forceinline__ void march_body(const Phys& P, const Ptrs& Q, const float* __restrict__ cur,
                                           const float* __restrict__ base, float* __restrict__ nxt,
                                           const float* __restrict__ pcur, float* __restrict__ pnxt,
                                           float* __restrict__ frhs, int ni, int bx, int by, int bz) {
  const int ntke = FL == FL_ANY ? P.ntke : 1;
  const int nmoist = FL == FL_ANY ? P.nmoist : ((FL == FL_MOIST || FL == FL_MOIST34) ? 2 : 0);
  const bool pgf = FL == FL_ANY ? (P.pgf != 0) : true;
  const bool tke = FL == FL_ANY ? (P.tke != 0) : true;
  // physics stages: every stage without oneRK, else the last; the flavours fix oneRK = 1
  const bool phys = FL == FL_ANY ? ((P.oneRK == 0) || (STAGE == 2)) : (STAGE == 2);
  const bool mpNow = phys && nmoist > 1 && P.moist && P.moistCond > 0 && ((*Q.clockIt) % P.mpFreq == 0);
  if ((MP == 0 && mpNow) || (MP == 1 && !mpNow)) return;  // the other half of the pair runs this step
  const bool mpStep = MP == 0 ? false : mpNow;
  // large-scale forcing inline only without the SGS kernel (which otherwise carries it)
  const bool lsfNow = STAGE == 2 && FL == FL_ANY && !P.turb && lsf_step(P, *Q.clockIt);
  using T = MarchTile<TJ>;
  constexpr int PK = T::PK, PLANE = T::PLANE;
  extern __shared__ __align__(16) float sm[];

  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * MK + tx;
  const int k0 = P.kMin + bx * MK, j0 = P.jMin + by * TJ;
  const int i0 = P.iMin + bz * ni;
  const int i1 = min(i0 + ni, P.iMax);
  const int k = k0 + tx, j = j0 + ty;
  const bool inArr = (k < P.nzh) && (j < P.nyh);     // the thread's column exists in memory
  const bool active = (k < P.kMax) && (j < P.jMax);  // ... and is an interior column
  const long long n = P.n;
  const int si = P.si, sj = P.sj;
  const long long col = (long long)j * sj + k;
  const long long tile0 = (long long)j0 * sj + k0;
  const int own = (ty + 3) * PK + (tx + 3);
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;

  // ring cells of the staged planes handled by this thread
  int rS[T::RPT], rG[T::RPT];
  bool rV[T::RPT], rN[T::RPT];
#pragma unroll
  for (int q = 0; q < T::RPT; q++) {
    const int r = tid + q * T::NT;
    rV[q] = false; rN[q] = false; rS[q] = 0; rG[q] = 0;
    if (r < T::RING) {
      int row, cl;
      march_ring_cell<TJ>(r, row, cl);
      const int jj = j0 + row - 3, kk = k0 + cl - 3;
      rV[q] = (jj < P.nyh) && (kk < P.nzh);
      rN[q] = row >= 2 && row <= TJ + 3 && cl >= 2 && cl <= MK + 3;  // within one cell (p' ring)
      rS[q] = row * PK + cl;
      rG[q] = (row - 3) * sj + (cl - 3);
    }
  }
  // velocity-plane ring task: cy at rows -1 and TJ, or cz at columns -1 and MK
  int rtKind = 0, rtS = 0;
  long long rtOff = 0;
  {
    int row = 0, cc = 0;
    if (tid < T::CYT) {
      rtKind = 1; row = (tid < MK) ? -1 : TJ; cc = tid & (MK - 1);
      rtS = (row + 1) * MK + cc;
    } else if (tid < T::CYT + T::CZT) {
      const int q = tid - T::CYT;
      rtKind = 2; row = q >> 1; cc = (q & 1) ? MK : -1;
      rtS = T::CYN + row * T::CZK + (cc + 1);
    }
    const int jj = j0 + row, kk = k0 + cc;
    if (rtKind && !(jj < P.nyh && kk < P.nzh)) rtKind = 0;
    rtOff = (long long)jj * sj + kk;
  }

  auto issue_ring = [&](int ip, float* buf) {
    const long long pl = (long long)ip * si + tile0;
#pragma unroll
    for (int s = 0; s < MSLOTS; s++) {
      if (!f_on<FL>(P, s)) continue;
      const float* src = f_src<FL>(P, cur, pcur, s) + pl;
#pragma unroll
      for (int q = 0; q < T::RPT; q++)
        if (rV[q] && (s != SL_P || rN[q])) cp_async4(buf + s * PLANE + rS[q], src + rG[q]);
    }
    cp_async_commit();
  };

  // ---------------------------------------------------------------- prologue (plane i0)
  // buffers: plane i0 -> 0, plane i0+1 -> 1 (holds s(i0-2) at the own cell until it is
  // refilled), plane i0-1 -> 2
  float w[8][4];
  float pc1 = 0.0f;   // p'(i+1)
  float Dc = 0.0f, Dn = 0.0f, J1c = 0.0f, J1n = 0.0f, J2c = 0.0f, J3c = 0.0f;
  const long long cA = (long long)i0 * si + col;
#pragma unroll
  for (int s = 0; s < 8; s++) {
#pragma unroll
    for (int d = 0; d < 4; d++) w[s][d] = 0.0f;
  }
  float* const B0 = sm;
  float* const B1 = sm + T::BUF;
  float* const B2 = sm + 2 * T::BUF;
  float* const aux = sm + T::NBUF * T::BUF;   // [2][NAUX][NT]
  float* const xcs = aux + T::AUX;            // [8][NT]
  // the inputs of step ib+1 (loaded during step ib): slots 0..7 s(ib+4), 8 p'(ib+2), 9 D(ib+2),
  // 10 J31(ib+2), 11 J32(ib+2), 12 J33(ib+2), 13 invD(ib+1)
  auto issue_aux = [&](int ib, float* tbl) {
    float* const buf = tbl + tid;  // this thread's entry of each slot
    const long long c = (long long)ib * si + col;
    if (inArr) {
      if (ib + 4 < P.nxh) {
#pragma unroll
        for (int s = 0; s < 8; s++)
          if (f_on<FL>(P, s)) cp_async4(buf + s * T::NT, f_src<FL>(P, cur, pcur, s) + c + 4 * (long long)si);
      }
      if (pgf) cp_async4(buf + 8 * T::NT, pcur + c + 2 * (long long)si);
      cp_async4(buf + 9 * T::NT, Q.D + c + 2 * (long long)si);
      cp_async4(buf + 10 * T::NT, Q.J31 + c + 2 * (long long)si);
      cp_async4(buf + 11 * T::NT, Q.J32 + c + 2 * (long long)si);
      cp_async4(buf + 12 * T::NT, Q.J33 + c + 2 * (long long)si);
      cp_async4(buf + 13 * T::NT, Q.invD + c + si);
    }
    cp_async_commit();
  };
  if (!inArr) {
    for (int q = 0; q < 2 * T::NAUX; q++) aux[q * T::NT + tid] = 0.0f;
    for (int q = 0; q < 8; q++) xcs[q * T::NT + tid] = 0.0f;
  }
  issue_aux(i0 - 1, aux + T::NAUX * T::NT);  // read by step i0 (buffer 1)
  float Dm1 = 0.0f, J1m1 = 0.0f, rm1 = 0.0f, um1 = 0.0f, wm1 = 0.0f, p0v = 0.0f, pm1 = 0.0f;
  if (inArr) {
    Dm1 = Q.D[cA - si]; Dc = Q.D[cA];
    J1m1 = Q.J31[cA - si]; J1c = Q.J31[cA];
    J2c = Q.J32[cA]; J3c = Q.J33[cA];
    if (pgf) { pm1 = pcur[cA - si]; p0v = pcur[cA]; }
  }
#pragma unroll
  for (int s = 0; s < 8; s++) {
    if (!f_on<FL>(P, s)) continue;
    const float* src = f_src<FL>(P, cur, pcur, s);
    float sm2 = 0.0f, sm1 = 0.0f;
    if (inArr) {
      sm2 = src[cA - 2 * (long long)si]; sm1 = src[cA - si];
#pragma unroll
      for (int d = 0; d < 3; d++) w[s][d] = src[cA + d * (long long)si];
    }
    B1[s * PLANE + own] = sm2;
    B2[s * PLANE + own] = sm1;
    B0[s * PLANE + own] = w[s][0];
    if (s == 0) rm1 = sm1;
    if (s == 1) um1 = sm1;
    if (s == 3) wm1 = sm1;
  }
  if (pgf) { B0[SL_P * PLANE + own] = p0v; B2[SL_P * PLANE + own] = pm1; }
  float cx0 = contra(Dc, w[0][0], w[1][0], w[3][0], J1c);
  float upPrev;
  {
    const float cxm = contra(Dm1, rm1, um1, wm1, J1m1);
    upPrev = (0.5f * dXi) * (cx0 + cxm);  // velocity of the face i0-1/2
#pragma unroll
    for (int s = 0; s < 8; s++) {
      if (!f_on<FL>(P, s)) continue;
      const float* src = f_src<FL>(P, cur, pcur, s);
      const float m3 = inArr ? src[cA - 3 * (long long)si] : 0.0f;
      const float m2 = B1[s * PLANE + own], m1 = B2[s * PLANE + own];
      const float f = adv_face<true>(f_sel<FL>(P, s), m3, m2, m1, w[s][0], w[s][1], w[s][2], upPrev, 1.0f - slot_b(P, s));
      xcs[s * T::NT + tid] = __fmul_rn(upPrev, f);
    }
  }
  float cyOwn, czOwn;
  {
    issue_ring(i0, B0);
    cyOwn = contra(Dc, w[0][0], w[2][0], w[3][0], J2c);
    czOwn = contra_z(Dc, w[0][0], w[3][0], J3c);
    float* v = B0 + MSLOTS * PLANE;
    v[(ty + 1) * MK + tx] = cyOwn;
    v[T::CYN + ty * T::CZK + tx + 1] = czOwn;
    if (rtKind) {
      const long long c = (long long)i0 * si + rtOff;
      const float D = Q.D[c], r = cur[c];
      v[rtS] = rtKind == 1 ? contra(D, r, cur[2 * n + c], cur[3 * n + c], Q.J32[c]) : contra_z(D, r, cur[3 * n + c], Q.J33[c]);
    }
    cp_async_wait_all();
    __syncthreads();
  }

  const bool same = (base == cur);  // first stage: the commit base is the input state

  // ---------------------------------------------------------------- march
  float *cs = B0, *ns = B1, *ps = B2;  // planes i, i+1 (own cell: s(i-2) until refilled), i-1
  for (int i = i0; i < i1; i++) {
    const bool more = (i + 1 < i1);
    const long long c = (long long)i * si + col;

    // this plane's table (loaded during the previous step): the new end of the x window and the
    // metrics of plane i+1; then start the next one
    const float* ax = aux + ((i - i0 + 1) & 1) * T::NAUX * T::NT + tid;
#pragma unroll
    for (int s = 0; s < 8; s++)
      if (f_on<FL>(P, s)) w[s][3] = ax[s * T::NT];
    if (pgf) pc1 = ax[8 * T::NT];
    Dn = ax[9 * T::NT];
    J1n = ax[10 * T::NT];
    // the next plane's single-cell reads (commit base, base state, SGS fields written by the
    // physics kernel) into L2 while this plane is computed
    if (more && active) {
      const long long cn = c + si;
      if (MODE != MODE_FRHS && !same) {
#pragma unroll
        for (int s = 0; s < 8; s++)
          if (f_on<FL>(P, s)) prefetch_l2(f_src<FL>(P, base, pcur, s) + cn);
      }
      if (MODE != MODE_FRHS) prefetch_l2(Q.pBS + cn);
      if (P.buoy || P.cor || P.damp) prefetch_l2(Q.rhoBS + cn);
      if (P.cor || P.damp) prefetch_l2(Q.zPos + cn);
      if (phys && P.turb) {
#pragma unroll
        for (int m = 0; m < 5; m++) prefetch_l2(Q.sgsF + m * n + cn);
        if (nmoist > 0 && P.moistSGS > 0)
          for (int m = 0; m < nmoist; m++) prefetch_l2(Q.sgsF + (5 + m) * n + cn);
      }
    }
    // inputs of this plane's commit, loaded before the advection so that their memory latency
    // overlaps it (and before any store of the plane: the stores may alias `base`)
    float cb[8];
    float pbs = 0.0f;
#pragma unroll
    for (int s = 0; s < 8; s++) cb[s] = 0.0f;
    if (MODE != MODE_FRHS && active) {
#pragma unroll
      for (int s = 0; s < 8; s++)
        if (f_on<FL>(P, s) && !same) cb[s] = f_src<FL>(P, base, pcur, s)[c];
      pbs = Q.pBS[c];
    }
    // SGS tendencies of this cell (k_sgs_tend): stress divergence on rho u, rho v, rho w, heat
    // flux divergence, the TKE budget, moisture flux divergences
    float sg[7];
#pragma unroll
    for (int m = 0; m < 7; m++) sg[m] = 0.0f;
    if (phys && P.turb && active) {
#pragma unroll
      for (int m = 0; m < 4; m++) sg[m] = Q.sgsF[m * n + c];
      if (tke) sg[4] = Q.sgsF[4 * n + c];
      if (nmoist > 0 && (P.moistSGS > 0 || P.lsf)) {
        sg[5] = Q.sgsF[5 * n + c];
        if (nmoist > 1 && P.moistSGS > 0) sg[6] = Q.sgsF[6 * n + c];
      }
    }
    // base state of the buoyancy, Rayleigh and Coriolis terms
    float zc = 0.0f, ztop = 0.0f, rbsc = 0.0f;
    if (inArr) {
      if (P.buoy || P.cor || P.damp) rbsc = Q.rhoBS[c];
      if (P.cor || P.damp) zc = Q.zPos[c];
      if (P.damp) ztop = Q.zPos[c - k + (P.kMax - 1)];
    }
    if (more) issue_aux(i, aux + ((i - i0) & 1) * T::NAUX * T::NT);
    if (more) issue_ring(i + 1, ns);
    float rD = 0.0f, rR = 1.0f, rM = 0.0f, rW = 0.0f, rJ = 0.0f;
    if (more && rtKind) {
      const long long cr = (long long)(i + 1) * si + rtOff;
      rD = Q.D[cr]; rR = cur[cr]; rW = cur[3 * n + cr];
      if (rtKind == 1) { rM = cur[2 * n + cr]; rJ = Q.J32[cr]; }
      else rJ = Q.J33[cr];
    }

    // face velocities of this cell (cuda_advectionDevice.cu:89-106)
    const float dr1 = __fdiv_rn(Dn, w[0][1]);  // D/rho of plane i+1, shared by its three velocities
    const float cxp1 = contra_dr(dr1, w[1][1], w[3][1], J1n);
    const float up = (0.5f * dXi) * (cxp1 + cx0);
    const float* cyP = cs + MSLOTS * PLANE;
    const float* czP = cyP + T::CYN;
    const float vm = (0.5f * dYi) * (cyOwn + cyP[ty * MK + tx]);
    const float vp = (0.5f * dYi) * (cyP[(ty + 2) * MK + tx] + cyOwn);
    const float wm = (k == P.kMin) ? 0.0f : (0.5f * dZi) * (czOwn + czP[ty * T::CZK + tx]);
    const float wp = (k + 1 >= P.kMax) ? 0.0f : (0.5f * dZi) * (czP[ty * T::CZK + tx + 2] + czOwn);

    const float J1 = J1c, J2 = J2c, J3 = J3c;
    const float invD = ax[13 * T::NT];
    const float r0 = w[0][0];
    // The moist PGF, Coriolis and Rayleigh terms divide by rho and rho_BS through one correctly
    // rounded reciprocal per block (phi * (1/rho) instead of phi / rho: within an ulp).
    float F[8];
    float fw = 0.0f;  // explicit filter of rho w (filterSelector = 1)
#pragma unroll
    for (int s = 0; s < 8; s++) F[s] = 0.0f;

    // pressure-gradient force (cuda_pressureDevice.cu:118-194)
    if (pgf) {
      const float* pp = cs + SL_P * PLANE + own;
      const float dpx = pc1 - ps[SL_P * PLANE + own];
      const float dpy = pp[PK] - pp[-PK];
      const float dpz = pp[1] - pp[-1];
      if (nmoist > 0) {
        const float rr0 = 1.0f / r0;
        float rmd = 1.0f;
        rmd = (float)((double)rmd + (double)(w[SL_QV][0] * rr0) * 1e-3);
        if (nmoist > 1) rmd = (float)((double)rmd + (double)(w[SL_QL][0] * rr0) * 1e-3);
        const float rdm = 1.0f / rmd;
        F[1] = (float)((double)F[1] - (double)rdm * 0.5 * (double)dXi * (double)dpx);
        F[2] = (float)((double)F[2] - (double)rdm * 0.5 * (double)dYi * (double)dpy);
        F[3] = (float)((double)F[3] - (double)rdm * 0.5 * (double)(dXi * J1 * dpx + dYi * J2 * dpy + dZi * J3 * dpz));
      } else {
        F[1] = F[1] - (0.5f * dXi) * dpx;
        F[2] = F[2] - (0.5f * dYi) * dpy;
        F[3] = F[3] - 0.5f * (dXi * J1 * dpx + dYi * J2 * dpy + dZi * J3 * dpz);
      }
    }

    // advection of every field (cuda_hydroCoreDevice.cu:631-736; WENO3/WENO5 as x, y, z updates)
    float fxNext = 0.0f;  // x face of field s + 1 when it was evaluated with field s
#pragma unroll
    for (int s = 0; s < 8; s++) {
      if (!f_on<FL>(P, s)) continue;
      const float* pl = cs + s * PLANE + own;
      const float z0 = w[s][0];
      const float xm2 = ns[s * PLANE + own], xm1 = ps[s * PLANE + own];
      const int sel = f_sel<FL>(P, s);
      const float bf = adv_split(sel) ? 1.0f : 1.0f - slot_b(P, s);
      // the x faces of an even and the following odd field as a lane pair when both use the same
      // packed scheme (compile-time flavours only)
      float fxp;
      if (x_paired<FL>(s)) {
        const int s1 = s + 1;
        const float bf1 = adv_split(sel) ? 1.0f : 1.0f - slot_b(P, s1);
        const float2 fx = adv_face2<true>(sel, f2(xm2, ns[s1 * PLANE + own]), f2(xm1, ps[s1 * PLANE + own]),
                                          f2(z0, w[s1][0]), f2(w[s][1], w[s1][1]), f2(w[s][2], w[s1][2]),
                                          f2(w[s][3], w[s1][3]), f2s(up), f2(bf, bf1));
        fxp = fx.x;
        fxNext = fx.y;
      } else if (s > 0 && x_paired<FL>(s - 1)) {
        fxp = fxNext;
      } else {
        fxp = adv_face<true>(sel, xm2, xm1, z0, w[s][1], w[s][2], w[s][3], up, bf);
      }
      const float pxp = __fmul_rn(up, fxp);
      const float Dx = __fsub_rn(pxp, xcs[s * T::NT + tid]);
      xcs[s * T::NT + tid] = pxp;
      // moist flavours: the two y faces, then the two z faces, as lane pairs (upper face, lower
      // face) on the packed pipe; the other flavours face by face (their register budget has no
      // room for the pairs)
      float Dy, Dz;
      {
        const float m3 = pl[-3 * PK], m2 = pl[-2 * PK], m1 = pl[-PK], p1 = pl[PK], p2 = pl[2 * PK], p3 = pl[3 * PK];
        if constexpr (FL == FL_MOIST || FL == FL_MOIST34) {
          const float2 v2 = f2(vp, vm);
          const float2 fy = adv_face2<true>(sel, f2(m2, m3), f2(m1, m2), f2(z0, m1), f2(p1, z0), f2(p2, p1), f2(p3, p2),
                                            v2, f2s(bf));
          const float2 py = mul2(v2, fy);
          Dy = __fsub_rn(py.x, py.y);
        } else {
          Dy = vp * adv_face<true>(sel, m2, m1, z0, p1, p2, p3, vp, bf) - vm * adv_face<true>(sel, m3, m2, m1, z0, p1, p2, vm, bf);
        }
      }
      {
        const float m3 = pl[-3], m2 = pl[-2], m1 = pl[-1], p1 = pl[1], p2 = pl[2], p3 = pl[3];
        if constexpr (FL == FL_MOIST || FL == FL_MOIST34) {
          const float2 w2 = f2(wp, wm);
          const float2 fz = adv_face2<true>(sel, f2(m2, m3), f2(m1, m2), f2(z0, m1), f2(p1, z0), f2(p2, p1), f2(p3, p2),
                                            w2, f2s(bf));
          const float2 pz = mul2(w2, fz);
          Dz = __fsub_rn(pz.x, pz.y);
        } else {
          Dz = wp * adv_face<true>(sel, m2, m1, z0, p1, p2, p3, wp, bf) - wm * adv_face<true>(sel, m3, m2, m1, z0, p1, p2, wm, bf);
        }
        // the explicit filter of rho w reads the same column; it is added after every other term
        if (s == 3 && P.filt) fw = filter6_tend(m3, m2, m1, z0, p1, p2, p3, P.filtCoef);
      }
      if (adv_split(sel)) {
        // WENO: x, y and z as three separate updates
        F[s] = F[s] - invD * Dx;
        F[s] = F[s] - invD * Dy;
        F[s] = F[s] - invD * Dz;
      } else {
        F[s] = F[s] - invD * (Dx + Dy + Dz);
      }
      if (s == 3) {
        // Rayleigh damping and buoyancy act on F_w right after its advection
        if (P.damp && inArr) {
          const float z = zc, zt = ztop;
          if (z >= (zt - P.dampDepth)) {
            const float rbs = rbsc, rr0 = 1.0f / r0, rrb = 1.0f / rbs;
            const float wbs = momentum_bs(P, 3, z, rbs);
            const float pio2 = 1.5707963267948966f;
            const double sn = (double)sinf((float)((double)pio2 * (1.0 - (double)((zt - z) / P.dampDepth))));
            F[3] = (float)((double)F[3] - 0.2 * (double)r0 * (sn * sn) * (double)(w[3][0] * rr0 - wbs * rrb));
          }
        }
        if (P.buoy) {
          const float rbs = rbsc;
          if (nmoist > 0) {
            double rm = (double)r0 + (double)w[SL_QV][0] * 1e-3;
            if (nmoist == 2) rm += (double)w[SL_QL][0] * 1e-3;
            const float ratio = r0 / (float)rm;
            F[3] = (float)((double)F[3] - (double)(ratio * P.g) * (rm - (double)rbs));
          } else {
            F[3] = F[3] - P.g * (r0 - rbs);
          }
        }
      }
    }

    // Coriolis (cuda_coriolisDevice.cu:50-58)
    if (P.cor && inArr) {
      const float z = zc, rbs = rbsc;
      const float ubs = momentum_bs(P, 1, z, rbs), vbs = momentum_bs(P, 2, z, rbs), wbs = momentum_bs(P, 3, z, rbs);
      const float rr0 = 1.0f / r0, rrb = 1.0f / rbs;
      const float u0 = w[1][0] * rr0, v0 = w[2][0] * rr0, w0 = w[3][0] * rr0;
      const float ug = P.fLS * ubs * rrb, vg = P.fLS * vbs * rrb, wg = P.fLS * wbs * rrb;
      F[1] = F[1] + (P.fHorz * (v0 - vg) - P.fVert * (w0 - wg));
      F[2] = F[2] - (P.fHorz * (u0 - ug));
      F[3] = F[3] + (P.fVert * (u0 - ug));
    }

    if (phys && P.turb && active) {
      F[1] = F[1] - sg[0];
      F[2] = F[2] - sg[1];
      F[3] = F[3] - sg[2];
      F[4] = F[4] - sg[3];
      if (tke) F[SL_E] = F[SL_E] + sg[4];
      if (nmoist > 0 && (P.moistSGS > 0 || P.lsf)) {
        F[SL_QV] = F[SL_QV] - sg[5];
        if (nmoist > 1 && P.moistSGS > 0) F[SL_QL] = F[SL_QL] - sg[6];
      }
    }

    // saturation adjustment (cuda_moistureDevice.cu:80-247)
    if (mpStep && active) {
      const float ri = rinv(r0);
      const float mth = w[4][0];
      const float thd = mth * ri;
      const float prd = P.condBasePres == 1 ? powf(Q.thBS[c] * P.c1, P.cp_cv) : powf(mth * P.c1, P.cp_cv);
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
      const float flim = w[SL_QL][0] * 1e-3f;
      if (P.moistCond == 1) {
        ffor = w[SL_QV][0] * 1e-3f - (pvs / (P.R_vapor * Td));
      } else if (P.moistCond == 2) {
        const float rv = w[SL_QV][0] * 1e-3f, rvs = pvs / (P.R_vapor * Td);
        ffor = (rv - rvs) / (1.0f + (powf(P.L_v, 2.0f) * rvs * ri / (P.cp_gas * P.R_vapor * powf(Td, 2.0f))));
      } else {
        const float rv = w[SL_QV][0] * 1e-3f;
        float rvs = pvs / (prd - pvs) / P.Rv_Rg;
        rvs = rvs / ri;
        ffor = (rv - rvs) / (1.0f + (powf(P.L_v, 2.0f) * rvs * ri / (P.cp_gas * P.R_vapor * powf(Td, 2.0f))));
      }
      float fc = fmaxf(ffor, 0.0f) - fmaxf(fminf(flim, -ffor), 0.0f);
      fc = fc / P.condTscale;
      F[SL_QV] = F[SL_QV] - fc * 1e3f;
      F[SL_QL] = F[SL_QL] + fc * 1e3f;
      const float prd2 = powf(mth * P.c1, P.cp_cv);
      const float Td2 = thd * powf(prd2 / P.p0, P.R_cp);
      F[4] = F[4] + ((thd * P.L_v) / (Td2 * P.cp_gas)) * fc;
    }
    // large-scale forcing in the last stage (cuda_hydroCoreDevice.cu:401-406)
    if (lsfNow && active) lsf_tend(P, Q, c, k, Q.zPos[c], r0, F[1], F[2], F[4], F[SL_QV]);
    // explicit filter of rho w, every stage, after all other terms (cuda_hydroCoreDevice.cu:414-416)
    if (P.filt) F[3] = __fadd_rn(F[3], fw);

    if (active) {
      if (MODE == MODE_FRHS) {
        frhs[c] = F[0];
        frhs[n + c] = F[1];
        frhs[2 * n + c] = F[2];
        frhs[3 * n + c] = F[3];
        frhs[4 * n + c] = F[4];
        if (ntke) frhs[5 * n + c] = F[SL_E];
        if (nmoist > 0) frhs[(5 + ntke) * n + c] = F[SL_QV];
        if (nmoist > 1) frhs[(6 + ntke) * n + c] = F[SL_QL];
      } else {
        if (STAGE == 2 && frhs) {
          // the last stage's tendencies, kept when asked (the reference's Frhs after a step)
          frhs[c] = F[0];
          frhs[n + c] = F[1];
          frhs[2 * n + c] = F[2];
          frhs[3 * n + c] = F[3];
          frhs[4 * n + c] = F[4];
          if (ntke) frhs[5 * n + c] = F[SL_E];
          if (nmoist > 0) frhs[(5 + ntke) * n + c] = F[SL_QV];
          if (nmoist > 1) frhs[(6 + ntke) * n + c] = F[SL_QL];
        }
        // WS2002 RK3 commit (cuda_RKschemes.cu:113-157), rounding as in the cell kernel
        auto rk = [&](float phi0, float Fv) -> float {
          if (STAGE == 0) return (float)fma((1.0 / 3.0) * (double)P.dt, (double)Fv, (double)phi0);
          if (STAGE == 1) return (float)fma(0.5 * (double)P.dt, (double)Fv, (double)phi0);
          return __fmaf_rn(P.dt, Fv, phi0);
        };
        auto b0 = [&](int s) -> float { return same ? w[s][0] : cb[s]; };
        const long long oq = (5 + ntke) * n;
        const float a0 = b0(0), a1 = b0(1), a2 = b0(2), a3 = b0(3), a4 = b0(4);
        const float ae = ntke ? b0(SL_E) : 0.0f;
        const float aq0 = nmoist > 0 ? b0(SL_QV) : 0.0f;
        const float aq1 = nmoist > 1 ? b0(SL_QL) : 0.0f;
        const bool atBot = (k == P.kMin), atTop = (k == P.kMax - 1);
        Level0 l0{};
        if (atBot) l0 = level0_inputs(Q, c - k);
        const float n0 = rk(a0, F[0]);
        const float n1 = rk(a1, F[1]);
        const float n2 = rk(a2, F[2]);
        const float n3 = rk(a3, F[3]);
        const float n4 = rk(a4, F[4]);
        const float ne = ntke ? fmaxf(rk(ae, F[SL_E]), 1e-10f) : 0.0f;
        const float nq0 = nmoist > 0 ? fmaxf(rk(aq0, F[SL_QV]), 0.0f) : 0.0f;
        const float nq1 = nmoist > 1 ? fmaxf(rk(aq1, F[SL_QL]), 0.0f) : 0.0f;
        float pn;
        {
          float rtm = n4;
          if (nmoist > 0) rtm = (float)((double)n4 * (1.0 + (double)(P.Rv_Rg * nq0 / n0) * 1e-3));
          pn = powf(rtm * P.c1, P.cp_cv) - pbs;
        }
        const float p0 = atBot ? level0_pressure(P, l0, nmoist, nq0) : 0.0f;
        // The stores: cells within 3 of an x or y edge also write their periodic images (and,
        // at the first and last level, the images' halo copies); every other cell writes one
        // value per field and, at the first and last level, the halo copies below and above.
        const bool xyEdge = (i < P.iMin + 3) || (i >= P.iMax - 3) || (j < P.jMin + 3) || (j >= P.jMax - 3);
        if (xyEdge) {
          store_images(P, nxt, i, j, k, n0, 0, false);
          store_images(P, nxt + n, i, j, k, n1, atBot ? 3 : 0, false);
          store_images(P, nxt + 2 * n, i, j, k, n2, atBot ? 3 : 0, false);
          store_images(P, nxt + 3 * n, i, j, k, n3, atBot ? 3 : 0, false);
          store_images(P, nxt + 4 * n, i, j, k, n4, 0, false);
          if (ntke) store_images(P, nxt + 5 * n, i, j, k, ne, atBot ? 3 : 0, false);
          if (nmoist > 0) store_images(P, nxt + oq, i, j, k, nq0, atBot ? 3 : 0, atTop);
          if (nmoist > 1) store_images(P, nxt + oq + n, i, j, k, nq1, atBot ? 3 : 0, atTop);
          store_images(P, pnxt, i, j, k, pn, atBot ? 2 : 0, atTop);
        } else {
          nxt[c] = n0;
          nxt[n + c] = n1;
          nxt[2 * n + c] = n2;
          nxt[3 * n + c] = n3;
          nxt[4 * n + c] = n4;
          if (ntke) nxt[5 * n + c] = ne;
          if (nmoist > 0) nxt[oq + c] = nq0;
          if (nmoist > 1) nxt[oq + n + c] = nq1;
          pnxt[c] = pn;
          if (atBot) {
#pragma unroll
            for (int h = 1; h <= 3; h++) {
              nxt[n + c - h] = n1;
              nxt[2 * n + c - h] = n2;
              nxt[3 * n + c - h] = n3;
              if (ntke) nxt[5 * n + c - h] = ne;
              if (nmoist > 0) nxt[oq + c - h] = nq0;
              if (nmoist > 1) nxt[oq + n + c - h] = nq1;
              if (h <= 2) pnxt[c - h] = pn;
            }
          }
          if (atTop) {
#pragma unroll
            for (int h = 1; h <= 3; h++) {
              if (nmoist > 0) nxt[oq + c + h] = nq0;
              if (nmoist > 1) nxt[oq + n + c + h] = nq1;
              pnxt[c + h] = pn;
            }
          }
        }
        if (atBot) store_images(P, pnxt, i, j, 0, p0, 0, false);
      }
    }

    // plane i+1 into the other buffer: own values, contravariant velocities, ring tasks
    float cyN = 0.0f, czN = 0.0f;
    if (more) {
#pragma unroll
      for (int s = 0; s < 8; s++)
        if (f_on<FL>(P, s)) ns[s * PLANE + own] = w[s][1];
      if (pgf) ns[SL_P * PLANE + own] = pc1;
      cyN = contra_dr(dr1, w[2][1], w[3][1], ax[11 * T::NT]);
      czN = contra_z_dr(dr1, w[3][1], ax[12 * T::NT]);
      float* v = ns + MSLOTS * PLANE;
      v[(ty + 1) * MK + tx] = cyN;
      v[T::CYN + ty * T::CZK + tx + 1] = czN;
      if (rtKind) v[rtS] = rtKind == 1 ? contra(rD, rR, rM, rW, rJ) : contra_z(rD, rR, rW, rJ);
    }
    // shift the x window and the carried values
#pragma unroll
    for (int s = 0; s < 8; s++) {
#pragma unroll
      for (int d = 0; d < 3; d++) w[s][d] = w[s][d + 1];
    }
    cx0 = cxp1; upPrev = up;
    Dc = Dn; J1c = J1n; J2c = ax[11 * T::NT]; J3c = ax[12 * T::NT];
    cyOwn = cyN; czOwn = czN;
    float* const t = ps;
    ps = cs; cs = ns; ns = t;
    cp_async_wait_all();
    __syncthreads();
  }
}

template <int STAGE, int MODE, int TJ, int FL, int MP = -1>
__global__ void __launch_bounds__(MK * TJ, 512 / (MK * TJ))
    k_march(Phys P, Ptrs Q, const float* __restrict__ cur, const float* __restrict__ base, float* __restrict__ nxt,
            const float* __restrict__ pcur, float* __restrict__ pnxt, float* __restrict__ frhs, int ni) {
  march_body<STAGE, MODE, TJ, FL, MP>(P, Q, cur, base, nxt, pcur, pnxt, frhs, ni, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One member of a batched launch: its domain, the buffers of the stage, its planes per block and
// its share of the launch's thread blocks (blocks first .. first + gx*gy*gz - 1).
struct MarchMember {
  Phys P;
  Ptrs Q;
  const float *cur, *base, *pcur;
  float *nxt, *pnxt;
  int ni, gx, gy, first;
};

// The stage kernel of several domains in one launch (a work list of tiles across uneven members):
// block b reads its member from the block map, copies that member's parameters into shared memory
// and runs the member's tile.
template <int STAGE, int TJ, int FL, int MP = -1>
__global__ void __launch_bounds__(MK * TJ, 512 / (MK * TJ))
    k_march_list(const MarchMember* __restrict__ mem, const int* __restrict__ bmap) {
  __shared__ MarchMember sm_m;
  __shared__ int sm_idx;
  const int tid = threadIdx.y * MK + threadIdx.x;
  if (tid == 0) sm_idx = bmap[blockIdx.x];
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(mem + sm_idx);
    int* dst = reinterpret_cast<int*>(&sm_m);
    for (int q = tid; q < (int)(sizeof(MarchMember) / sizeof(int)); q += MK * TJ) dst[q] = src[q];
  }
  __syncthreads();
  const MarchMember& m = sm_m;
  const int local = (int)blockIdx.x - m.first;
  const int bx = local % m.gx, by = (local / m.gx) % m.gy, bz = local / (m.gx * m.gy);
  march_body<STAGE, MODE_COMMIT, TJ, FL, MP>(m.P, m.Q, m.cur, m.base, m.nxt, m.pcur, m.pnxt, nullptr, m.ni, bx, by, bz);
}

}  // namespace fe
