// fe_sgs_march.cuh -- the last RK stage's SGS physics and the tendencies it gives, in one
// i-marching kernel (sm_100a).
//
// The SGS tendencies of a cell (stress and heat-flux divergences, cuda_sgsTurbDevice.cu:447-547;
// the TKE budget, cuda_sgstkeDevice.cu:155-397; moisture flux divergences) read the closure's
// stresses and fluxes at the cell and one cell forward in each direction, and the TKE transport
// fluxes one cell back and forward. Evaluating those per point into global scratch and reading
// them back in a second kernel moves ~300 B per cell through HBM; here a thread block owns a tile
// of 32 levels (one warp) x TJ rows and marches along i:
//
//   primitives   phi/rho of 8 fields in three rotating shared-memory planes (i, i+1, i+2), each
//                with the ring the physics stencil needs (rows j0-2..j0+TJ+1, levels k0-3..k0+33)
//   physics      the closure's outputs of plane i+1 for rows j0-1..j0+TJ, levels k0-1..k0+32 into
//                the "next" physics buffer (turb_point, the same arithmetic as the per-point
//                kernels), the length scale first into its own table
//   tendencies   of plane i from the "current" (i) and "next" (i+1) physics planes; what plane i-1
//                contributes (u, v, w for the shear production, the x and z TKE fluxes) is carried
//                in registers by each thread
//
// and writes only the 7 SGS tendency fields the last stage's march kernel reads (and, when asked,
// the stresses and fluxes themselves, for callers that copy them back). The first-level stresses
// of the surface columns come from the surface-layer kernel, launched before this one. With the
// learned closure, the 9 stresses of every ring point come from the network's output (written by
// the inference kernel, launched before this one), the other closure outputs from the closure.
// Results equal the two-kernel form (k_turb_t + k_turb_ring [+ inference] + k_sgs_tend) bit for bit.
#pragma once
#include "fe_kernels.cuh"

namespace fe {

constexpr int SG_K = 32;  // output levels per tile

template <int TJ>
struct SgsTile {
  static constexpr int NT = SG_K * TJ;
  static constexpr int PRJ = TJ + 4, PRK = SG_K + 5, PRN = PRJ * PRK;  // rows j0-2.., levels k0-3..
  static constexpr int NPF = 8;                                      // rho, u, v, w, th, e, qv, ql (phi/rho)
  static constexpr int PHJ = TJ + 2, PHK = SG_K + 2, PHN = PHJ * PHK;  // rows j0-1.., levels k0-1..
  static constexpr int NPH = 19;                                     // tau 0..8, tkeQ 9..11, mtau 12..17, ls 18
  static constexpr int LSK = SG_K + 3, LSN = PHJ * LSK;              // levels k0-2..k0+32
  static constexpr int FLOATS = 3 * NPF * PRN + 2 * NPH * PHN + 2 * LSN + 4 * LSN;  // + J31, J32, J33, delta
  static constexpr int SMEM_BYTES = FLOATS * 4;
};

// Primitive variables of a point from three shared-memory planes (the point's plane and its two
// neighbours in i).
template <int TJ>
struct RingPrims {
  const float* pm;  // plane i-1
  const float* p0;  // plane i
  const float* pp;  // plane i+1
  int o;            // the point within a plane
  __device__ __forceinline__ float at(int f, int di, int dj, int dk) const {
    const float* b = di < 0 ? pm : (di > 0 ? pp : p0);
    return b[f * SgsTile<TJ>::PRN + o + dj * SgsTile<TJ>::PRK + dk];
  }
  __device__ __forceinline__ float r(int di, int dj, int dk) const { return at(0, di, dj, dk); }
  __device__ __forceinline__ float u(int di, int dj, int dk) const { return at(1, di, dj, dk); }
  __device__ __forceinline__ float v(int di, int dj, int dk) const { return at(2, di, dj, dk); }
  __device__ __forceinline__ float w(int di, int dj, int dk) const { return at(3, di, dj, dk); }
  __device__ __forceinline__ float th(int di, int dj, int dk) const { return at(4, di, dj, dk); }
  __device__ __forceinline__ float ev(int di, int dj, int dk) const { return at(5, di, dj, dk); }
  __device__ __forceinline__ float qm(int m, int di, int dj, int dk) const { return at(6 + m, di, dj, dk); }
};

// Primitive plane i of the tile, in two halves so the global loads of one plane are in flight
// while the block computes on the others: sgs_fetch_plane() loads the raw state of this thread's
// cells into registers, sgs_put_plane() forms the primitives (the per-point kernels' expressions:
// rho and phi * rinv(rho)) into shared memory. Cells outside the array read as 0.
template <int TJ>
struct PlaneRegs {
  static constexpr int PER = (SgsTile<TJ>::PRN + SgsTile<TJ>::NT - 1) / SgsTile<TJ>::NT;  // cells per thread
  float v[PER][SgsTile<TJ>::NPF];
};

template <int TJ>
__device__ __forceinline__ void sgs_fetch_plane(const Phys& P, const float* __restrict__ st, int i, int j0, int k0,
                                                int tid, PlaneRegs<TJ>& r) {
  using T = SgsTile<TJ>;
  const long long n = P.n;
#pragma unroll
  for (int e = 0; e < PlaneRegs<TJ>::PER; e++) {
    const int q = tid + e * T::NT;
    const int row = q / T::PRK, col = q - row * T::PRK;
    const int j = j0 - 2 + row, k = k0 - 3 + col;
#pragma unroll
    for (int f = 0; f < T::NPF; f++) r.v[e][f] = 0.0f;
    if (q < T::PRN && i < P.nxh && j < P.nyh && k < P.nzh) {
      const long long c = (long long)i * P.si + (long long)j * P.sj + k;
      r.v[e][0] = st[c];
      r.v[e][1] = st[n + c];
      r.v[e][2] = st[2 * n + c];
      r.v[e][3] = st[3 * n + c];
      r.v[e][4] = st[4 * n + c];
      if (P.ntke) r.v[e][5] = st[5 * n + c];
      if (P.nmoist > 0) r.v[e][6] = st[(long long)(5 + P.ntke) * n + c];
      if (P.nmoist > 1) r.v[e][7] = st[(long long)(6 + P.ntke) * n + c];
    }
  }
}

template <int TJ>
__device__ __forceinline__ void sgs_put_plane(int tid, const PlaneRegs<TJ>& r, float* __restrict__ dst) {
  using T = SgsTile<TJ>;
#pragma unroll
  for (int e = 0; e < PlaneRegs<TJ>::PER; e++) {
    const int q = tid + e * T::NT;
    if (q < T::PRN) {
      const float rr = r.v[e][0];
      const float ri = rinv(rr);
      dst[q] = rr;
#pragma unroll
      for (int f = 1; f < T::NPF; f++) dst[f * T::PRN + q] = r.v[e][f] * ri;
    }
  }
}

template <int TJ>
__device__ __forceinline__ void sgs_load_plane(const Phys& P, const float* __restrict__ st, int i, int j0, int k0,
                                               int tid, float* __restrict__ dst) {
  PlaneRegs<TJ> r;
  sgs_fetch_plane<TJ>(P, st, i, j0, k0, tid, r);
  sgs_put_plane<TJ>(tid, r, dst);
}

// The metric terms and grid scale of plane i for rows j0-1..j0+TJ, levels k0-2..k0+32 (the points
// the length scales and the physics of the plane read), fetched into registers ahead of use and
// then put into a shared-memory table [4][LSN].
template <int TJ>
struct MetricRegs {
  static constexpr int PER = (SgsTile<TJ>::LSN + SgsTile<TJ>::NT - 1) / SgsTile<TJ>::NT;
  PointMetrics m[PER];
};
template <int TJ>
__device__ __forceinline__ void sgs_fetch_metrics(const Phys& P, const Ptrs& Q, int i, int j0, int k0, int tid,
                                                  MetricRegs<TJ>& r) {
  using T = SgsTile<TJ>;
#pragma unroll
  for (int e = 0; e < MetricRegs<TJ>::PER; e++) {
    const int q = tid + e * T::NT;
    const int row = q / T::LSK, lv = q - row * T::LSK;
    const int j = j0 - 1 + row, k = k0 - 2 + lv;
    r.m[e] = PointMetrics{0.0f, 0.0f, 0.0f, 0.0f};
    if (q < T::LSN && i < P.nxh && j < P.nyh && k < P.nzh)
      r.m[e] = point_metrics(P, Q, (long long)i * P.si + (long long)j * P.sj + k);
  }
}
template <int TJ>
__device__ __forceinline__ void sgs_put_metrics(int tid, const MetricRegs<TJ>& r, float* __restrict__ dst) {
  using T = SgsTile<TJ>;
#pragma unroll
  for (int e = 0; e < MetricRegs<TJ>::PER; e++) {
    const int q = tid + e * T::NT;
    if (q < T::LSN) {
      dst[q] = r.m[e].J1;
      dst[T::LSN + q] = r.m[e].J2;
      dst[2 * T::LSN + q] = r.m[e].J3;
      dst[3 * T::LSN + q] = r.m[e].delta;
    }
  }
}
template <int TJ>
__device__ __forceinline__ PointMetrics sgs_metrics_at(const float* mt, int q) {
  constexpr int L = SgsTile<TJ>::LSN;
  return PointMetrics{mt[q], mt[L + q], mt[2 * L + q], mt[3 * L + q]};
}

// Length scale and sqrt(e/rho) of plane i (prims planes pm, p0, pp) for rows j0-1..j0+TJ and
// levels k0-2..k0+32 (0 outside the ring [iMin-1, iMax] x [jMin-1, jMax] x [1, kMax]).
template <int TJ>
__device__ __forceinline__ void sgs_length_scales(const Phys& P, const Ptrs& Q, int i, int j0, int k0, int tid,
                                                  const float* pm, const float* p0, const float* pp, float* lsT,
                                                  float* seT, const float* mt) {
  using T = SgsTile<TJ>;
  for (int q = tid; q < T::LSN; q += T::NT) {
    const int row = q / T::LSK, lv = q - row * T::LSK;
    const int j = j0 - 1 + row, k = k0 - 2 + lv;
    float ls = 0.0f, se = 0.0f;
    if (i >= P.iMin - 1 && i <= P.iMax && j >= P.jMin - 1 && j <= P.jMax && k >= 1 && k <= P.kMax) {
      const long long c = (long long)i * P.si + (long long)j * P.sj + k;
      const RingPrims<TJ> pr{pm, p0, pp, (row + 1) * T::PRK + (lv + 1)};
      (void)c;
      ls = length_scale_m(P, pr, 0, sgs_metrics_at<TJ>(mt, q));
      se = sqrtf(pr.ev(0, 0, 0));
    }
    lsT[q] = ls;
    seT[q] = se;
  }
}

// The closure's outputs of plane i for rows j0-1..j0+TJ, levels k0-1..k0+32 into `ph` [NPH][PHN]
// (zero outside the ring and below kMin); the first-level stresses of the surface columns from
// the surface-layer kernel's output; with `learned`, all 9 stresses from Q.tau (the network's,
// the surface columns' first-level ones left there by the surface layer). With `store`, the
// per-point kernels' scratch fields too.
template <int TJ>
__device__ __forceinline__ void sgs_physics_plane(const Phys& P, const Ptrs& Q, int i, int j0, int k0, int tid,
                                                  const float* pm, const float* p0, const float* pp,
                                                  const float* lsT, const float* seT, const float* mt, float* ph,
                                                  bool store, bool learned) {
  using T = SgsTile<TJ>;
  const long long n = P.n;
  for (int q = tid; q < T::PHN; q += T::NT) {
    const int row = q / T::PHK, col = q - row * T::PHK;
    const int j = j0 - 1 + row, k = k0 - 1 + col;
    TurbOut o;
    bool on = i >= P.iMin - 1 && i <= P.iMax && j >= P.jMin - 1 && j <= P.jMax && k >= P.kMin && k <= P.kMax;
    const long long c = (long long)i * P.si + (long long)j * P.sj + k;
    if (on) {
      const RingPrims<TJ> pr{pm, p0, pp, (row + 1) * T::PRK + (col + 2)};
      const int l = row * T::LSK + (col + 1);  // this level in the length-scale table; l - 1 below
      const bool tke = P.tke != 0;
      turb_point_m(P, pr, k, tke ? lsT[l] : 0.0f, tke ? lsT[l - 1] : 0.0f, tke ? seT[l - 1] : 0.0f,
                   tke ? seT[l] : -1.0f, sgs_metrics_at<TJ>(mt, l), o);
      const bool surfCell = P.surf > 0 && k == P.kMin && i >= P.iMin && j >= P.jMin;
      if (learned) {
#pragma unroll
        for (int t = 0; t < 9; t++) o.tau[t] = Q.tau[t * n + c];
      } else if (surfCell) {
        o.tau[2] = Q.tau[2 * n + c];
        o.tau[3] = Q.tau[3 * n + c];
        o.tau[8] = Q.tau[8 * n + c];
      }
      if (surfCell && P.moist && P.moistSGS > 0) o.mtau[2] = Q.mtau[2 * n + c];
      if (store) {
        float* Tt = Q.tau;
#pragma unroll
        for (int t = 0; t < 9; t++)
          if (!learned && !(surfCell && (t == 2 || t == 3 || t == 8))) Tt[t * n + c] = o.tau[t];
        if (P.tke) {
          Q.ls[c] = o.ls;
#pragma unroll
          for (int t = 0; t < 3; t++) Q.tkeQ[t * n + c] = o.tkeQ[t];
        }
        if (P.moist && P.moistSGS > 0)
          for (int m = 0; m < P.nmoist && m < 2; m++)
#pragma unroll
            for (int t = 0; t < 3; t++)
              if (!(surfCell && m == 0 && t == 2)) Q.mtau[(3 * m + t) * n + c] = o.mtau[3 * m + t];
      }
    } else {
#pragma unroll
      for (int t = 0; t < 9; t++) o.tau[t] = 0.0f;
#pragma unroll
      for (int t = 0; t < 3; t++) o.tkeQ[t] = 0.0f;
#pragma unroll
      for (int t = 0; t < 6; t++) o.mtau[t] = 0.0f;
      o.ls = 0.0f;
    }
#pragma unroll
    for (int t = 0; t < 9; t++) ph[t * T::PHN + q] = o.tau[t];
#pragma unroll
    for (int t = 0; t < 3; t++) ph[(9 + t) * T::PHN + q] = o.tkeQ[t];
#pragma unroll
    for (int t = 0; t < 6; t++) ph[(12 + t) * T::PHN + q] = o.mtau[t];
    ph[18 * T::PHN + q] = o.ls;
  }
}

// SGS tendencies of the last stage into the seven fields of Q.sgsF (fe_march.cuh k_sgs_tend's
// arithmetic, term by term), on the large-scale forcing steps with the forcing folded in.
// The body of one thread block: tile (bx, by, bz) of the domain P / Q.
template <bool TKE, int NQ, int TJ>
__device__ __forceinline__ void sgs_march_body(const Phys& P, const Ptrs& Q, const float* __restrict__ st, int stage,
                                               int ni, int store, int learned, int bx, int by, int bz) {
  using T = SgsTile<TJ>;
  extern __shared__ __align__(16) float sm[];
  float* const prim = sm;                          // [3][NPF][PRN]
  float* const phys = prim + 3 * T::NPF * T::PRN;  // [2][NPH][PHN]
  float* const lsT = phys + 2 * T::NPH * T::PHN;   // [PHJ][LSK]
  float* const seT = lsT + T::LSN;
  float* const mtT = seT + T::LSN;                 // [4][PHJ][LSK] metrics of the physics plane
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SG_K + tx;
  const int k0 = P.kMin + bx * SG_K, j0 = P.jMin + by * TJ;
  const int i0 = P.iMin + bz * ni;
  const int i1 = min(i0 + ni, P.iMax);
  const int j = j0 + ty, k = k0 + tx;
  const bool active = j < P.jMax && k < P.kMax;
  const long long n = P.n;
  const float dXi = P.dXi, dYi = P.dYi, dZi = P.dZi;
  const int ownP = (ty + 2) * T::PRK + (tx + 3);  // own cell in a primitive plane
  const int ownH = (ty + 1) * T::PHK + (tx + 1);  // own cell in a physics plane
  auto plane = [&](int ii) -> float* { return prim + ((ii - i0 + 3) % 3) * (T::NPF * T::PRN); };

  // ---------------------------------------------------------------- prologue
  // plane i0-1: this thread's own point only (its x and z TKE fluxes and u, v, w)
  sgs_load_plane<TJ>(P, st, i0 - 2, j0, k0, tid, plane(i0 - 2));
  sgs_load_plane<TJ>(P, st, i0 - 1, j0, k0, tid, plane(i0 - 1));
  sgs_load_plane<TJ>(P, st, i0, j0, k0, tid, plane(i0));
  __syncthreads();
  float qxm = 0.0f, qzm = 0.0f, um = 0.0f, vm = 0.0f, wm = 0.0f;
  {
    const RingPrims<TJ> pr{plane(i0 - 2), plane(i0 - 1), plane(i0), ownP};
    const RingPrims<TJ> prd{plane(i0 - 2), plane(i0 - 1), plane(i0), ownP - 1};  // the level below
    const int im = i0 - 1;
    if (TKE && active) {
      const long long c = (long long)im * P.si + (long long)j * P.sj + k;
      const float lsc = length_scale_a(P, Q, pr, c, 0);
      const float lsm = length_scale_a(P, Q, prd, c - 1, 0);
      const float sem = sqrtf(prd.ev(0, 0, 0));
      TurbOut o;
      turb_point(P, Q, pr, c, k, lsc, lsm, sem, -1.0f, o);
      qxm = o.tkeQ[0];
      qzm = o.tkeQ[2];
    }
  }
  __syncthreads();  // plane i0-2 is about to be replaced
  sgs_load_plane<TJ>(P, st, i0 + 1, j0, k0, tid, plane(i0 + 1));
  {
    MetricRegs<TJ> m0;
    sgs_fetch_metrics<TJ>(P, Q, i0, j0, k0, tid, m0);
    sgs_put_metrics<TJ>(tid, m0, mtT);
  }
  __syncthreads();
  sgs_length_scales<TJ>(P, Q, i0, j0, k0, tid, plane(i0 - 1), plane(i0), plane(i0 + 1), lsT, seT, mtT);
  __syncthreads();
  float* cur = phys;
  float* nxt = phys + T::NPH * T::PHN;
  PlaneRegs<TJ> ahead;     // the raw state of the plane after next, in flight during the computation
  MetricRegs<TJ> mahead;   // the metrics of the next physics plane, likewise
  sgs_fetch_plane<TJ>(P, st, i0 + 2, j0, k0, tid, ahead);
  sgs_fetch_metrics<TJ>(P, Q, i0 + 1, j0, k0, tid, mahead);
  sgs_physics_plane<TJ>(P, Q, i0, j0, k0, tid, plane(i0 - 1), plane(i0), plane(i0 + 1), lsT, seT, mtT, cur,
                        store != 0, learned != 0);

  // ---------------------------------------------------------------- march
  for (int i = i0; i < i1; i++) {
    // u, v, w of plane i-1 at this thread's cell, then plane i+2 (fetched during the previous
    // step) into its buffer and the fetch of plane i+3 started
    {
      const float* pl = plane(i - 1);
      um = pl[1 * T::PRN + ownP];
      vm = pl[2 * T::PRN + ownP];
      wm = pl[3 * T::PRN + ownP];
    }
    __syncthreads();
    sgs_put_plane<TJ>(tid, ahead, plane(i + 2));
    sgs_put_metrics<TJ>(tid, mahead, mtT);
    if (i + 1 < i1) {
      sgs_fetch_plane<TJ>(P, st, i + 3, j0, k0, tid, ahead);
      sgs_fetch_metrics<TJ>(P, Q, i + 2, j0, k0, tid, mahead);
    }
    __syncthreads();
    sgs_length_scales<TJ>(P, Q, i + 1, j0, k0, tid, plane(i), plane(i + 1), plane(i + 2), lsT, seT, mtT);
    __syncthreads();
    sgs_physics_plane<TJ>(P, Q, i + 1, j0, k0, tid, plane(i), plane(i + 1), plane(i + 2), lsT, seT, mtT, nxt,
                          store != 0, learned != 0);
    __syncthreads();

    if (active) {
      const long long c = (long long)i * P.si + (long long)j * P.sj + k;
      const float J1 = Q.J31[c], J2 = Q.J32[c], J3 = Q.J33[c];
      // closure outputs: TC at the cell, TI / TJ_ / TK one cell forward in i / j / k
      auto TC = [&](int m) -> float { return cur[m * T::PHN + ownH]; };
      auto TI = [&](int m) -> float { return nxt[m * T::PHN + ownH]; };
      auto TJp = [&](int m) -> float { return cur[m * T::PHN + ownH + T::PHK]; };
      auto TKp = [&](int m) -> float { return cur[m * T::PHN + ownH + 1]; };
      const float s0 = dXi * (TI(0) - TC(0)) + dYi * (TJp(1) - TC(1)) + J1 * dXi * (TI(2) - TC(2)) +
                       J2 * dYi * (TJp(2) - TC(2)) + J3 * dZi * (TKp(2) - TC(2));
      const float s1 = dXi * (TI(1) - TC(1)) + dYi * (TJp(4) - TC(4)) + J1 * dXi * (TI(3) - TC(3)) +
                       J2 * dYi * (TJp(3) - TC(3)) + J3 * dZi * (TKp(3) - TC(3));
      const float s2 = dXi * (TI(2) - TC(2)) + dYi * (TJp(3) - TC(3)) + J1 * dXi * (TI(5) - TC(5)) +
                       J2 * dYi * (TJp(5) - TC(5)) + J3 * dZi * (TKp(5) - TC(5));
      const float s3 = dXi * (TI(6) - TC(6)) + dYi * (TJp(7) - TC(7)) + J1 * dXi * (TI(8) - TC(8)) +
                       J2 * dYi * (TJp(8) - TC(8)) + J3 * dZi * (TKp(8) - TC(8));
      float sq[2] = {0.0f, 0.0f};
#pragma unroll
      for (int m = 0; m < NQ; m++) {
        const int b = 12 + 3 * m;
        sq[m] = dXi * (TI(b) - TC(b)) + dYi * (TJp(b + 1) - TC(b + 1)) + J1 * dXi * (TI(b + 2) - TC(b + 2)) +
                J2 * dYi * (TJp(b + 2) - TC(b + 2)) + J3 * dZi * (TKp(b + 2) - TC(b + 2));
      }
      float se = 0.0f;
      const float* p0 = plane(i);
      const float* pp = plane(i + 1);
      if (TKE) {
        const float r0 = p0[ownP];
        const float ri = rinv(r0);
        const float delta = grid_scale(P, Q, c);
        const float lsc = TC(18);
        const float mec = st[5 * n + c];
        float Se = P.g / p0[4 * T::PRN + ownP] * TC(8);
        const float ce = (float)(1.9 * (double)P.c_k + (0.93 - 1.9 * (double)P.c_k) * (double)lsc / (double)delta);
        const float ec = mec * ri;
        Se = Se + (-ce * mec * sqrtf(ec) / lsc);
        // (rho phi)/rho of field f at the neighbours: i+1 from the next primitive plane, i-1 carried
        auto G = [&](int f, int dj, int dk) -> float { return p0[f * T::PRN + ownP + dj * T::PRK + dk]; };
        const float ux = pp[1 * T::PRN + ownP] - um, uy = G(1, 1, 0) - G(1, -1, 0), uz = G(1, 0, 1) - G(1, 0, -1);
        const float vx = pp[2 * T::PRN + ownP] - vm, vy = G(2, 1, 0) - G(2, -1, 0), vz = G(2, 0, 1) - G(2, 0, -1);
        const float wx = pp[3 * T::PRN + ownP] - wm, wy = G(3, 1, 0) - G(3, -1, 0), wz = G(3, 0, 1) - G(3, 0, -1);
        const float dux = 0.5f * (dXi * ux), duy = 0.5f * (dYi * uy);
        const float duz = 0.5f * (J1 * dXi * ux + J2 * dYi * uy + J3 * dZi * uz);
        const float dvx = 0.5f * (dXi * vx), dvy = 0.5f * (dYi * vy);
        const float dvz = 0.5f * (J1 * dXi * vx + J2 * dYi * vy + J3 * dZi * vz);
        const float dwx = 0.5f * (dXi * wx), dwy = 0.5f * (dYi * wy);
        const float dwz = 0.5f * (J1 * dXi * wx + J2 * dYi * wy + J3 * dZi * wz);
        const float shear = (-TC(0) * dux) + (-TC(1) * duy) + (-TC(2) * duz) + (-TC(1) * dvx) + (-TC(4) * dvy) +
                            (-TC(3) * dvz) + (-TC(2) * dwx) + (-TC(3) * dwy) + (-TC(5) * dwz);
        Se = Se + shear;
        const float tx_ = -(dXi * (TI(9) - qxm));
        const float ty_ = -(dYi * (TJp(10) - cur[10 * T::PHN + ownH - T::PHK]));
        const float tz_ = -(J1 * dXi * (TI(11) - qzm) + J2 * dYi * (TJp(11) - cur[11 * T::PHN + ownH - T::PHK]) +
                            J3 * dZi * (TKp(11) - cur[11 * T::PHN + ownH - 1]));
        Se = Se + (-(tx_ + ty_ + tz_));
        se = Se;
      }
      // large-scale forcing of the last stage (cuda_hydroCoreDevice.cu:401-406)
      float lu = 0.0f, lv = 0.0f, lth = 0.0f, lqv = 0.0f;
      if (stage == 2 && lsf_step(P, *Q.clockIt)) lsf_tend(P, Q, c, k, Q.zPos[c], p0[ownP], lu, lv, lth, lqv);
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
    // plane i becomes plane i-1: its x and z TKE fluxes at this cell are carried
    qxm = cur[9 * T::PHN + ownH];
    qzm = cur[11 * T::PHN + ownH];
    float* const t = cur;
    cur = nxt;
    nxt = t;
  }
}

template <bool TKE, int NQ, int TJ>
__global__ void __launch_bounds__(SG_K * TJ, TJ <= 8 ? 2 : 1)
    k_sgs_march(Phys P, Ptrs Q, const float* __restrict__ st, int stage, int ni, int store, int learned) {
  sgs_march_body<TKE, NQ, TJ>(P, Q, st, stage, ni, store, learned, blockIdx.x, blockIdx.y, blockIdx.z);
}

// One member of a batched launch of the fused SGS kernel (see MarchMember).
struct SgsMember {
  Phys P;
  Ptrs Q;
  const float* st;
  int ni, gx, gy, first;
};

// The fused SGS kernel of several domains in one launch: block b runs a tile of the member the
// block map names, with that member's parameters copied into shared memory.
template <bool TKE, int NQ, int TJ>
__global__ void __launch_bounds__(SG_K * TJ, TJ <= 8 ? 2 : 1)
    k_sgs_march_list(const SgsMember* __restrict__ mem, const int* __restrict__ bmap, int stage) {
  __shared__ SgsMember sm_m;
  __shared__ int sm_idx;
  const int tid = threadIdx.y * SG_K + threadIdx.x;
  if (tid == 0) sm_idx = bmap[blockIdx.x];
  __syncthreads();
  {
    const int* src = reinterpret_cast<const int*>(mem + sm_idx);
    int* dst = reinterpret_cast<int*>(&sm_m);
    for (int q = tid; q < (int)(sizeof(SgsMember) / sizeof(int)); q += SG_K * TJ) dst[q] = src[q];
  }
  __syncthreads();
  const SgsMember& m = sm_m;
  const int local = (int)blockIdx.x - m.first;
  sgs_march_body<TKE, NQ, TJ>(m.P, m.Q, m.st, stage, m.ni, 0, 0, local % m.gx, (local / m.gx) % m.gy,
                              local / (m.gx * m.gy));
}

}  // namespace fe
