// fe_march_launch.cuh -- host entry points of the i-marching stage kernel (fe_march.cuh).
//
// The kernel's instantiations (3 RK stages x commit/tendency modes x compile-time flavours)
// are compiled in three translation units, one per RK stage (fe_march_s0.cu, fe_march_s1.cu,
// fe_march_s2.cu), so they build in parallel; the engine calls them through these functions.
#pragma once
#include <cuda_runtime.h>

#include "fe_device.cuh"

namespace fe {

// Compile-time configurations ("flavours") of the march kernel. FL_ANY reads every selector at
// run time; the others fix the field set and the advection schemes of the common cases (PGF on,
// prognostic TKE, HYB56 for the hydro fields and TKE, HYB56 or HYB34 for q_v, WENO5 for q_l, SGS
// physics in the last RK stage only), so the field loop has no run-time branches and the first
// two stages carry no physics code.
constexpr int FL_ANY = 0;
constexpr int FL_DRY = 1;      // rho, rho u, rho v, rho w, rho theta, rho e
constexpr int FL_MOIST = 2;    // ... plus rho q_v and rho q_l
constexpr int FL_MOIST34 = 3;  // the moist set with HYB34 for q_v (the BOMEX tutorial's selectors)

// The flavour that matches the configuration.
inline int march_flavor(const Phys& P) {
  if (P.pgf && P.tke && P.ntke == 1 && P.advSel == 3 && P.tkeAdvSel == 3 && P.oneRK == 1) {
    if (P.nmoist == 0) return FL_DRY;
    if (P.nmoist == 2 && P.qlSch == ADV_WENO5) {
      if (P.qvAdvSel == 3) return FL_MOIST;
      if (P.qvAdvSel == 2) return FL_MOIST34;
    }
  }
  return FL_ANY;
}

// Whether the last committing stage runs as a pair of kernels (the moist flavours at 8 rows: the
// kernel of the steps without saturation adjustment carries none of its code).
inline bool march_split_last_stage(const Phys& P, int tj) {
  const int fl = march_flavor(P);
  return tj == 8 && (fl == FL_MOIST || fl == FL_MOIST34);
}

// Launch the stage kernel of RK stage STAGE in mode MODE (commit or tendency only) with tiles of
// tj rows (4 or 8) marching ni planes per thread block.
template <int STAGE, int MODE>
void march_launch(const Phys& P, const Ptrs& Q, int tj, int ni, cudaStream_t s, const float* cur, const float* base,
                  float* nxt, const float* pcur, float* pnxt, float* frhs);

// Dynamic shared-memory limits of every instantiation of the stage; set on the current device
// before any launch or capture.
template <int STAGE, int MODE>
cudaError_t march_set_attrs();

}  // namespace fe
