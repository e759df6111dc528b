// fe_march_impl.cuh -- definitions behind fe_march_launch.cuh, included by the per-stage
// translation units fe_march_s0.cu, fe_march_s1.cu and fe_march_s2.cu.
#pragma once
#include "fe_march.cuh"
#include "fe_march_launch.cuh"

namespace fe {

template <int STAGE, int MODE, int TJ, int FL, int MP = -1>
static void march_launch_one(const Phys& P, const Ptrs& Q, int ni, cudaStream_t s, const float* cur, const float* base,
                             float* nxt, const float* pcur, float* pnxt, float* frhs) {
  const dim3 g((P.Nz + MK - 1) / MK, (P.Ny + TJ - 1) / TJ, (P.Nx + ni - 1) / ni);
  k_march<STAGE, MODE, TJ, FL, MP><<<g, dim3(MK, TJ), MarchTile<TJ>::SMEM_BYTES, s>>>(P, Q, cur, base, nxt, pcur, pnxt,
                                                                                   frhs, ni);
}

// A moist flavour's stage kernel: the last committing stage as its pair (MP = 0, then MP = 1).
template <int STAGE, int MODE, int FL>
static void march_launch_moist(const Phys& P, const Ptrs& Q, int ni, cudaStream_t s, const float* cur, const float* base,
                               float* nxt, const float* pcur, float* pnxt, float* frhs) {
  if constexpr (STAGE == 2 && MODE == MODE_COMMIT) {
    march_launch_one<STAGE, MODE, 8, FL, 0>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs);
    march_launch_one<STAGE, MODE, 8, FL, 1>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs);
  } else {
    march_launch_one<STAGE, MODE, 8, FL>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs);
  }
}

template <int STAGE, int MODE>
void march_launch(const Phys& P, const Ptrs& Q, int tj, int ni, cudaStream_t s, const float* cur, const float* base,
                  float* nxt, const float* pcur, float* pnxt, float* frhs) {
  if (tj == 4) {
    march_launch_one<STAGE, MODE, 4, FL_ANY>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs);
    return;
  }
  switch (march_flavor(P)) {
    case FL_DRY: march_launch_one<STAGE, MODE, 8, FL_DRY>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs); break;
    case FL_MOIST: march_launch_moist<STAGE, MODE, FL_MOIST>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs); break;
    case FL_MOIST34: march_launch_moist<STAGE, MODE, FL_MOIST34>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs); break;
    default: march_launch_one<STAGE, MODE, 8, FL_ANY>(P, Q, ni, s, cur, base, nxt, pcur, pnxt, frhs); break;
  }
}

template <int STAGE, int MODE>
cudaError_t march_set_attrs() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, int bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  set((const void*)k_march<STAGE, MODE, 8, FL_ANY>, MarchTile<8>::SMEM_BYTES);
  set((const void*)k_march<STAGE, MODE, 8, FL_DRY>, MarchTile<8>::SMEM_BYTES);
  set((const void*)k_march<STAGE, MODE, 8, FL_MOIST>, MarchTile<8>::SMEM_BYTES);
  set((const void*)k_march<STAGE, MODE, 8, FL_MOIST34>, MarchTile<8>::SMEM_BYTES);
  if constexpr (STAGE == 2 && MODE == MODE_COMMIT) {
    set((const void*)k_march<STAGE, MODE, 8, FL_MOIST, 0>, MarchTile<8>::SMEM_BYTES);
    set((const void*)k_march<STAGE, MODE, 8, FL_MOIST, 1>, MarchTile<8>::SMEM_BYTES);
    set((const void*)k_march<STAGE, MODE, 8, FL_MOIST34, 0>, MarchTile<8>::SMEM_BYTES);
    set((const void*)k_march<STAGE, MODE, 8, FL_MOIST34, 1>, MarchTile<8>::SMEM_BYTES);
  }
  set((const void*)k_march<STAGE, MODE, 4, FL_ANY>, MarchTile<4>::SMEM_BYTES);
  return e;
}

}  // namespace fe

// Explicit instantiations of one RK stage (both modes) in the including translation unit.
#define FE_MARCH_INSTANTIATE(STAGE)                                                                                     \
  template void fe::march_launch<STAGE, fe::MODE_COMMIT>(const fe::Phys&, const fe::Ptrs&, int, int, cudaStream_t,    \
                                                         const float*, const float*, float*, const float*, float*,   \
                                                         float*);                                                      \
  template void fe::march_launch<STAGE, fe::MODE_FRHS>(const fe::Phys&, const fe::Ptrs&, int, int, cudaStream_t,      \
                                                       const float*, const float*, float*, const float*, float*,     \
                                                       float*);                                                        \
  template cudaError_t fe::march_set_attrs<STAGE, fe::MODE_COMMIT>();                                                  \
  template cudaError_t fe::march_set_attrs<STAGE, fe::MODE_FRHS>();
