// fe_batch.cu -- the batched (work-list) launches of fe_batch.h.
#include "fe_batch.h"

namespace fe {

namespace {
template <int STAGE, int FL, int MP>
cudaError_t march_list(const MarchMember* mem, const int* bmap, int blocks, cudaStream_t s) {
  k_march_list<STAGE, 8, FL, MP><<<blocks, dim3(MK, 8), MarchTile<8>::SMEM_BYTES, s>>>(mem, bmap);
  return cudaGetLastError();
}
template <int FL>
cudaError_t march_flavour(int stage, const MarchMember* mem, const int* bmap, int blocks, cudaStream_t s) {
  if (stage == 0) return march_list<0, FL, -1>(mem, bmap, blocks, s);
  if (stage == 1) return march_list<1, FL, -1>(mem, bmap, blocks, s);
  return march_list<2, FL, -1>(mem, bmap, blocks, s);
}
template <bool TKE, int NQ>
cudaError_t sgs_list(const SgsMember* mem, const int* bmap, int blocks, int stage, cudaStream_t s) {
  k_sgs_march_list<TKE, NQ, 8><<<blocks, dim3(SG_K, 8), SgsTile<8>::SMEM_BYTES, s>>>(mem, bmap, stage);
  return cudaGetLastError();
}
}  // namespace

cudaError_t batch_march(int flavour, int stage, const MarchMember* mem, const int* bmap, int blocks, cudaStream_t s) {
  if (flavour == FL_DRY) return march_flavour<FL_DRY>(stage, mem, bmap, blocks, s);
  return cudaErrorInvalidValue;
}

cudaError_t batch_sgs(const SgsMember* mem, const int* bmap, int blocks, int stage, cudaStream_t s) {
  return sgs_list<true, 0>(mem, bmap, blocks, stage, s);
}

cudaError_t batch_surface(const SurfMember* mem, const int* bmap, int blocks, int stage, cudaStream_t s) {
  k_surface_list<<<blocks, 128, 0, s>>>(mem, bmap, stage);
  return cudaGetLastError();
}

cudaError_t batch_clock(const ClockMember* mem, int nmem, cudaStream_t s) {
  k_clock_list<<<(nmem + 127) / 128, 128, 0, s>>>(mem, nmem);
  return cudaGetLastError();
}

cudaError_t batch_set_attrs() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, int bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  const int bm = MarchTile<8>::SMEM_BYTES, bs = SgsTile<8>::SMEM_BYTES;
  set((const void*)k_march_list<0, 8, FL_DRY, -1>, bm);
  set((const void*)k_march_list<1, 8, FL_DRY, -1>, bm);
  set((const void*)k_march_list<2, 8, FL_DRY, -1>, bm);
  set((const void*)k_sgs_march_list<true, 0, 8>, bs);
  return e;
}

}  // namespace fe
