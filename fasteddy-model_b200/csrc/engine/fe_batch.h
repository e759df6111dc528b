// fe_batch.h -- batched launches of several domains' kernels (the ensemble's work-list form).
//
// Each launch runs one kernel over the tiles of every member: the members' parameter blocks
// (MarchMember, SgsMember, SurfMember, ClockMember) sit in a device table, and a block map gives
// each thread block its member (one load at the block's start). The batched kernels cover the
// dry flavour (FL_DRY: prognostic TKE, HYB56, physics in the last stage) at 8 rows per tile with
// the fused SGS kernel; an ensemble outside it keeps one graph branch per member. (The moist
// flavour's batched stage kernels spill 36-52 bytes per thread: their parameters come from shared
// memory instead of the constant bank, and that flavour has no registers to spare.)
#pragma once
#include <cuda_runtime.h>

#include "fe_kernels.cuh"
#include "fe_march.cuh"
#include "fe_sgs_march.cuh"

namespace fe {

// The stage kernel of RK stage `stage`.
cudaError_t batch_march(int flavour, int stage, const MarchMember* mem, const int* bmap, int blocks, cudaStream_t s);
// The fused SGS kernel (prognostic TKE, no moisture fluxes, 8 rows per tile), the surface layer and
// the device clocks.
cudaError_t batch_sgs(const SgsMember* mem, const int* bmap, int blocks, int stage, cudaStream_t s);
cudaError_t batch_surface(const SurfMember* mem, const int* bmap, int blocks, int stage, cudaStream_t s);
cudaError_t batch_clock(const ClockMember* mem, int nmem, cudaStream_t s);
// Dynamic shared-memory limits of the batched kernels; set on the current device before any launch.
cudaError_t batch_set_attrs();

}  // namespace fe
