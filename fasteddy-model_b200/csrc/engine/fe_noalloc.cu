// fe_noalloc.cu -- fe_frhs_noalloc(): the tendency evaluation without any device allocation.
//
// Who needs it: callers that cannot call cudaMalloc -- allocators that forbid side
// allocations (a caching pool owning all device memory), or embedders that must not
// change the device's memory footprint after start-up. They own their input and output buffers but cannot give this
// library scratch space.
//
// How: all intermediates (device-evaluated constants, base-state pressure term,
// perturbation pressure, the last-stage SGS stresses, TKE fluxes, length scale, moisture
// fluxes, the step clock) live in one file-scope __device__ array of FE_NOALLOC_SCRATCH_BYTES,
// allocated once per GPU when the library is loaded and kept until exit. Its device
// address is fetched with cudaGetSymbolAddress on every call, on the caller's current device
// (the name of a __device__ array in host code is only a host-side stand-in, never a device
// address).
//
// The kernels are the engine's own (fe_kernels.cuh), compiled into a private namespace of
// this translation unit so they do not collide with the engine's copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "fasteddy_b200.h"

namespace fe_noalloc_impl {
#include "fe_kernels.cuh"
#include "fe_config_phys.cuh"
}  // namespace fe_noalloc_impl

using fe_noalloc_impl::fe::Phys;
using fe_noalloc_impl::fe::Ptrs;
namespace K = fe_noalloc_impl::fe;

// Scratch layout (floats): [0,64) clock and constants, then 21 fields of n cells:
// pBS, p', 9 stresses, 3 TKE fluxes, length scale, 6 moisture fluxes.
static constexpr int kHeaderFloats = 64;
static constexpr int kScratchFields = 21;
static constexpr size_t kScratchFloats = FE_NOALLOC_SCRATCH_BYTES / sizeof(float);

static __device__ __align__(256) float g_noalloc_scratch[kScratchFloats];

namespace {
thread_local std::string g_na_err;

int na_err(int code, const std::string& m) {
  g_na_err = m;
  return code;
}

__global__ void k_na_clock(int* it, float* t, int simIt, float simTime) {
  *it = simIt;
  *t = simTime;
}

// The engine's own validation (the checks fe_create applies), then this path's narrower set:
// the per-cell stage kernel here has no explicit filter and no large-scale forcing, and its
// advection is HYB56 (3) or WENO5 (5) for the hydro fields, TKE and q_v, WENO5 for q_l.
int check(const fe_config& c) {
  int rc = fe_check_config(&c);
  if (rc) return na_err(rc, fe_last_error());
  if (c.advectionSelector != 3 && c.advectionSelector != 5)
    return na_err(FE_ERR_CONFIG, "advectionSelector must be 3 or 5");
  if (c.turbulenceSelector > 0 && c.TKESelector > 0 && c.TKEAdvSelector != 3 && c.TKEAdvSelector != 5)
    return na_err(FE_ERR_CONFIG, "TKEAdvSelector must be 3 or 5");
  if (c.filterSelector || c.lsfSelector)
    return na_err(FE_ERR_CONFIG, "the explicit filter and large-scale forcing are not on this path");
  if (c.moistureSelector > 0 && ((c.moistureAdvSelectorQv != 3 && c.moistureAdvSelectorQv != 5) ||
                                 (c.moistureNvars > 1 && c.moistureAdvSelectorQi != 2)))
    return na_err(FE_ERR_CONFIG, "unsupported moisture selectors");
  return FE_OK;
}

// The device address of the scratch array on the current device, looked up on every call: a
// cached address would outlive a cudaDeviceReset or a re-created primary context (the module is
// loaded again there), and a per-call lookup is cheap next to the synchronising call it serves.
int scratch_address(float** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return na_err(FE_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  }
  *out = (float*)p;
  return FE_OK;
}
}  // namespace

extern "C" long long fe_noalloc_max_cells(void) {
  return (long long)((kScratchFloats - kHeaderFloats) / kScratchFields);
}

extern "C" const char* fe_noalloc_last_error(void) { return g_na_err.c_str(); }

extern "C" int fe_frhs_noalloc(const fe_config* cfg, int stage, float simTime, int simTime_it,
                               const fe_noalloc_args* a, void* stream) {
  if (!cfg || !a || stage < 0 || stage > 2) return na_err(FE_ERR_ARG, "NULL argument or stage outside 0..2");
  if (!a->zPos || !a->J31 || !a->J32 || !a->J33 || !a->D_Jac || !a->invD_Jac || !a->baseState || !a->state ||
      !a->frhs || (cfg->surflayerSelector > 0 && !a->surface))
    return na_err(FE_ERR_ARG, "NULL device pointer");
  int rc = check(*cfg);
  if (rc) return rc;
  Phys P;
  K::phys_from_config(*cfg, P);
  if (P.n > fe_noalloc_max_cells())
    return na_err(FE_ERR_ARG, "domain of " + std::to_string(P.n) + " halo-inclusive cells exceeds the " +
                                  std::to_string(fe_noalloc_max_cells()) + "-cell scratch of fe_frhs_noalloc");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return na_err(FE_ERR_NO_DEVICE, "no current CUDA device");
  }
  float* S = nullptr;
  rc = scratch_address(&S);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  const size_t n = (size_t)P.n, n2 = (size_t)P.n2;
  float* fields = S + kHeaderFloats;
  Ptrs Q;
  std::memset(&Q, 0, sizeof(Q));
  Q.zPos = a->zPos; Q.J31 = a->J31; Q.J32 = a->J32; Q.J33 = a->J33; Q.D = a->D_Jac; Q.invD = a->invD_Jac;
  Q.rhoBS = a->baseState;
  Q.thBS = a->baseState + n;
  float* pBS = fields;
  float* pres = fields + n;
  Q.pBS = pBS;
  Q.tau = fields + 2 * n;
  Q.tkeQ = fields + 11 * n;
  Q.ls = fields + 14 * n;
  Q.mtau = fields + 15 * n;
  if (a->surface) {
    float* sf = a->surface;
    Q.cd = sf; Q.ch = sf + n2; Q.cq = sf + 2 * n2; Q.fricVel = sf + 3 * n2; Q.htFlux = sf + 4 * n2;
    Q.tskin = sf + 5 * n2; Q.invOblen = sf + 6 * n2; Q.z0m = sf + 7 * n2; Q.z0t = sf + 8 * n2;
    Q.qFlux = sf + 9 * n2; Q.qskin = sf + 10 * n2;
  }
  Q.clockIt = (int*)S;
  Q.clockTime = S + 1;
  // device-evaluated constants into the header, read back (a copy, not an allocation)
  K::k_consts<<<1, 1, 0, s>>>(P.R_gas, P.p0, P.R_cp, P.presGrnd, S + 8);
  float hc[2] = {0.0f, 0.0f};
  cudaError_t e = cudaMemcpyAsync(hc, S + 8, sizeof(hc), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return na_err(FE_ERR_CUDA, std::string("constant setup: ") + cudaGetErrorString(e));
  P.c1 = hc[0];
  P.presFac = hc[1];
  // every scratch value the kernels read below is written earlier in this call
  k_na_clock<<<1, 1, 0, s>>>(Q.clockIt, Q.clockTime, simTime_it, simTime);
  const unsigned nb = (unsigned)((n + 255) / 256);
  K::k_pbs<<<nb, 256, 0, s>>>((long long)n, Q.thBS, P.c1, P.cp_cv, pBS);
  K::k_pressure<<<nb, 256, 0, s>>>(P, Q, a->state, pres);
  const dim3 blk(32, 4, 2);
  const bool phys = (P.oneRK == 0) || (stage == 2);
  if (phys && (P.turb || P.surf > 0)) {
    const dim3 gt((P.Nz + 2 + 31) / 32, (P.Ny + 2 + 3) / 4, (P.Nx + 2 + 1) / 2);
    K::k_turb<<<gt, blk, 0, s>>>(P, Q, a->state, stage);
  }
  const dim3 g((P.Nz + 31) / 32, (P.Ny + 3) / 4, (P.Nx + 1) / 2);
  switch (stage) {
    case 0: K::k_stage<0, K::MODE_FRHS><<<g, blk, 0, s>>>(P, Q, a->state, a->state, nullptr, pres, nullptr, a->frhs); break;
    case 1: K::k_stage<1, K::MODE_FRHS><<<g, blk, 0, s>>>(P, Q, a->state, a->state, nullptr, pres, nullptr, a->frhs); break;
    default: K::k_stage<2, K::MODE_FRHS><<<g, blk, 0, s>>>(P, Q, a->state, a->state, nullptr, pres, nullptr, a->frhs); break;
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return na_err(FE_ERR_CUDA, std::string("fe_frhs_noalloc: ") + cudaGetErrorString(e));
  return FE_OK;
}
