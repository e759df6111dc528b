// fe_engine.cu -- host side of the B200 engine: domains, device memory, stage sequencing,
// CUDA-graph replay of RK3 steps, ensembles and the autotuner. C ABI in fasteddy_b200.h.
//
// Memory plan of one domain (all fields halo-inclusive, reference layout):
//   state A, B, C      nf fields each: A = phi^n (and phi^{n+1}), B = phi*, C = phi**
//   pres pA, pB, pC    perturbation pressure of A, B, C
//                      (A, B, C, pA, pB, pC are one allocation, the state arena, so that one
//                      offset per neighbour reaches the same buffer of a neighbouring slab)
//   grid               zPos, J31, J32, J33, D_Jac, invD_Jac
//   base               rho_BS, (rho theta)_BS, powf((rho theta)_BS c1, cp/cv)
//   scratch            9 stresses, 3 TKE fluxes, length scale, 3 per moisture species
//   surface (2-D)      cd, ch, cq, u*, w'th', T_skin, 1/L, z0m, z0t, w'q', q_skin
//   clock              simTime_it, simTime of the step in flight
// A stage reads its input state at the stencil neighbours and the step-start state A at
// its own cell only, so stage 3 can write phi^{n+1} into A in place. The commit of every
// stage writes the next state's halo cells, so the next stage needs no halo pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fasteddy_b200.h"
#include "fe_kernels.cuh"
#include "fe_march.cuh"
#include "fe_march_launch.cuh"
#include "fe_sgs_march.cuh"
#include "fe_learn.h"
#include "fe_sgs.cuh"
#include "fe_config_phys.cuh"
#include "fe_comm.h"
#include "fe_batch.h"

using fe::Phys;
using fe::Ptrs;

namespace {
thread_local std::string g_err;

int set_err(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CU(call)                                                                                   \
  do {                                                                                             \
    cudaError_t e__ = (call);                                                                      \
    if (e__ != cudaSuccess)                                                                        \
      return set_err(FE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__));           \
  } while (0)
}  // namespace

struct fe_domain {
  fe_config cfg;
  Phys P;
  Ptrs Q;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                         // second branch of a step (ring-level SGS kernel)
  cudaEvent_t fork = nullptr, join = nullptr;          // ordering between stream and side
  float* st[3] = {nullptr, nullptr, nullptr};
  float* pr[3] = {nullptr, nullptr, nullptr};
  float* arena = nullptr;                              // the allocation holding st[] and pr[]
  std::vector<void*> peerMaps;                         // neighbours' arenas opened by IPC handle
  fe_comm* comm = nullptr;                             // stage barrier of a multi-process decomposition
  float* grid = nullptr;
  float* base = nullptr;
  float* scratch = nullptr;
  float* surf = nullptr;
  float* frhs = nullptr;
  void* lsfMem = nullptr;                              // slab means and their per-block partial sums
  int lsfBlocks = 0;                                   // blocks of the slab-mean kernel
  void* clock = nullptr;
  unsigned long long* counter = nullptr;
  float simTime = 0.0f;
  int simIt = 0;
  bool haveGrid = false, haveBase = false, haveState = false;
  int tk = 32, tj = 4, ti = 2;       // cell-kernel tiling
  int kind = FE_KERNEL_MARCH;        // stage-kernel form
  int mtj = 8, mni = 64;             // march kernel: rows per tile, planes per thread block
  int sgsNi = 32;                    // fused SGS kernel: planes per thread block
  int sgsRows = 8;                   // fused last-stage physics: rows per tile (8 or 16; 0 = kernel chain)
  int mniDefault = 64;               // planes per block chosen for the domain size at creation
  fe_mlp* mlp = nullptr;             // learned SGS closure (nullptr: TKE closure)
  float* feat = nullptr;             // its inputs per ring cell (allocated with the first network)
  cudaGraphExec_t graph = nullptr;
  int graphSteps = 0;
  long long launches = 0;
  size_t bytes = 0;
  bool captureFrhs = false;          // keep the last-stage tendencies of the last step of an advance
};

struct fe_ensemble {
  std::vector<fe_domain*> m;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graphSteps = 0;
  bool coupled = false;  // slabs of one decomposed domain: every stage of all waits for the last
  // work-list form: one launch per kernel of a step over the tiles of every member
  bool wantBatched = true;
  bool batched = false;               // the graph and the eager steps use the work-list launches
  void* batchMem = nullptr;           // the member tables on the device
  fe::MarchMember* bMarch[3] = {nullptr, nullptr, nullptr};
  fe::SgsMember* bSgs[3] = {nullptr, nullptr, nullptr};
  fe::SurfMember* bSurf[3] = {nullptr, nullptr, nullptr};
  fe::ClockMember* bClock = nullptr;
  int *bMapMarch = nullptr, *bMapSgs = nullptr, *bMapSurf = nullptr;  // member of each thread block
  int bMarchBlocks = 0, bSgsBlocks = 0, bSurfBlocks = 0;
  long long launches = 0;             // the work-list launches (the members count their own otherwise)
};

extern "C" const char* fe_last_error(void) { return g_err.c_str(); }

int fe_internal_error(int code, const char* msg) { return set_err(code, msg ? msg : ""); }

extern "C" int fe_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" void fe_config_defaults(fe_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->Nh = 3;
  c->hydroBCs = 2;
  c->pgfSelector = 1;
  c->buoyancySelector = 1;
  c->coriolisSelector = 0;
  c->c_s = 0.18f;
  c->c_k = 0.10f;
  c->advectionSelector = 3;
  c->b_hyb = 0.0f;
  c->surflayer_z0 = 0.1f;
  c->surflayer_z0t = 0.1f;
  c->moistureCond = 1;
  c->moistureCondTscale = 1.0f;
  c->moistureMPcallTscale = 1.0f;
  c->dampingLayerDepth = 100.0f;
  c->z_Ug = 10000.0f;
  c->z_Vg = 10000.0f;
  c->physics_oneRKonly = 1;
  c->temp_grnd = 300.0f;
  c->pres_grnd = 1.0e5f;
  c->dt = 1.0f;
  c->dX = c->dY = c->dZ = 1.0f;
  c->surflayer_ideal_amp = 0.1f;
  c->surflayer_ideal_qamp = 0.1f;
  c->filter_6th_coeff = 0.12f;
  c->lsf_freq = 1.0f;
  c->lsf_w_zlev1 = c->lsf_th_zlev1 = c->lsf_qv_zlev1 = 100.0f;
  c->lsf_w_zlev2 = c->lsf_th_zlev2 = c->lsf_qv_zlev2 = 200.0f;
  fe_config_derive(c, 54.0f);
}

extern "C" void fe_config_derive(fe_config* c, float lat) {
  c->kappa = 0.4f;
  c->accel_g = 9.81f;
  c->R_gas = 287.04f;
  c->R_vapor = 461.60f;
  c->cv_gas = 718.0f;
  c->cp_gas = c->R_gas + c->cv_gas;
  c->L_v = 2.5e6f;
  c->R_cp = c->R_gas / c->cp_gas;
  c->cp_R = c->cp_gas / c->R_gas;
  c->cp_cv = c->cp_gas / c->cv_gas;
  c->refPressure = 1.0e5f;
  c->Rv_Rg = c->R_vapor / c->R_gas;
  const double pi = std::acos(-1.0);
  if (c->coriolisSelector > 0) {
    c->corioConstHorz = (float)(1.45842e-4 * std::sin(pi / 180.0 * lat));
    c->corioConstVert = c->coriolisSelector > 1 ? (float)(1.45842e-4 * std::cos(pi / 180.0 * lat)) : 0.0f;
    c->corioLS_fact = 1.0f;
  } else {
    c->corioConstHorz = c->corioConstVert = 0.0f;
  }
}

extern "C" int fe_check_config(const fe_config* c) {
  if (!c) return set_err(FE_ERR_ARG, "NULL configuration");
  if (c->Nh != 3) return set_err(FE_ERR_CONFIG, "Nh must be 3");
  if (c->Nx < 3 || c->Ny < 3 || c->Nz < 2) return set_err(FE_ERR_CONFIG, "need Nx,Ny >= 3 and Nz >= 2");
  if (c->hydroBCs != 2) return set_err(FE_ERR_CONFIG, "only hydroBCs = 2 (periodic horizontal, ABL vertical)");
  // selector ranges as the reference's parameter reader checks them (hydro_core.c:221-349)
  if (c->advectionSelector < 0 || c->advectionSelector > 6) return set_err(FE_ERR_CONFIG, "advectionSelector must be 0..6");
  if (!(c->b_hyb >= 0.0f && c->b_hyb <= 1.0f)) return set_err(FE_ERR_CONFIG, "b_hyb must be in [0, 1]");
  if (c->turbulenceSelector > 0 && c->TKESelector > 0) {
    if (c->TKEAdvSelector < 0 || c->TKEAdvSelector > 6) return set_err(FE_ERR_CONFIG, "TKEAdvSelector must be 0..6");
    if (!(c->TKEAdvSelector_b_hyb >= 0.0f && c->TKEAdvSelector_b_hyb <= 1.0f))
      return set_err(FE_ERR_CONFIG, "TKEAdvSelector_b_hyb must be in [0, 1]");
  }
  if (c->diffusionSelector != 0) return set_err(FE_ERR_CONFIG, "molecular diffusion is not on this path");
  if (c->lsfSelector < 0 || c->lsfSelector > 1) return set_err(FE_ERR_CONFIG, "lsfSelector must be 0 or 1");
  if (c->lsfSelector > 0) {
    if (!(c->lsf_freq >= 1e-3f && c->lsf_freq <= 1e3f)) return set_err(FE_ERR_CONFIG, "lsf_freq must be in [1e-3, 1e3]");
    if ((int)roundf(c->lsf_freq / c->dt) < 1) return set_err(FE_ERR_CONFIG, "lsf_freq must be at least dt/2");
    if (c->lsf_horMnSubTerms < 0 || c->lsf_horMnSubTerms > 1) return set_err(FE_ERR_CONFIG, "lsf_horMnSubTerms must be 0 or 1");
  }
  if (c->filterSelector < 0 || c->filterSelector > 1) return set_err(FE_ERR_CONFIG, "filterSelector must be 0 or 1");
  if (c->filterSelector > 0 && !(c->filter_6th_coeff >= 0.0f && c->filter_6th_coeff <= 1.0f))
    return set_err(FE_ERR_CONFIG, "filter_6th_coeff must be in [0, 1]");
  if (c->moistureSelector > 0) {
    if (c->moistureNvars < 1 || c->moistureNvars > 2) return set_err(FE_ERR_CONFIG, "moistureNvars must be 1 or 2");
    if (c->moistureAdvSelectorQv < 0 || c->moistureAdvSelectorQv > 6)
      return set_err(FE_ERR_CONFIG, "moistureAdvSelectorQv must be 0..6");
    if (!(c->moistureAdvSelectorQv_b >= 0.0f && c->moistureAdvSelectorQv_b <= 1.0f))
      return set_err(FE_ERR_CONFIG, "moistureAdvSelectorQv_b must be in [0, 1]");
    if (c->moistureNvars > 1 && (c->moistureAdvSelectorQi < 0 || c->moistureAdvSelectorQi > 2))
      return set_err(FE_ERR_CONFIG, "moistureAdvSelectorQi must be 0..2");
  }
  if (c->surflayerSelector < 0 || c->surflayerSelector > 2) return set_err(FE_ERR_CONFIG, "surflayerSelector 0..2");
  if (c->TKESelector > 1) return set_err(FE_ERR_CONFIG, "TKESelector must be 0 or 1");
  if (!(c->dt > 0.0f)) return set_err(FE_ERR_CONFIG, "dt must be positive");
  const long long n = (long long)(c->Nx + 6) * (c->Ny + 6) * (c->Nz + 6);
  if (n >= (1LL << 31)) return set_err(FE_ERR_CONFIG, "a single field exceeds 2^31 cells");
  return FE_OK;
}

static void make_phys(fe_domain* d) { fe::phys_from_config(d->cfg, d->P); }

static int dev_alloc(fe_domain* d, float** p, size_t nfloats) {
  cudaError_t e = cudaMalloc((void**)p, nfloats * sizeof(float));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(FE_ERR_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
  }
  d->bytes += nfloats * sizeof(float);
  CU(cudaMemsetAsync(*p, 0, nfloats * sizeof(float), d->stream));
  return FE_OK;
}

static void free_domain(fe_domain* d) {
  if (!d) return;
  if (d->graph) cudaGraphExecDestroy(d->graph);
  for (void* m : d->peerMaps) cudaIpcCloseMemHandle(m);
  cudaFree(d->arena);
  cudaFree(d->grid);
  cudaFree(d->base);
  cudaFree(d->scratch);
  cudaFree(d->surf);
  cudaFree(d->frhs);
  cudaFree(d->lsfMem);
  cudaFree(d->feat);
  cudaFree(d->clock);
  cudaFree(d->counter);
  if (d->fork) cudaEventDestroy(d->fork);
  if (d->join) cudaEventDestroy(d->join);
  if (d->side) cudaStreamDestroy(d->side);
  if (d->stream) cudaStreamDestroy(d->stream);
  delete d;
}

static int march_attrs();
static cudaError_t sgs_march_attrs();

extern "C" int fe_create(const fe_config* cfg, int device, fe_domain** out) {
  if (!cfg || !out) return set_err(FE_ERR_ARG, "NULL argument");
  *out = nullptr;
  int rc = fe_check_config(cfg);
  if (rc) return rc;
  int ndev = fe_device_count();
  if (ndev <= 0) return set_err(FE_ERR_NO_DEVICE, "no CUDA device visible");
  if (device < 0 || device >= ndev) return set_err(FE_ERR_ARG, "device index out of range");
  fe_domain* d = new fe_domain();
  d->cfg = *cfg;
  d->device = device;
  make_phys(d);
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&d->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    free_domain(d);
    return set_err(FE_ERR_CUDA, "cannot create streams and events on the device");
  }
  const Phys& P = d->P;
  const size_t n = (size_t)P.n, n2 = (size_t)P.n2;
  {
    // default march shape: the most planes per thread block of 32 levels x 8 rows (64, 32, 16, 8)
    // that still leaves 20 waves of two blocks per SM (many blocks balance the SMs, long blocks
    // amortise each block's first plane: 16 at 512x512x128, 64 at 1024x1024x256, as the
    // autotuner finds), else 8
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const long long cols = (long long)((P.Nz + fe::MK - 1) / fe::MK) * ((P.Ny + 7) / 8);
    d->mni = 8;
    for (int ni = 64; ni >= 8; ni /= 2)
      if (cols * ((P.Nx + ni - 1) / ni) >= 40LL * nsm) {
        d->mni = ni;
        break;
      }
    d->mniDefault = d->mni;
    // fused SGS kernel (tiles of 32 levels x 8 rows, two blocks per SM): the most planes per block
    // of 64, 32, 16, 8 that still leaves 10 waves
    d->sgsNi = 8;
    for (int ni = 64; ni >= 8; ni /= 2)
      if (cols * ((P.Nx + ni - 1) / ni) >= 20LL * nsm) {
        d->sgsNi = ni;
        break;
      }
    d->lsfBlocks = P.lsfSub ? 2 * nsm : 0;
  }
  rc = march_attrs();
  if (rc == FE_OK) {
    cudaError_t ea = sgs_march_attrs();
    if (ea == cudaSuccess) ea = fe::batch_set_attrs();
    if (ea != cudaSuccess) rc = set_err(FE_ERR_CUDA, std::string("SGS kernel attributes: ") + cudaGetErrorString(ea));
  }
  if (rc == FE_OK) rc = dev_alloc(d, &d->arena, 3 * n * (P.nf + 1));
  for (int b = 0; b < 3 && rc == FE_OK; b++) {
    d->st[b] = d->arena + b * n * P.nf;
    d->pr[b] = d->arena + 3 * n * P.nf + b * n;
  }
  const size_t nsgs = (size_t)(9 + 3 + 1 + 3 * std::max(P.nmoist, 1));
  const size_t nscr = nsgs + (P.turb ? 7 : 0);  // + the march kernel's SGS tendencies
  if (rc == FE_OK) rc = dev_alloc(d, &d->grid, n * 7);
  if (rc == FE_OK) rc = dev_alloc(d, &d->base, n * 3);
  if (rc == FE_OK) rc = dev_alloc(d, &d->scratch, n * nscr);
  if (rc == FE_OK) rc = dev_alloc(d, &d->surf, n2 * 11);
  const size_t lsfProfBytes = ((size_t)5 * P.nzh * sizeof(float) + 255) / 256 * 256;
  if (rc == FE_OK && P.lsfSub) {
    const size_t bytes = lsfProfBytes + (size_t)d->lsfBlocks * 5 * P.nzh * sizeof(double);
    if (cudaMalloc(&d->lsfMem, bytes) != cudaSuccess) {
      cudaGetLastError();
      rc = set_err(FE_ERR_NOMEM, "slab-mean buffer allocation failed");
    } else {
      cudaMemsetAsync(d->lsfMem, 0, bytes, d->stream);
    }
  }
  if (rc == FE_OK) {
    cudaError_t e = cudaMalloc(&d->clock, 64);
    if (e == cudaSuccess) e = cudaMalloc(&d->counter, sizeof(unsigned long long));
    if (e != cudaSuccess) rc = set_err(FE_ERR_NOMEM, "clock allocation failed");
    else cudaMemsetAsync(d->clock, 0, 64, d->stream);
  }
  if (rc != FE_OK) {
    free_domain(d);
    return rc;
  }
  Ptrs& Q = d->Q;
  Q.zPos = d->grid;
  Q.J31 = d->grid + n;
  Q.J32 = d->grid + 2 * n;
  Q.J33 = d->grid + 3 * n;
  Q.D = d->grid + 4 * n;
  Q.invD = d->grid + 5 * n;
  Q.delta = d->grid + 6 * n;
  Q.rhoBS = d->base;
  Q.thBS = d->base + n;
  Q.pBS = d->base + 2 * n;
  Q.tau = d->scratch;
  Q.tkeQ = d->scratch + 9 * n;
  Q.ls = d->scratch + 12 * n;
  Q.mtau = d->scratch + 13 * n;
  Q.sgsF = P.turb ? d->scratch + nsgs * n : nullptr;
  Q.lsfProf = P.lsfSub ? (float*)d->lsfMem : nullptr;
  Q.lsfPart = P.lsfSub ? (double*)((char*)d->lsfMem + lsfProfBytes) : nullptr;
  float* s = d->surf;
  Q.cd = s; Q.ch = s + n2; Q.cq = s + 2 * n2; Q.fricVel = s + 3 * n2; Q.htFlux = s + 4 * n2; Q.tskin = s + 5 * n2;
  Q.invOblen = s + 6 * n2; Q.z0m = s + 7 * n2; Q.z0t = s + 8 * n2; Q.qFlux = s + 9 * n2; Q.qskin = s + 10 * n2;
  Q.clockIt = (int*)d->clock;
  Q.clockTime = (float*)((char*)d->clock + 16);
  // device-evaluated constants (the reference evaluates them with device powf in every kernel)
  float* kc = nullptr;
  if (cudaMalloc(&kc, 2 * sizeof(float)) != cudaSuccess) {
    free_domain(d);
    return set_err(FE_ERR_NOMEM, "constant buffer allocation failed");
  }
  fe::k_consts<<<1, 1, 0, d->stream>>>(P.R_gas, P.p0, P.R_cp, P.presGrnd, kc);
  float hc[2] = {0, 0};
  cudaError_t e = cudaMemcpyAsync(hc, kc, sizeof(hc), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  cudaFree(kc);
  if (e != cudaSuccess) {
    free_domain(d);
    return set_err(FE_ERR_CUDA, std::string("constant setup failed: ") + cudaGetErrorString(e));
  }
  d->P.c1 = hc[0];
  d->P.presFac = hc[1];
  d->launches = 1;
  *out = d;
  return FE_OK;
}

extern "C" int fe_destroy(fe_domain* d) {
  if (!d) return FE_OK;
  cudaSetDevice(d->device);
  cudaStreamSynchronize(d->stream);
  free_domain(d);
  return FE_OK;
}

extern "C" size_t fe_device_bytes(const fe_domain* d) { return d ? d->bytes : 0; }
extern "C" void* fe_stream(fe_domain* d) { return d ? (void*)d->stream : nullptr; }
extern "C" long long fe_launch_count(const fe_domain* d) { return d ? d->launches : 0; }

static int h2d(fe_domain* d, float* dst, const float* src, size_t nfloats) {
  if (!src) return FE_OK;
  CU(cudaMemcpyAsync(dst, src, nfloats * sizeof(float), cudaMemcpyHostToDevice, d->stream));
  return FE_OK;
}

static void invalidate_graph(fe_domain* d) {
  if (d->graph) {
    cudaGraphExecDestroy(d->graph);
    d->graph = nullptr;
    d->graphSteps = 0;
  }
}

extern "C" int fe_set_grid(fe_domain* d, const float* zPos, const float* J31, const float* J32, const float* J33,
                           const float* D_Jac, const float* invD_Jac) {
  if (!d || !zPos || !J31 || !J32 || !J33 || !D_Jac || !invD_Jac) return set_err(FE_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(d->device));
  const size_t n = (size_t)d->P.n;
  int rc = h2d(d, d->grid, zPos, n);
  if (!rc) rc = h2d(d, d->grid + n, J31, n);
  if (!rc) rc = h2d(d, d->grid + 2 * n, J32, n);
  if (!rc) rc = h2d(d, d->grid + 3 * n, J33, n);
  if (!rc) rc = h2d(d, d->grid + 4 * n, D_Jac, n);
  if (!rc) rc = h2d(d, d->grid + 5 * n, invD_Jac, n);
  if (rc) return rc;
  fe::k_delta<<<(unsigned)((n + 255) / 256), 256, 0, d->stream>>>(d->P, (long long)n, d->grid + 4 * n, d->grid + 6 * n);
  d->launches++;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(d->stream));
  d->haveGrid = true;
  return FE_OK;
}

extern "C" int fe_set_base_state(fe_domain* d, const float* bs) {
  if (!d || !bs) return set_err(FE_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(d->device));
  const size_t n = (size_t)d->P.n;
  int rc = h2d(d, d->base, bs, 2 * n);
  if (rc) return rc;
  const int thr = 256;
  fe::k_pbs<<<(unsigned)((n + thr - 1) / thr), thr, 0, d->stream>>>((long long)n, d->base + n, d->P.c1, d->P.cp_cv,
                                                                    d->base + 2 * n);
  d->launches++;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(d->stream));
  d->haveBase = true;
  return FE_OK;
}

extern "C" int fe_set_surface(fe_domain* d, const float* z0m, const float* z0t, const float* htFlux, const float* tskin,
                              const float* fricVel, const float* qFlux, const float* qskin) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  const size_t n2 = (size_t)d->P.n2;
  int rc = h2d(d, d->Q.z0m, z0m, n2);
  if (!rc) rc = h2d(d, d->Q.z0t, z0t, n2);
  if (!rc) rc = h2d(d, d->Q.htFlux, htFlux, n2);
  if (!rc) rc = h2d(d, d->Q.tskin, tskin, n2);
  if (!rc) rc = h2d(d, d->Q.fricVel, fricVel, n2);
  if (!rc) rc = h2d(d, d->Q.qFlux, qFlux, n2);
  if (!rc) rc = h2d(d, d->Q.qskin, qskin, n2);
  if (rc) return rc;
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

static int finish_state(fe_domain* d);

// ------------------------------------------------------------------ checkpoint / resume
// A checkpoint holds everything a step reads that a step also changes: the prognostic state A,
// the 11 surface planes (the surface layer starts from the previous drag, friction velocity,
// Obukhov length, fluxes and skin values), the clock and, with slab-mean subsidence, the third
// state buffer (the next forcing step's slab means read its halo cells: the previous step's
// last-stage input). Scratch, the second state buffer and the perturbation pressure are rebuilt
// on load, so a resumed run repeats the continuous one bit for bit. Version 2 records whether the
// third buffer is present; a checkpoint loads only into a domain of the same shape, field set and
// subsidence setting.
namespace {
struct CkptHeader {
  char magic[8];
  int version, Nx, Ny, Nz, nf, simIt;
  float simTime;
  int lsfSub;  // 1: the third state buffer follows the surface planes
  int pad[7];
};
constexpr int kCkptVersion = 2;
const char kCkptMagic[8] = {'F', 'E', 'B', '2', '0', '0', 'C', 'K'};
}  // namespace

extern "C" size_t fe_checkpoint_bytes(const fe_domain* d) {
  if (!d) return 0;
  // with slab-mean subsidence, also the third state buffer: the next forcing step's slab means read
  // its halo cells (the previous step's last-stage input)
  const size_t ns = (size_t)d->P.nf * (size_t)d->P.n;
  return sizeof(CkptHeader) + sizeof(float) * (ns + 11 * (size_t)d->P.n2 + (d->P.lsfSub ? ns : 0));
}

extern "C" int fe_checkpoint_save(fe_domain* d, void* buf, size_t bytes) {
  if (!d || !buf) return set_err(FE_ERR_ARG, "NULL argument");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  if (bytes < fe_checkpoint_bytes(d)) return set_err(FE_ERR_ARG, "checkpoint buffer too small");
  CU(cudaSetDevice(d->device));
  CU(cudaStreamSynchronize(d->stream));
  CkptHeader h;
  std::memset(&h, 0, sizeof(h));
  std::memcpy(h.magic, kCkptMagic, 8);
  h.version = kCkptVersion; h.Nx = d->P.Nx; h.Ny = d->P.Ny; h.Nz = d->P.Nz; h.nf = d->P.nf;
  h.lsfSub = d->P.lsfSub ? 1 : 0;
  h.simIt = d->simIt; h.simTime = d->simTime;
  std::memcpy(buf, &h, sizeof(h));
  float* f = reinterpret_cast<float*>(static_cast<char*>(buf) + sizeof(h));
  const size_t ns = (size_t)d->P.nf * (size_t)d->P.n, n2 = 11 * (size_t)d->P.n2;
  CU(cudaMemcpyAsync(f, d->st[0], ns * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
  CU(cudaMemcpyAsync(f + ns, d->surf, n2 * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
  if (d->P.lsfSub) CU(cudaMemcpyAsync(f + ns + n2, d->st[2], ns * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_checkpoint_load(fe_domain* d, const void* buf, size_t bytes) {
  if (!d || !buf) return set_err(FE_ERR_ARG, "NULL argument");
  if (!d->haveGrid || !d->haveBase) return set_err(FE_ERR_STATE, "set the grid and base state before loading");
  if (bytes < sizeof(CkptHeader)) return set_err(FE_ERR_ARG, "checkpoint too short");
  CkptHeader h;
  std::memcpy(&h, buf, sizeof(h));
  if (std::memcmp(h.magic, kCkptMagic, 8) != 0) return set_err(FE_ERR_ARG, "not a checkpoint of this engine");
  if (h.version != kCkptVersion) return set_err(FE_ERR_ARG, "checkpoint of another format version");
  if (h.Nx != d->P.Nx || h.Ny != d->P.Ny || h.Nz != d->P.Nz || h.nf != d->P.nf)
    return set_err(FE_ERR_ARG, "checkpoint of a different domain shape or field set");
  if (h.lsfSub != (d->P.lsfSub ? 1 : 0))
    return set_err(FE_ERR_ARG, "checkpoint of a domain with a different large-scale subsidence setting");
  if (bytes < fe_checkpoint_bytes(d)) return set_err(FE_ERR_ARG, "checkpoint too short");
  CU(cudaSetDevice(d->device));
  const float* f = reinterpret_cast<const float*>(static_cast<const char*>(buf) + sizeof(h));
  const size_t ns = (size_t)d->P.nf * (size_t)d->P.n, n2 = 11 * (size_t)d->P.n2;
  CU(cudaMemcpyAsync(d->st[0], f, ns * sizeof(float), cudaMemcpyHostToDevice, d->stream));
  CU(cudaMemcpyAsync(d->surf, f + ns, n2 * sizeof(float), cudaMemcpyHostToDevice, d->stream));
  int rc = finish_state(d);
  if (rc) return rc;
  if (d->P.lsfSub) {
    CU(cudaMemcpyAsync(d->st[2], f + ns + n2, ns * sizeof(float), cudaMemcpyHostToDevice, d->stream));
    CU(cudaStreamSynchronize(d->stream));
  }
  return fe_set_clock(d, h.simTime, h.simIt);
}

extern "C" int fe_set_clock(fe_domain* d, float simTime, int simTime_it) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  int it = simTime_it;
  CU(cudaMemcpyAsync(d->Q.clockIt, &it, sizeof(int), cudaMemcpyHostToDevice, d->stream));
  CU(cudaMemcpyAsync(d->Q.clockTime, &simTime, sizeof(float), cudaMemcpyHostToDevice, d->stream));
  CU(cudaStreamSynchronize(d->stream));
  d->simTime = simTime;
  d->simIt = simTime_it;
  return FE_OK;
}

extern "C" int fe_get_clock(const fe_domain* d, float* simTime, int* simTime_it) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (simTime) *simTime = d->simTime;
  if (simTime_it) *simTime_it = d->simIt;
  return FE_OK;
}

static unsigned blocks1d(long long n, int thr) { return (unsigned)((n + thr - 1) / thr); }

static int finish_state(fe_domain* d);

extern "C" int fe_set_state(fe_domain* d, const float* hydro, const float* sgstke, const float* moist) {
  if (!d || !hydro) return set_err(FE_ERR_ARG, "NULL argument");
  if (!d->haveGrid || !d->haveBase) return set_err(FE_ERR_STATE, "set the grid and base state before the state");
  if (d->P.ntke && !sgstke) return set_err(FE_ERR_ARG, "TKE field required");
  if (d->P.nmoist && !moist) return set_err(FE_ERR_ARG, "moisture fields required");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  const size_t n = (size_t)P.n;
  float* A = d->st[0];
  int rc = h2d(d, A, hydro, 5 * n);
  if (!rc && P.ntke) rc = h2d(d, A + 5 * n, sgstke, n);
  if (!rc && P.nmoist) rc = h2d(d, A + (5 + P.ntke) * n, moist, n * P.nmoist);
  if (rc) return rc;
  return finish_state(d);
}

// Halo values, perturbation pressure and the copies into B and C of the state just put into A.
static int finish_state(fe_domain* d) {
  const Phys& P = d->P;
  const size_t n = (size_t)P.n;
  float* A = d->st[0];
  fe::k_fill<<<blocks1d(P.n, 256), 256, 0, d->stream>>>(P, d->Q, A);
  CU(cudaGetLastError());
  fe::k_pressure<<<blocks1d(P.n, 256), 256, 0, d->stream>>>(P, d->Q, A, d->pr[0]);
  CU(cudaGetLastError());
  d->launches += 2;
  // the boundary values that never change (base-state and constant halos) must be valid
  // in every buffer, so start B and C as copies of the filled A
  for (int b = 1; b < 3; b++) {
    CU(cudaMemcpyAsync(d->st[b], A, n * P.nf * sizeof(float), cudaMemcpyDeviceToDevice, d->stream));
    CU(cudaMemcpyAsync(d->pr[b], d->pr[0], n * sizeof(float), cudaMemcpyDeviceToDevice, d->stream));
  }
  CU(cudaStreamSynchronize(d->stream));
  d->haveState = true;
  return FE_OK;
}

static dim3 stage_grid(const fe_domain* d) {
  const Phys& P = d->P;
  return dim3((P.Nz + d->tk - 1) / d->tk, (P.Ny + d->tj - 1) / d->tj, (P.Nx + d->ti - 1) / d->ti);
}
// Last-stage SGS physics on the +1 ring (k_turb_t: shared-memory tiles of primitives).
// The last-stage SGS physics of the +1 ring: the tiled kernel for the interior levels on stream s
// and, beside it on the side stream, the surface layer of the ring's columns (first-level tau31,
// tau32, tauTH3 and q_v flux, which the tiled kernel leaves alone) and the ring-level kernel for
// the level above; the three write disjoint values. Returns the number of kernels launched.
static int launch_turb(const fe_domain* d, cudaStream_t s, const float* st, int stage) {
  const Phys& P = d->P;
  const dim3 g((P.Nz + fe::TT_K - 1) / fe::TT_K, (P.Ny + 2 + fe::TT_J - 1) / fe::TT_J, (P.Nx + 2 + fe::TT_I - 1) / fe::TT_I);
  const long long ring = (long long)(P.Nx + 2) * (P.Ny + 2);
  cudaEventRecord(d->fork, s);
  cudaStreamWaitEvent(d->side, d->fork, 0);
  if (P.surf > 0) fe::k_surface<<<dim3((P.Ny + 1 + 127) / 128, P.Nx + 1), 128, 0, d->side>>>(P, d->Q, st, stage);
  fe::k_turb_ring<<<(unsigned)((ring + 255) / 256), 256, 0, d->side>>>(P, d->Q, st, stage);
  cudaEventRecord(d->join, d->side);
  fe::k_turb_t<<<g, dim3(fe::TT_K, fe::TT_J, fe::TT_I), 0, s>>>(P, d->Q, st, stage);
  cudaStreamWaitEvent(s, d->join, 0);
  return P.surf > 0 ? 3 : 2;
}

// The fused SGS kernel (fe_sgs_march.cuh) of the configuration's field set.
template <bool TKE, int NQ, int TJ>
static void launch_sgs_march_tj(const fe_domain* d, cudaStream_t s, const float* st, int stage, bool store) {
  const Phys& P = d->P;
  const int ni = d->sgsNi;
  const dim3 g((P.Nz + fe::SG_K - 1) / fe::SG_K, (P.Ny + TJ - 1) / TJ, (P.Nx + ni - 1) / ni);
  fe::k_sgs_march<TKE, NQ, TJ><<<g, dim3(fe::SG_K, TJ), fe::SgsTile<TJ>::SMEM_BYTES, s>>>(P, d->Q, st, stage, ni,
                                                                                         store ? 1 : 0, d->mlp ? 1 : 0);
}
template <bool TKE, int NQ>
static void launch_sgs_march_nq(const fe_domain* d, cudaStream_t s, const float* st, int stage, bool store) {
  if (d->sgsRows == 16) launch_sgs_march_tj<TKE, NQ, 16>(d, s, st, stage, store);
  else launch_sgs_march_tj<TKE, NQ, 8>(d, s, st, stage, store);
}
static void launch_sgs_march(const fe_domain* d, cudaStream_t s, const float* st, int stage, bool store) {
  const Phys& P = d->P;
  const int nq = (P.nmoist > 0 && P.moistSGS > 0) ? std::min(P.nmoist, 2) : 0;
  if (P.tke) {
    if (nq == 2) launch_sgs_march_nq<true, 2>(d, s, st, stage, store);
    else if (nq == 1) launch_sgs_march_nq<true, 1>(d, s, st, stage, store);
    else launch_sgs_march_nq<true, 0>(d, s, st, stage, store);
  } else {
    if (nq == 2) launch_sgs_march_nq<false, 2>(d, s, st, stage, store);
    else if (nq == 1) launch_sgs_march_nq<false, 1>(d, s, st, stage, store);
    else launch_sgs_march_nq<false, 0>(d, s, st, stage, store);
  }
}
static cudaError_t sgs_march_attrs() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f, int bytes) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  };
  const int b8 = fe::SgsTile<8>::SMEM_BYTES, b16 = fe::SgsTile<16>::SMEM_BYTES;
  set((const void*)fe::k_sgs_march<true, 0, 8>, b8);
  set((const void*)fe::k_sgs_march<true, 1, 8>, b8);
  set((const void*)fe::k_sgs_march<true, 2, 8>, b8);
  set((const void*)fe::k_sgs_march<false, 0, 8>, b8);
  set((const void*)fe::k_sgs_march<false, 1, 8>, b8);
  set((const void*)fe::k_sgs_march<false, 2, 8>, b8);
  set((const void*)fe::k_sgs_march<true, 0, 16>, b16);
  set((const void*)fe::k_sgs_march<true, 1, 16>, b16);
  set((const void*)fe::k_sgs_march<true, 2, 16>, b16);
  set((const void*)fe::k_sgs_march<false, 0, 16>, b16);
  set((const void*)fe::k_sgs_march<false, 1, 16>, b16);
  set((const void*)fe::k_sgs_march<false, 2, 16>, b16);
  return e;
}

// Whether the last-stage physics runs as the fused kernel: the march stage kernel, SGS closure
// on, no learned closure (whose stresses replace the closure's between the two kernels).
static bool fused_sgs(const fe_domain* d) {
  return d->sgsRows > 0 && d->kind == FE_KERNEL_MARCH && d->P.turb;
}

// Everything a physics stage needs before its stage kernel, on state st: the SGS kernel and
// surface layer, the learned closure's stresses (when a network is set) and, for the march
// kernel, the SGS tendencies it reads. With `store`, the closure's stresses and fluxes are left
// in the scratch fields too (the fused kernel keeps them on chip otherwise). Returns the number
// of kernels launched.
static int launch_physics(const fe_domain* d, cudaStream_t s, const float* st, int stage, bool store = false) {
  const Phys& P = d->P;
  if (fused_sgs(d)) {
    // the surface layer first: the fused kernel reads its first-level stresses; with the learned
    // closure, the network's stresses of the ring (inputs from the state) before the fused kernel
    if (P.surf > 0) fe::k_surface<<<dim3((P.Ny + 1 + 127) / 128, P.Nx + 1), 128, 0, s>>>(P, d->Q, st, stage);
    if (d->mlp) fe_learn_enqueue_tau(d->mlp, P, d->Q, st, s, true);
    launch_sgs_march(d, s, st, stage, store);
    return (P.surf > 0 ? 2 : 1) + (d->mlp ? 1 : 0);
  }
  int l = launch_turb(d, s, st, stage);
  if (d->mlp && P.turb) {
    fe_learn_enqueue_tau(d->mlp, P, d->Q, st, s, false);
    l++;
  }
  if (d->kind == FE_KERNEL_MARCH && P.turb) {
    const dim3 g((P.Nz + 31) / 32, (P.Ny + 7) / 8, P.Nx), b(32, 8);
    const int nq = (P.nmoist > 0 && P.moistSGS > 0) ? std::min(P.nmoist, 2) : 0;
    if (P.tke) {
      if (nq == 2) fe::k_sgs_tend<true, 2><<<g, b, 0, s>>>(P, d->Q, st, stage);
      else if (nq == 1) fe::k_sgs_tend<true, 1><<<g, b, 0, s>>>(P, d->Q, st, stage);
      else fe::k_sgs_tend<true, 0><<<g, b, 0, s>>>(P, d->Q, st, stage);
    } else {
      if (nq == 2) fe::k_sgs_tend<false, 2><<<g, b, 0, s>>>(P, d->Q, st, stage);
      else if (nq == 1) fe::k_sgs_tend<false, 1><<<g, b, 0, s>>>(P, d->Q, st, stage);
      else fe::k_sgs_tend<false, 0><<<g, b, 0, s>>>(P, d->Q, st, stage);
    }
    l++;
  }
  return l;
}

static bool stage_has_physics(const fe_domain* d, int stage) { return d->P.oneRK == 0 || stage == 2; }

// Dynamic shared memory limits of the march kernels (three plane buffers exceed the 48 KB
// default at 8 rows); set on the current device before any launch or capture.
static int march_attrs() {
  cudaError_t e = fe::march_set_attrs<0, fe::MODE_COMMIT>();
  if (e == cudaSuccess) e = fe::march_set_attrs<1, fe::MODE_COMMIT>();
  if (e == cudaSuccess) e = fe::march_set_attrs<2, fe::MODE_COMMIT>();
  if (e == cudaSuccess) e = fe::march_set_attrs<0, fe::MODE_FRHS>();
  if (e == cudaSuccess) e = fe::march_set_attrs<1, fe::MODE_FRHS>();
  if (e == cudaSuccess) e = fe::march_set_attrs<2, fe::MODE_FRHS>();
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, std::string("march kernel attributes: ") + cudaGetErrorString(e));
  return FE_OK;
}

// The moist flavour's last stage as a pair (k_march MP = 0 then 1): the kernel that runs in the
// steps without saturation adjustment carries none of its code.
static bool split_last_stage(const fe_domain* d) {
  return d->kind == FE_KERNEL_MARCH && fe::march_split_last_stage(d->P, d->mtj);
}

// Launch the fused stage kernel of stage STAGE in the domain's chosen form.
template <int STAGE, int MODE>
static void launch_stage(const fe_domain* d, cudaStream_t s, const float* cur, const float* base, float* nxt,
                         const float* pcur, float* pnxt, float* frhs) {
  const Phys& P = d->P;
  if (d->kind == FE_KERNEL_MARCH) {
    fe::march_launch<STAGE, MODE>(P, d->Q, d->mtj, d->mni, s, cur, base, nxt, pcur, pnxt, frhs);
  } else {
    fe::k_stage<STAGE, MODE><<<stage_grid(d), dim3(d->tk, d->tj, d->ti), 0, s>>>(P, d->Q, cur, base, nxt, pcur, pnxt, frhs);
  }
}

// Slab means of the large-scale subsidence terms; the kernels return at once unless the device
// clock says the step takes them (or `force`). Returns the number of kernels launched.
static int launch_slab_means(const fe_domain* d, cudaStream_t s, const float* cur, const float* halo, bool force) {
  const Phys& P = d->P;
  fe::k_slab_partial<<<d->lsfBlocks, std::min(256, (P.nzh + 31) / 32 * 32), 0, s>>>(P, d->Q, cur, halo, force ? 1 : 0);
  fe::k_slab_final<<<(5 * P.nzh + 127) / 128, 128, 0, s>>>(P, d->Q, d->lsfBlocks, force ? 1 : 0);
  return 2;
}

// Enqueue RK3 stage `stage` on stream s (no host synchronisation; graph-capturable). With
// `frhs`, the last stage also stores its tendencies there (the reference's Frhs after a step).
// A slab of a multi-process decomposition ends each stage on the stage barrier: its commit
// wrote the neighbours' halos, and their commits wrote its own.
static void enqueue_stage(fe_domain* d, cudaStream_t s, int stage, float* frhs = nullptr) {
  const Phys& P = d->P;
  float *A = d->st[0], *B = d->st[1], *C = d->st[2];
  const bool physPrep = (P.turb || P.surf > 0);
  if (stage == 0) {
    // slab means of the subsidence terms at the start of a forcing step (phi^n in A; C still
    // holds the previous step's phi** with its boundary images, the reference's halo values)
    if (P.lsfSub) d->launches += launch_slab_means(d, s, A, C, false);
    if (physPrep && stage_has_physics(d, 0)) d->launches += launch_physics(d, s, A, 0);
    launch_stage<0, fe::MODE_COMMIT>(d, s, A, A, B, d->pr[0], d->pr[1], nullptr);
  } else if (stage == 1) {
    if (physPrep && stage_has_physics(d, 1)) d->launches += launch_physics(d, s, B, 1);
    launch_stage<1, fe::MODE_COMMIT>(d, s, B, A, C, d->pr[1], d->pr[2], nullptr);
  } else {
    if (physPrep && stage_has_physics(d, 2)) d->launches += launch_physics(d, s, C, 2, frhs != nullptr);
    launch_stage<2, fe::MODE_COMMIT>(d, s, C, A, A, d->pr[2], d->pr[0], frhs);
    fe::k_clock<<<1, 1, 0, s>>>(d->Q, P.dt);
    d->launches += 1 + (split_last_stage(d) ? 1 : 0);
  }
  d->launches += 1;
  if (d->comm) fe_comm_barrier(d->comm, s);
}

// Enqueue one RK3 step on stream s.
static void enqueue_step(fe_domain* d, cudaStream_t s, float* frhs = nullptr) {
  for (int stage = 0; stage < 3; stage++) enqueue_stage(d, s, stage, stage == 2 ? frhs : nullptr);
}

static const int kGraphSteps = 8;

static int build_graph(fe_domain* d) {
  invalidate_graph(d);
  cudaGraph_t g = nullptr;
  CU(cudaStreamBeginCapture(d->stream, cudaStreamCaptureModeThreadLocal));
  const long long before = d->launches;
  for (int s = 0; s < kGraphSteps; s++) enqueue_step(d, d->stream);
  d->launches = before;
  cudaError_t e = cudaStreamEndCapture(d->stream, &g);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&d->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    d->graph = nullptr;
    return set_err(FE_ERR_CUDA, std::string("graph instantiate failed: ") + cudaGetErrorString(e));
  }
  d->graphSteps = kGraphSteps;
  return FE_OK;
}

static int launches_per_step(const fe_domain* d) {
  const Phys& P = d->P;
  int l = 4 + (split_last_stage(d) ? 1 : 0) + (P.lsfSub ? 2 : 0);
  if (P.turb || P.surf > 0) {
    const int phys = fused_sgs(d) ? 1 + (P.surf > 0) + (d->mlp ? 1 : 0)
                                  : 2 + (P.surf > 0) + ((d->mlp && P.turb) ? 1 : 0) +
                                        ((d->kind == FE_KERNEL_MARCH && P.turb) ? 1 : 0);
    l += (P.oneRK ? 1 : 3) * phys;
  }
  return l;
}

extern "C" int fe_advance(fe_domain* d, int nsteps) {
  if (!d || nsteps < 0) return set_err(FE_ERR_ARG, "bad argument");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  CU(cudaSetDevice(d->device));
  const bool capture = d->captureFrhs && nsteps > 0;
  if (capture && !d->frhs) {
    int rc = dev_alloc(d, &d->frhs, (size_t)d->P.n * d->P.nf);
    if (rc) return rc;
  }
  // with tendency capture the last step runs on its own, its last stage storing the tendencies
  int left = capture ? nsteps - 1 : nsteps;
  if (left >= kGraphSteps) {
    if (!d->graph) {
      int rc = build_graph(d);
      if (rc) return rc;
    }
    while (left >= kGraphSteps) {
      CU(cudaGraphLaunch(d->graph, d->stream));
      d->launches += (long long)kGraphSteps * launches_per_step(d);
      left -= kGraphSteps;
    }
  }
  for (; left > 0; left--) enqueue_step(d, d->stream);
  if (capture) enqueue_step(d, d->stream, d->frhs);
  CU(cudaGetLastError());
  for (int s = 0; s < nsteps; s++) {
    d->simTime = d->simTime + d->P.dt;
    d->simIt += 1;
  }
  return FE_OK;
}

extern "C" int fe_sync(fe_domain* d) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  CU(cudaStreamSynchronize(d->stream));
  CU(cudaGetLastError());
  if (d->mlp) return fe_mlp_check(d->mlp);
  return FE_OK;
}

static int d2h(fe_domain* d, float* dst, const float* src, size_t nfloats) {
  if (!dst) return FE_OK;
  CU(cudaMemcpyAsync(dst, src, nfloats * sizeof(float), cudaMemcpyDeviceToHost, d->stream));
  return FE_OK;
}

extern "C" int fe_get_state(fe_domain* d, float* hydro, float* sgstke, float* moist, float* pres) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  const size_t n = (size_t)P.n;
  int rc = d2h(d, hydro, d->st[0], 5 * n);
  if (!rc && P.ntke) rc = d2h(d, sgstke, d->st[0] + 5 * n, n);
  if (!rc && P.nmoist) rc = d2h(d, moist, d->st[0] + (5 + P.ntke) * n, n * P.nmoist);
  if (!rc) rc = d2h(d, pres, d->pr[0], n);
  if (rc) return rc;
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_get_surface(fe_domain* d, float* cd, float* ch, float* fricVel, float* htFlux, float* invOblen,
                              float* tskin, float* qFlux, float* qskin) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  const size_t n2 = (size_t)d->P.n2;
  const Ptrs& Q = d->Q;
  int rc = d2h(d, cd, Q.cd, n2);
  if (!rc) rc = d2h(d, ch, Q.ch, n2);
  if (!rc) rc = d2h(d, fricVel, Q.fricVel, n2);
  if (!rc) rc = d2h(d, htFlux, Q.htFlux, n2);
  if (!rc) rc = d2h(d, invOblen, Q.invOblen, n2);
  if (!rc) rc = d2h(d, tskin, Q.tskin, n2);
  if (!rc) rc = d2h(d, qFlux, Q.qFlux, n2);
  if (!rc) rc = d2h(d, qskin, Q.qskin, n2);
  if (rc) return rc;
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_build_frhs(fe_domain* d, int stage) {
  if (!d || stage < 0 || stage > 2) return set_err(FE_ERR_ARG, "bad argument");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  if (!d->frhs) {
    int rc = dev_alloc(d, &d->frhs, (size_t)P.n * P.nf);
    if (rc) return rc;
  }
  float* A = d->st[0];
  // the last stage's large-scale forcing on a forcing step uses the slab means of this state
  if (stage == 2 && P.lsfSub) d->launches += launch_slab_means(d, d->stream, A, A, false);
  if ((P.turb || P.surf > 0) && stage_has_physics(d, stage)) {
    d->launches += launch_physics(d, d->stream, A, stage, true);
    CU(cudaGetLastError());
  }
  switch (stage) {
    case 0: launch_stage<0, fe::MODE_FRHS>(d, d->stream, A, A, nullptr, d->pr[0], nullptr, d->frhs); break;
    case 1: launch_stage<1, fe::MODE_FRHS>(d, d->stream, A, A, nullptr, d->pr[0], nullptr, d->frhs); break;
    default: launch_stage<2, fe::MODE_FRHS>(d, d->stream, A, A, nullptr, d->pr[0], nullptr, d->frhs); break;
  }
  d->launches++;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_get_frhs(fe_domain* d, float* hydroFrhs, float* sgstkeFrhs, float* moistFrhs, float* taus) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (!d->frhs) return set_err(FE_ERR_STATE, "no tendency evaluated yet");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  const size_t n = (size_t)P.n;
  int rc = d2h(d, hydroFrhs, d->frhs, 5 * n);
  if (!rc && P.ntke) rc = d2h(d, sgstkeFrhs, d->frhs + 5 * n, n);
  if (!rc && P.nmoist) rc = d2h(d, moistFrhs, d->frhs + (5 + P.ntke) * n, n * P.nmoist);
  if (!rc) rc = d2h(d, taus, d->Q.tau, 9 * n);
  if (rc) return rc;
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_set_forcing_capture(fe_domain* d, int on) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  d->captureFrhs = on != 0;
  return FE_OK;
}

extern "C" int fe_get_sgs_fluxes(fe_domain* d, float* taus, float* moistTaus) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  const size_t n = (size_t)P.n;
  if (taus && !P.turb) return set_err(FE_ERR_STATE, "no SGS stresses without turbulenceSelector");
  if (moistTaus && !(P.turb && P.nmoist > 0 && P.moistSGS > 0))
    return set_err(FE_ERR_STATE, "no moisture SGS fluxes in this configuration");
  int rc = d2h(d, taus, d->Q.tau, 9 * n);
  if (!rc) rc = d2h(d, moistTaus, d->Q.mtau, 3 * n * (size_t)P.nmoist);
  if (rc) return rc;
  CU(cudaStreamSynchronize(d->stream));
  return FE_OK;
}

extern "C" int fe_count_nonfinite(fe_domain* d, long long* count) {
  if (!d || !count) return set_err(FE_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(d->device));
  unsigned long long* dc = d->counter;
  cudaMemsetAsync(dc, 0, sizeof(unsigned long long), d->stream);
  fe::k_nonfinite<<<blocks1d(d->P.n, 256), 256, 0, d->stream>>>(d->P, d->st[0], dc);
  d->launches++;
  unsigned long long h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, dc, sizeof(h), cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, cudaGetErrorString(e));
  *count = (long long)h;
  return FE_OK;
}

extern "C" int fe_domain_means(fe_domain* d, double* means) {
  if (!d || !means) return set_err(FE_ERR_ARG, "NULL argument");
  CU(cudaSetDevice(d->device));
  double* dm = nullptr;
  const int nf = d->P.nf;
  CU(cudaMalloc(&dm, sizeof(double) * nf));
  cudaMemsetAsync(dm, 0, sizeof(double) * nf, d->stream);
  fe::k_means<<<blocks1d(d->P.n, 256), 256, 0, d->stream>>>(d->P, d->st[0], dm);
  d->launches++;
  cudaError_t e = cudaMemcpyAsync(means, dm, sizeof(double) * nf, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  cudaFree(dm);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, cudaGetErrorString(e));
  const double cells = (double)d->P.Nx * d->P.Ny * d->P.Nz;
  for (int f = 0; f < nf; f++) means[f] /= cells;
  return FE_OK;
}

extern "C" int fe_set_tiling(fe_domain* d, int tk, int tj, int ti) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (tk <= 0) tk = 32;
  if (tj <= 0) tj = 4;
  if (ti <= 0) ti = 2;
  if (tk * tj * ti > 256 || tk % 32 != 0) return set_err(FE_ERR_ARG, "tile must have <= 256 threads and tk a multiple of 32");
  d->tk = tk; d->tj = tj; d->ti = ti;
  invalidate_graph(d);
  return FE_OK;
}

extern "C" int fe_set_stage_kernel(fe_domain* d, int kind, int tj, int ni) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (kind != FE_KERNEL_CELL && kind != FE_KERNEL_MARCH) return set_err(FE_ERR_ARG, "unknown stage-kernel form");
  if (kind == FE_KERNEL_MARCH) {
    if (tj <= 0) tj = 8;
    if (ni <= 0) ni = d->mniDefault;
    if (tj != 4 && tj != 8) return set_err(FE_ERR_ARG, "march kernel: tj must be 4 or 8");
    d->mtj = tj;
    d->mni = ni;
  }
  d->kind = kind;
  invalidate_graph(d);
  return FE_OK;
}

extern "C" int fe_set_sgs_kernel(fe_domain* d, int rows) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (rows != 0 && rows != 8 && rows != 16) return set_err(FE_ERR_ARG, "fused SGS kernel: rows must be 0, 8 or 16");
  d->sgsRows = rows;
  invalidate_graph(d);
  return FE_OK;
}

extern "C" int fe_set_sgs_shape(fe_domain* d, int rows, int ni) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (ni < 1) return set_err(FE_ERR_ARG, "fused SGS kernel: planes per block must be >= 1");
  int rc = fe_set_sgs_kernel(d, rows);
  if (rc) return rc;
  d->sgsNi = ni;
  return FE_OK;
}

extern "C" int fe_get_sgs_shape(const fe_domain* d, int* rows, int* ni) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (rows) *rows = d->sgsRows;
  if (ni) *ni = d->sgsNi;
  return FE_OK;
}

extern "C" int fe_get_stage_kernel(const fe_domain* d, int* kind, int* tj, int* ni) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (kind) *kind = d->kind;
  if (tj) *tj = d->kind == FE_KERNEL_MARCH ? d->mtj : d->tj;
  if (ni) *ni = d->kind == FE_KERNEL_MARCH ? d->mni : d->ti;
  return FE_OK;
}

// While alive, the domain's commits write their halo images into its own buffers only: the
// timing launches below must not write into a neighbouring slab's halos (their own halo cells
// of C are rewritten by the neighbours' next stage-2 commit before any read).
struct LocalImages {
  fe_domain* d;
  long long nbr[9];
  explicit LocalImages(fe_domain* dd) : d(dd) {
    std::memcpy(nbr, d->P.nbr, sizeof(nbr));
    std::memset(d->P.nbr, 0, sizeof(nbr));
  }
  ~LocalImages() { std::memcpy(d->P.nbr, nbr, sizeof(nbr)); }
};

// Autotuner: times the dynamics stage kernel (writes only the stage-2 buffer C, which
// every step overwrites) for each candidate form and launch shape and keeps the fastest.
extern "C" int fe_autotune(fe_domain* d, int* tk, int* tj, int* ti) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  CU(cudaSetDevice(d->device));
  struct Cand { int kind, a, b, c; };
  std::vector<Cand> cand;
  for (int tjm : {8, 4})
    for (int ni : {16, 32, 64, 128, 256})
      if (ni <= std::max(16, d->P.Nx)) cand.push_back({FE_KERNEL_MARCH, tjm, ni, 0});
  static const int cell[][3] = {{32, 4, 2}, {32, 8, 1}, {32, 2, 4}, {64, 2, 2}, {64, 4, 1}, {32, 4, 1}, {32, 2, 2}};
  for (auto& c : cell)
    if (!(c[0] > 32 * ((d->P.Nz + 31) / 32) && c[0] > 32)) cand.push_back({FE_KERNEL_CELL, c[0], c[1], c[2]});
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  float best = 1e30f;
  size_t bi = 0;
  const int reps = 5;
  LocalImages local(d);
  const int saved_kind = d->kind, saved_mtj = d->mtj, saved_mni = d->mni, saved_tk = d->tk, saved_tj = d->tj,
            saved_ti = d->ti;
  for (size_t c = 0; c < cand.size(); c++) {
    d->kind = cand[c].kind;
    if (d->kind == FE_KERNEL_MARCH) { d->mtj = cand[c].a; d->mni = cand[c].b; }
    else { d->tk = cand[c].a; d->tj = cand[c].b; d->ti = cand[c].c; }
    launch_stage<1, fe::MODE_COMMIT>(d, d->stream, d->st[1], d->st[0], d->st[2], d->pr[1], d->pr[2], nullptr);
    cudaEventRecord(e0, d->stream);
    for (int r = 0; r < reps; r++)
      launch_stage<1, fe::MODE_COMMIT>(d, d->stream, d->st[1], d->st[0], d->st[2], d->pr[1], d->pr[2], nullptr);
    cudaEventRecord(e1, d->stream);
    d->launches += reps + 1;
    if (cudaEventSynchronize(e1) != cudaSuccess) break;
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) { best = ms; bi = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CU(cudaGetLastError());
  d->kind = saved_kind; d->mtj = saved_mtj; d->mni = saved_mni; d->tk = saved_tk; d->tj = saved_tj; d->ti = saved_ti;
  const Cand& b = cand[bi];
  d->kind = b.kind;
  if (b.kind == FE_KERNEL_MARCH) { d->mtj = b.a; d->mni = b.b; }
  else { d->tk = b.a; d->tj = b.b; d->ti = b.c; }
  // the fused SGS kernel's tile rows and planes per block (it writes only its 7 tendency fields,
  // which the next physics stage rewrites)
  if (fused_sgs(d)) {
    const int saveRows = d->sgsRows, saveNi = d->sgsNi;
    float sbest = 1e30f;
    int brow = saveRows, bni = saveNi;
    cudaEvent_t s0, s1;
    CU(cudaEventCreate(&s0));
    CU(cudaEventCreate(&s1));
    for (int rows : {8, 16})
      for (int ni : {8, 16, 32, 64}) {
        if (ni > std::max(8, d->P.Nx)) continue;
        d->sgsRows = rows;
        d->sgsNi = ni;
        launch_sgs_march(d, d->stream, d->st[0], 2, false);
        cudaEventRecord(s0, d->stream);
        for (int r = 0; r < 3; r++) launch_sgs_march(d, d->stream, d->st[0], 2, false);
        cudaEventRecord(s1, d->stream);
        d->launches += 4;
        if (cudaEventSynchronize(s1) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, s0, s1);
        if (ms < sbest) { sbest = ms; brow = rows; bni = ni; }
      }
    cudaEventDestroy(s0);
    cudaEventDestroy(s1);
    d->sgsRows = brow;
    d->sgsNi = bni;
  }
  invalidate_graph(d);
  if (tk) *tk = d->tk;
  if (tj) *tj = d->tj;
  if (ti) *ti = d->ti;
  return FE_OK;
}

extern "C" int fe_host_register(void* ptr, size_t bytes) {
  if (!ptr || !bytes) return FE_OK;
  cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(FE_ERR_CUDA, std::string("cudaHostRegister: ") + cudaGetErrorString(e));
  }
  return FE_OK;
}

extern "C" int fe_host_unregister(void* ptr) {
  if (!ptr) return FE_OK;
  cudaError_t e = cudaHostUnregister(ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_err(FE_ERR_CUDA, std::string("cudaHostUnregister: ") + cudaGetErrorString(e));
  }
  return FE_OK;
}

// ------------------------------------------------------------------ learned SGS closure: data
namespace fe {
// inputs, closure stresses and density of every `every`-th interior cell (row-major i, j, k)
__global__ void k_sgs_sample(Phys P, Ptrs Q, const float* __restrict__ st, long long every, float* __restrict__ X,
                             float* __restrict__ tau, float* __restrict__ rho) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cells = (long long)P.Nx * P.Ny * P.Nz;
  const long long t = s * every;
  if (t >= cells) return;
  const int k = (int)(t % P.Nz), j = (int)((t / P.Nz) % P.Ny), i = (int)(t / ((long long)P.Nz * P.Ny));
  const long long c = (long long)(i + P.iMin) * P.si + (long long)(j + P.jMin) * P.sj + (k + P.kMin);
  float x[SGS_NIN];
  sgs_inputs(P, Q, st, c, x);
  if (X)
    for (int q = 0; q < SGS_NIN; q++) X[s * SGS_NIN + q] = x[q];
  if (tau)
    for (int q = 0; q < SGS_NOUT; q++) tau[s * SGS_NOUT + q] = Q.tau[q * P.n + c];
  if (rho) rho[s] = st[c];
}

// 2x2x2 box filter (flux form, Favre averages) of a fine state onto a coarse interior, and the
// subfilter fluxes of the coarse cells divided by the filtered density:
//   tau_ij/rho = [<rho u_i u_j> - <rho u_i><rho u_j>/<rho> + <tau_ij^fine>] / <rho>
//   tauTH_j/rho likewise with theta for u_i; the coarse TKE gains the resolved subfilter energy.
__global__ void k_coarsen(Phys Pf, Ptrs Qf, const float* __restrict__ fs, Phys Pc, float* __restrict__ cs,
                          float* __restrict__ tgt) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long cells = (long long)Pc.Nx * Pc.Ny * Pc.Nz;
  if (t >= cells) return;
  const int K = (int)(t % Pc.Nz), J = (int)((t / Pc.Nz) % Pc.Ny), I = (int)(t / ((long long)Pc.Nz * Pc.Ny));
  const long long nf = Pf.n;
  double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};           // rho, rho u, rho v, rho w, rho theta, rho e, rho qv, rho ql
  double uu[6] = {0, 0, 0, 0, 0, 0};                 // rho u u, rho v u, rho w u, rho w v, rho v v, rho w w
  double ut[3] = {0, 0, 0};                          // rho theta u_j
  double tf[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};        // fine closure stresses
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int g = 0; g < 2; g++) {
        const long long c = (long long)(2 * I + a + Pf.iMin) * Pf.si + (long long)(2 * J + b + Pf.jMin) * Pf.sj +
                            (2 * K + g + Pf.kMin);
        const double r = fs[c], ru = fs[nf + c], rv = fs[2 * nf + c], rw = fs[3 * nf + c], rt = fs[4 * nf + c];
        m[0] += r; m[1] += ru; m[2] += rv; m[3] += rw; m[4] += rt;
        if (Pf.ntke) m[5] += fs[5 * nf + c];
        for (int q = 0; q < Pf.nmoist; q++) m[6 + q] += fs[(5 + Pf.ntke + q) * nf + c];
        uu[0] += ru * ru / r; uu[1] += rv * ru / r; uu[2] += rw * ru / r;
        uu[3] += rw * rv / r; uu[4] += rv * rv / r; uu[5] += rw * rw / r;
        ut[0] += rt * ru / r; ut[1] += rt * rv / r; ut[2] += rt * rw / r;
        for (int q = 0; q < 9; q++) tf[q] += Qf.tau[q * nf + c];
      }
  for (int q = 0; q < 8; q++) m[q] *= 0.125;
  for (int q = 0; q < 6; q++) uu[q] *= 0.125;
  for (int q = 0; q < 3; q++) ut[q] *= 0.125;
  for (int q = 0; q < 9; q++) tf[q] *= 0.125;
  const double r = m[0];
  const double s11 = uu[0] - m[1] * m[1] / r, s21 = uu[1] - m[2] * m[1] / r, s31 = uu[2] - m[3] * m[1] / r;
  const double s32 = uu[3] - m[3] * m[2] / r, s22 = uu[4] - m[2] * m[2] / r, s33 = uu[5] - m[3] * m[3] / r;
  const double h1 = ut[0] - m[4] * m[1] / r, h2 = ut[1] - m[4] * m[2] / r, h3 = ut[2] - m[4] * m[3] / r;
  const long long cc = (long long)(I + Pc.iMin) * Pc.si + (long long)(J + Pc.jMin) * Pc.sj + (K + Pc.kMin);
  const long long nc = Pc.n;
  for (int q = 0; q < 5; q++) cs[q * nc + cc] = (float)m[q];
  if (Pc.ntke) cs[5 * nc + cc] = (float)(m[5] + 0.5 * (s11 + s22 + s33));
  for (int q = 0; q < Pc.nmoist; q++) cs[(5 + Pc.ntke + q) * nc + cc] = (float)m[6 + q];
  if (tgt) {
    const double v[9] = {s11 + tf[0], s21 + tf[1], s31 + tf[2], s32 + tf[3], s22 + tf[4],
                         s33 + tf[5], h1 + tf[6], h2 + tf[7], h3 + tf[8]};
    for (int q = 0; q < 9; q++) tgt[t * 9 + q] = (float)(v[q] / r);
  }
}
}  // namespace fe

extern "C" int fe_set_sgs_mlp(fe_domain* d, fe_mlp* m) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  if (m && fe_learn_device(m) != d->device) return set_err(FE_ERR_ARG, "network and domain must be on one device");
  if (m && !d->P.turb) return set_err(FE_ERR_CONFIG, "the learned closure needs turbulenceSelector > 0");
  if (m && !d->feat) {
    CU(cudaSetDevice(d->device));
    int rc = dev_alloc(d, &d->feat, (size_t)d->P.n * fe::SGS_NIN);
    if (rc) return rc;
  }
  d->Q.feat = m ? d->feat : nullptr;
  d->mlp = m;
  invalidate_graph(d);
  return FE_OK;
}

// Evaluate the closure (TKE, or the network when set) on the current state and sample every
// `every`-th interior cell: inputs X (samples x 11), stresses tau (samples x 9), density rho.
extern "C" int fe_sgs_sample(fe_domain* d, long long every, float* X, float* tau, float* rho) {
  if (!d || every < 1) return set_err(FE_ERR_ARG, "bad argument");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  if (!d->P.turb) return set_err(FE_ERR_CONFIG, "no SGS closure configured");
  CU(cudaSetDevice(d->device));
  const Phys& P = d->P;
  const long long cells = ((long long)P.Nx * P.Ny * P.Nz + every - 1) / every;
  float* A = d->st[0];
  d->launches += launch_turb(d, d->stream, A, 2);
  if (d->mlp) {
    CU(fe_learn_enqueue_tau(d->mlp, P, d->Q, A, d->stream, false));
    d->launches++;
  }
  float *dX = nullptr, *dT = nullptr, *dR = nullptr;
  cudaError_t e = cudaMalloc(&dX, sizeof(float) * cells * fe::SGS_NIN);
  if (e == cudaSuccess) e = cudaMalloc(&dT, sizeof(float) * cells * fe::SGS_NOUT);
  if (e == cudaSuccess) e = cudaMalloc(&dR, sizeof(float) * cells);
  if (e == cudaSuccess) {
    fe::k_sgs_sample<<<blocks1d(cells, 256), 256, 0, d->stream>>>(P, d->Q, A, every, dX, dT, dR);
    d->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && X) e = cudaMemcpyAsync(X, dX, sizeof(float) * cells * fe::SGS_NIN, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess && tau)
    e = cudaMemcpyAsync(tau, dT, sizeof(float) * cells * fe::SGS_NOUT, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess && rho) e = cudaMemcpyAsync(rho, dR, sizeof(float) * cells, cudaMemcpyDeviceToHost, d->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(d->stream);
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dR);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, cudaGetErrorString(e));
  if (d->mlp) return fe_mlp_check(d->mlp);
  return FE_OK;
}

// Coarse-grain the state of `fine` (twice the cells per direction, same physical domain) into
// `coarse` and return the subfilter targets (coarse cells x 9, divided by the filtered density).
extern "C" int fe_coarsen(fe_domain* fine, fe_domain* coarse, float* tau_target) {
  if (!fine || !coarse) return set_err(FE_ERR_ARG, "NULL handle");
  if (!fine->haveState || !coarse->haveGrid || !coarse->haveBase) return set_err(FE_ERR_STATE, "states not ready");
  const Phys &Pf = fine->P, &Pc = coarse->P;
  if (Pf.Nx != 2 * Pc.Nx || Pf.Ny != 2 * Pc.Ny || Pf.Nz != 2 * Pc.Nz || Pf.ntke != Pc.ntke || Pf.nmoist != Pc.nmoist)
    return set_err(FE_ERR_ARG, "fine domain must have twice the coarse cells per direction and the same fields");
  if (fine->device != coarse->device) return set_err(FE_ERR_ARG, "domains must be on one device");
  if (!Pf.turb) return set_err(FE_ERR_CONFIG, "the fine domain needs an SGS closure");
  CU(cudaSetDevice(fine->device));
  // the fine model's own subgrid stresses of its current state
  fine->launches += launch_turb(fine, fine->stream, fine->st[0], 2);
  const long long cells = (long long)Pc.Nx * Pc.Ny * Pc.Nz;
  float* dT = nullptr;
  if (tau_target) CU(cudaMalloc(&dT, sizeof(float) * cells * 9));
  fe::k_coarsen<<<blocks1d(cells, 256), 256, 0, fine->stream>>>(Pf, fine->Q, fine->st[0], Pc, coarse->st[0], dT);
  fine->launches++;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && dT) e = cudaMemcpyAsync(tau_target, dT, sizeof(float) * cells * 9, cudaMemcpyDeviceToHost, fine->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(fine->stream);
  cudaFree(dT);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, cudaGetErrorString(e));
  invalidate_graph(coarse);
  int rc = finish_state(coarse);
  if (rc) return rc;
  return FE_OK;
}

extern "C" int fe_time_stage_kernel(fe_domain* d, int reps, float* ms) {
  if (!d || !ms || reps <= 0) return set_err(FE_ERR_ARG, "bad argument");
  if (!d->haveState) return set_err(FE_ERR_STATE, "state not set");
  CU(cudaSetDevice(d->device));
  cudaEvent_t e0, e1;
  CU(cudaEventCreate(&e0));
  CU(cudaEventCreate(&e1));
  LocalImages local(d);
  cudaEventRecord(e0, d->stream);
  for (int r = 0; r < reps; r++)
    launch_stage<1, fe::MODE_COMMIT>(d, d->stream, d->st[1], d->st[0], d->st[2], d->pr[1], d->pr[2], nullptr);
  cudaEventRecord(e1, d->stream);
  d->launches += reps;
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return set_err(FE_ERR_CUDA, cudaGetErrorString(e));
  *ms = t / reps;
  return FE_OK;
}

// ------------------------------------------------------------------ ensembles
extern "C" int fe_ensemble_create(fe_domain** members, int n, fe_ensemble** out) {
  if (!members || n <= 0 || !out) return set_err(FE_ERR_ARG, "bad argument");
  fe_ensemble* e = new fe_ensemble();
  for (int i = 0; i < n; i++) {
    if (!members[i] || members[i]->device != members[0]->device) {
      delete e;
      return set_err(FE_ERR_ARG, "members must be valid and on one device");
    }
    e->m.push_back(members[i]);
  }
  if (cudaSetDevice(members[0]->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return set_err(FE_ERR_CUDA, "cannot create ensemble stream");
  }
  *out = e;
  return FE_OK;
}

// ------------------------------------------------------------------ work-list (batched) form
// Members that all run the dry flavour with the fused SGS kernel (prognostic TKE, no moisture,
// no subsidence means, no network, undecomposed) advance with one launch per kernel of a step:
// each launch walks the tiles of every member (fe_batch.h). Every block marches kListPlanes planes
// (the launch holds all members' blocks, so long blocks keep the GPU full while their start-up --
// the member lookup, the parameter copy and the first planes -- is paid less often); the results
// equal the per-member launches bit for bit (march shapes and SGS tile rows do not change bits).
static const int kListPlanes = 64;
static bool batchable(const fe_ensemble* e) {
  if (!e->wantBatched || e->coupled || e->m.empty()) return false;
  const Phys& P0 = e->m[0]->P;
  for (const fe_domain* d : e->m) {
    const Phys& P = d->P;
    if (fe::march_flavor(P) != fe::FL_DRY || !P.turb || P.lsfSub || P.moist || d->mlp || d->comm || d->sgsRows == 0)
      return false;
    if (P.surf != P0.surf || P.oneRK != P0.oneRK) return false;
    for (int t = 0; t < 9; t++)
      if (P.nbr[t]) return false;
  }
  return true;
}

static int ens_build_batch(fe_ensemble* e) {
  const int nm = (int)e->m.size();
  std::vector<fe::MarchMember> mm[3];
  std::vector<fe::SgsMember> sg[3];
  std::vector<fe::SurfMember> sf[3];
  std::vector<fe::ClockMember> ck;
  std::vector<int> mapM, mapS, mapF;
  int mB = 0, sB = 0, fB = 0;
  for (fe_domain* d : e->m) {
    const Phys& P = d->P;
    const int ni = kListPlanes;
    const int mgx = (P.Nz + fe::MK - 1) / fe::MK, mgy = (P.Ny + 7) / 8, mgz = (P.Nx + ni - 1) / ni;
    const int sni = kListPlanes;
    const int sgx = (P.Nz + fe::SG_K - 1) / fe::SG_K, sgy = (P.Ny + 7) / 8, sgz = (P.Nx + sni - 1) / sni;
    const int gj = (P.Ny + 1 + 127) / 128;
    float *A = d->st[0], *B = d->st[1], *C = d->st[2];
    const float* stIn[3] = {A, B, C};
    const float* base[3] = {A, A, A};
    float* out[3] = {B, C, A};
    const float* pin[3] = {d->pr[0], d->pr[1], d->pr[2]};
    float* pout[3] = {d->pr[1], d->pr[2], d->pr[0]};
    for (int st = 0; st < 3; st++) {
      fe::MarchMember x;
      std::memset(&x, 0, sizeof(x));
      x.P = P;
      x.Q = d->Q;
      x.cur = stIn[st]; x.base = base[st]; x.nxt = out[st]; x.pcur = pin[st]; x.pnxt = pout[st];
      x.ni = ni; x.gx = mgx; x.gy = mgy; x.first = mB;
      mm[st].push_back(x);
      fe::SgsMember y;
      std::memset(&y, 0, sizeof(y));
      y.P = P; y.Q = d->Q; y.st = stIn[st]; y.ni = sni; y.gx = sgx; y.gy = sgy; y.first = sB;
      sg[st].push_back(y);
      fe::SurfMember z;
      std::memset(&z, 0, sizeof(z));
      z.P = P; z.Q = d->Q; z.st = stIn[st]; z.gj = gj; z.first = fB;
      sf[st].push_back(z);
    }
    ck.push_back({d->Q.clockIt, d->Q.clockTime, P.dt});
    const int mi = (int)ck.size() - 1;
    mB += mgx * mgy * mgz;
    sB += sgx * sgy * sgz;
    fB += gj * (P.Nx + 1);
    mapM.resize(mB, mi);
    mapS.resize(sB, mi);
    mapF.resize(fB, mi);
  }
  const size_t szM = sizeof(fe::MarchMember) * nm, szS = sizeof(fe::SgsMember) * nm;
  const size_t szF = sizeof(fe::SurfMember) * nm, szC = sizeof(fe::ClockMember) * nm;
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t total = 3 * (up(szM) + up(szS) + up(szF)) + up(szC) + up(4 * mB) + up(4 * sB) + up(4 * fB);
  if (e->batchMem) cudaFree(e->batchMem);
  e->batchMem = nullptr;
  if (cudaMalloc(&e->batchMem, total) != cudaSuccess) {
    cudaGetLastError();
    return set_err(FE_ERR_NOMEM, "ensemble table allocation failed");
  }
  char* p = (char*)e->batchMem;
  for (int st = 0; st < 3; st++) {
    e->bMarch[st] = (fe::MarchMember*)p;
    CU(cudaMemcpyAsync(p, mm[st].data(), szM, cudaMemcpyHostToDevice, e->stream));
    p += up(szM);
    e->bSgs[st] = (fe::SgsMember*)p;
    CU(cudaMemcpyAsync(p, sg[st].data(), szS, cudaMemcpyHostToDevice, e->stream));
    p += up(szS);
    e->bSurf[st] = (fe::SurfMember*)p;
    CU(cudaMemcpyAsync(p, sf[st].data(), szF, cudaMemcpyHostToDevice, e->stream));
    p += up(szF);
  }
  e->bClock = (fe::ClockMember*)p;
  CU(cudaMemcpyAsync(p, ck.data(), szC, cudaMemcpyHostToDevice, e->stream));
  p += up(szC);
  e->bMapMarch = (int*)p;
  CU(cudaMemcpyAsync(p, mapM.data(), 4 * (size_t)mB, cudaMemcpyHostToDevice, e->stream));
  p += up(4 * mB);
  e->bMapSgs = (int*)p;
  CU(cudaMemcpyAsync(p, mapS.data(), 4 * (size_t)sB, cudaMemcpyHostToDevice, e->stream));
  p += up(4 * sB);
  e->bMapSurf = (int*)p;
  CU(cudaMemcpyAsync(p, mapF.data(), 4 * (size_t)fB, cudaMemcpyHostToDevice, e->stream));
  CU(cudaStreamSynchronize(e->stream));
  e->bMarchBlocks = mB;
  e->bSgsBlocks = sB;
  e->bSurfBlocks = fB;
  return FE_OK;
}

// Work-list launches of one step (the count ens_enqueue_batched_step enqueues).
static int ens_batched_launches(const fe_ensemble* e) {
  const fe_domain* d0 = e->m[0];
  int l = 1;  // clocks
  for (int stage = 0; stage < 3; stage++) l += 1 + (stage_has_physics(d0, stage) ? 1 + (d0->P.surf > 0 ? 1 : 0) : 0);
  return l;
}

// One RK3 step of every member in work-list launches on stream s; returns the launches enqueued.
static int ens_enqueue_batched_step(fe_ensemble* e, cudaStream_t s) {
  const fe_domain* d0 = e->m[0];
  const int nm = (int)e->m.size();
  int l = 0;
  for (int stage = 0; stage < 3; stage++) {
    if (stage_has_physics(d0, stage)) {
      if (d0->P.surf > 0) {
        fe::batch_surface(e->bSurf[stage], e->bMapSurf, e->bSurfBlocks, stage, s);
        l++;
      }
      fe::batch_sgs(e->bSgs[stage], e->bMapSgs, e->bSgsBlocks, stage, s);
      l++;
    }
    fe::batch_march(fe::FL_DRY, stage, e->bMarch[stage], e->bMapMarch, e->bMarchBlocks, s);
    l++;
  }
  fe::batch_clock(e->bClock, nm, s);
  return l + 1;
}

// One graph holds kGraphSteps steps of every member, members as independent branches (or, in the
// work-list form, kGraphSteps steps of work-list launches).
static int ens_build_graph(fe_ensemble* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  cudaGraph_t g = nullptr;
  std::vector<cudaEvent_t> ev(e->m.size());
  cudaEvent_t fork;
  CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (auto& x : ev) CU(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
  CU(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  std::vector<long long> before;
  for (auto* d : e->m) before.push_back(d->launches);
  if (e->batched) {
    for (int s = 0; s < kGraphSteps; s++) ens_enqueue_batched_step(e, e->stream);
  } else if (e->coupled) {
    // slabs of one domain: each stage of every slab, then the next stage (its halos are the
    // neighbours' commits)
    for (int s = 0; s < kGraphSteps; s++)
      for (int stage = 0; stage < 3; stage++) {
        cudaEventRecord(fork, e->stream);
        for (size_t i = 0; i < e->m.size(); i++) {
          fe_domain* d = e->m[i];
          cudaStreamWaitEvent(d->stream, fork, 0);
          enqueue_stage(d, d->stream, stage);
          cudaEventRecord(ev[i], d->stream);
          cudaStreamWaitEvent(e->stream, ev[i], 0);
        }
      }
  } else {
    cudaEventRecord(fork, e->stream);
    for (size_t i = 0; i < e->m.size(); i++) {
      fe_domain* d = e->m[i];
      cudaStreamWaitEvent(d->stream, fork, 0);
      for (int s = 0; s < kGraphSteps; s++) enqueue_step(d, d->stream);
      cudaEventRecord(ev[i], d->stream);
      cudaStreamWaitEvent(e->stream, ev[i], 0);
    }
  }
  for (size_t i = 0; i < e->m.size(); i++) e->m[i]->launches = before[i];
  cudaError_t err = cudaStreamEndCapture(e->stream, &g);
  cudaEventDestroy(fork);
  for (auto& x : ev) cudaEventDestroy(x);
  if (err != cudaSuccess) return set_err(FE_ERR_CUDA, std::string("ensemble capture failed: ") + cudaGetErrorString(err));
  err = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) {
    e->graph = nullptr;
    return set_err(FE_ERR_CUDA, std::string("ensemble instantiate failed: ") + cudaGetErrorString(err));
  }
  e->graphSteps = kGraphSteps;
  return FE_OK;
}

extern "C" int fe_ensemble_advance(fe_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return set_err(FE_ERR_ARG, "bad argument");
  for (auto* d : e->m)
    if (!d->haveState) return set_err(FE_ERR_STATE, "member state not set");
  CU(cudaSetDevice(e->m[0]->device));
  int left = nsteps;
  if (!e->graph) {
    // the form (and, for the work-list form, the member tables) is fixed when the graph is made
    e->batched = batchable(e);
    if (e->batched && !e->batchMem) {
      int rc = ens_build_batch(e);
      if (rc) return rc;
    }
  }
  // earlier work on the members' own streams (their inputs, ...) comes first
  {
    cudaEvent_t prior;
    CU(cudaEventCreateWithFlags(&prior, cudaEventDisableTiming));
    for (auto* d : e->m) {
      cudaEventRecord(prior, d->stream);
      cudaStreamWaitEvent(e->stream, prior, 0);
    }
    cudaEventDestroy(prior);
  }
  if (left >= kGraphSteps && !e->graph) {
    int rc = ens_build_graph(e);
    if (rc) return rc;
  }
  while (left >= kGraphSteps) {
    CU(cudaGraphLaunch(e->graph, e->stream));
    if (e->batched) e->launches += (long long)kGraphSteps * ens_batched_launches(e);
    else
      for (auto* d : e->m) d->launches += (long long)kGraphSteps * launches_per_step(d);
    left -= kGraphSteps;
  }
  if (e->batched)
    for (; left > 0; left--) e->launches += ens_enqueue_batched_step(e, e->stream);
  if (left > 0) {
    cudaEvent_t fork;
    CU(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    // one pass per stage for coupled slabs, one pass over all steps otherwise
    const int passes = e->coupled ? 3 * left : 1;
    for (int p = 0; p < passes; p++) {
      cudaEventRecord(fork, e->stream);
      for (auto* d : e->m) {
        cudaStreamWaitEvent(d->stream, fork, 0);
        if (e->coupled) enqueue_stage(d, d->stream, p % 3);
        else
          for (int s = 0; s < left; s++) enqueue_step(d, d->stream);
        cudaEvent_t done;
        cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
        cudaEventRecord(done, d->stream);
        cudaStreamWaitEvent(e->stream, done, 0);
        cudaEventDestroy(done);
      }
    }
    cudaEventDestroy(fork);
  }
  // later work on a member's own stream (fe_get_state, fe_advance, ...) waits for the ensemble's
  {
    cudaEvent_t done;
    CU(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
    cudaEventRecord(done, e->stream);
    for (auto* d : e->m) cudaStreamWaitEvent(d->stream, done, 0);
    cudaEventDestroy(done);
  }
  CU(cudaGetLastError());
  for (auto* d : e->m)
    for (int s = 0; s < nsteps; s++) {
      d->simTime = d->simTime + d->P.dt;
      d->simIt += 1;
    }
  return FE_OK;
}

extern "C" int fe_ensemble_sync(fe_ensemble* e) {
  if (!e) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(e->m[0]->device));
  CU(cudaStreamSynchronize(e->stream));
  for (auto* d : e->m) CU(cudaStreamSynchronize(d->stream));
  CU(cudaGetLastError());
  return FE_OK;
}

extern "C" void* fe_ensemble_stream(fe_ensemble* e) { return e ? (void*)e->stream : nullptr; }

extern "C" int fe_ensemble_set_batched(fe_ensemble* e, int on) {
  if (!e) return set_err(FE_ERR_ARG, "NULL handle");
  e->wantBatched = on != 0;
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graphSteps = 0;
  if (e->batchMem) {
    cudaStreamSynchronize(e->stream);
    cudaFree(e->batchMem);
  }
  e->batchMem = nullptr;
  e->batched = false;
  return FE_OK;
}

extern "C" int fe_ensemble_is_batched(const fe_ensemble* e) { return e && e->batched ? 1 : 0; }

extern "C" long long fe_ensemble_launch_count(const fe_ensemble* e) {
  if (!e) return 0;
  long long l = e->launches;
  for (const fe_domain* d : e->m) l += d->launches;
  return l;
}

extern "C" int fe_ensemble_destroy(fe_ensemble* e) {
  if (!e) return FE_OK;
  cudaStreamSynchronize(e->stream);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  cudaFree(e->batchMem);
  cudaStreamDestroy(e->stream);
  delete e;
  return FE_OK;
}

// ------------------------------------------------------------------ domain decomposition
// A domain decomposed over px x py slabs (FastEddy's numProcsX x numProcsY ranks, fempi.c:
// 98-160, with the periodic rank topology of fempi.c:226-245): slab r covers the x range
// rx*Nxp.. and y range ry*Nyp.. (rx = r % px, ry = r / px) and is created with Nx = Nxp,
// Ny = Nyp. Each commit writes the slab's own cells and, for its cells within 3 of a slab
// edge, their images in the neighbouring slabs' halos (the per-stage halo exchange of
// cuda_hydroCoreDevice.cu:276-314 and fecuda_Utils.cu:205-418, fused into the commit).
static int check_decomposable(const fe_domain* d, int px, int py) {
  if (px < 1 || py < 1) return set_err(FE_ERR_ARG, "slab counts must be >= 1");
  if (d->P.lsfSub) return set_err(FE_ERR_CONFIG, "the large-scale subsidence means span the whole domain; not decomposable");
  if ((px > 1 && d->P.Nx < 3) || (py > 1 && d->P.Ny < 3))
    return set_err(FE_ERR_CONFIG, "a decomposed direction needs at least 3 cells per slab (the halo width)");
  return FE_OK;
}

static void set_decomposed(fe_domain* d, int px, int py, const long long nbr[9]) {
  std::memcpy(d->P.nbr, nbr, sizeof(d->P.nbr));
  d->P.peerX = px > 1;
  d->P.peerY = py > 1;
  invalidate_graph(d);
}

extern "C" int fe_slab_group_create(fe_domain** slabs, int px, int py, fe_ensemble** out) {
  if (!slabs || !out || px < 1 || py < 1) return set_err(FE_ERR_ARG, "bad argument");
  const int n = px * py;
  for (int r = 0; r < n; r++) {
    if (!slabs[r] || slabs[r]->device != slabs[0]->device) return set_err(FE_ERR_ARG, "slabs must be valid and on one device");
    const Phys &a = slabs[r]->P, &b = slabs[0]->P;
    if (a.Nx != b.Nx || a.Ny != b.Ny || a.Nz != b.Nz || a.nf != b.nf)
      return set_err(FE_ERR_ARG, "slabs must have the same shape and fields");
    int rc = check_decomposable(slabs[r], px, py);
    if (rc) return rc;
  }
  int rc = fe_ensemble_create(slabs, n, out);
  if (rc) return rc;
  (*out)->coupled = true;
  for (int r = 0; r < n; r++) {
    const int rx = r % px, ry = r / px;
    long long nbr[9];
    for (int dx = -1; dx <= 1; dx++)
      for (int dy = -1; dy <= 1; dy++) {
        const int nr = ((ry + dy + py) % py) * px + (rx + dx + px) % px;
        nbr[(dx + 1) * 3 + (dy + 1)] = (long long)(slabs[nr]->arena - slabs[r]->arena);
      }
    set_decomposed(slabs[r], px, py, nbr);
  }
  return FE_OK;
}

extern "C" size_t fe_ipc_handle_bytes(void) { return sizeof(cudaIpcMemHandle_t); }

extern "C" int fe_arena_ipc_handle(fe_domain* d, void* out, size_t bytes) {
  if (!d || !out || bytes < sizeof(cudaIpcMemHandle_t)) return set_err(FE_ERR_ARG, "bad argument");
  CU(cudaSetDevice(d->device));
  cudaIpcMemHandle_t h;
  CU(cudaIpcGetMemHandle(&h, d->arena));
  std::memcpy(out, &h, sizeof(h));
  return FE_OK;
}

extern "C" int fe_set_halo_peers(fe_domain* d, int px, int py, const void* const* handles) {
  if (!d || !handles) return set_err(FE_ERR_ARG, "bad argument");
  int rc = check_decomposable(d, px, py);
  if (rc) return rc;
  CU(cudaSetDevice(d->device));
  long long nbr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::vector<std::pair<std::string, float*>> opened;  // one mapping per distinct peer
  for (int t = 0; t < 9; t++) {
    if (!handles[t] || t == 4) continue;
    const std::string key((const char*)handles[t], sizeof(cudaIpcMemHandle_t));
    float* base = nullptr;
    for (auto& o : opened)
      if (o.first == key) base = o.second;
    if (!base) {
      cudaIpcMemHandle_t h;
      std::memcpy(&h, handles[t], sizeof(h));
      void* p = nullptr;
      cudaError_t e = cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(FE_ERR_CUDA, std::string("cudaIpcOpenMemHandle: ") + cudaGetErrorString(e));
      }
      d->peerMaps.push_back(p);
      base = (float*)p;
      opened.emplace_back(key, base);
    }
    nbr[t] = (long long)(base - d->arena);
  }
  set_decomposed(d, px, py, nbr);
  return FE_OK;
}

extern "C" int fe_clear_halo_peers(fe_domain* d) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  CU(cudaSetDevice(d->device));
  CU(cudaStreamSynchronize(d->stream));
  for (void* m : d->peerMaps) cudaIpcCloseMemHandle(m);
  d->peerMaps.clear();
  const long long none[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  set_decomposed(d, 1, 1, none);
  return FE_OK;
}

extern "C" int fe_set_halo_comm(fe_domain* d, fe_comm* c) {
  if (!d) return set_err(FE_ERR_ARG, "NULL handle");
  d->comm = c;
  invalidate_graph(d);
  return FE_OK;
}

