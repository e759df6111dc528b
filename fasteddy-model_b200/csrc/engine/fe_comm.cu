// fe_comm.cu -- NCCL communicator of a multi-process domain decomposition (stage barrier).
// See fe_comm.h. The NCCL entry points are resolved with dlopen/dlsym; the types come from
// nccl.h so the calls match the library's ABI.
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <string>

#include "fe_comm.h"

int fe_internal_error(int code, const char* msg);

struct fe_comm {
  ncclComm_t comm = nullptr;
  float* flag = nullptr;  // the all-reduced element
  int nranks = 0, rank = 0, device = 0;
};

namespace {
struct Nccl {
  void* lib = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*allReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t) = nullptr;
  const char* (*errorString)(ncclResult_t) = nullptr;
};

// Resolve the NCCL entry points once; returns nullptr (with the reason set) when unavailable.
const Nccl* nccl() {
  static Nccl n;
  static bool tried = false;
  if (tried) return n.lib ? &n : nullptr;
  tried = true;
  void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!lib) return nullptr;
  n.getUniqueId = (decltype(n.getUniqueId))dlsym(lib, "ncclGetUniqueId");
  n.commInitRank = (decltype(n.commInitRank))dlsym(lib, "ncclCommInitRank");
  n.commDestroy = (decltype(n.commDestroy))dlsym(lib, "ncclCommDestroy");
  n.allReduce = (decltype(n.allReduce))dlsym(lib, "ncclAllReduce");
  n.errorString = (decltype(n.errorString))dlsym(lib, "ncclGetErrorString");
  if (!n.getUniqueId || !n.commInitRank || !n.commDestroy || !n.allReduce || !n.errorString) return nullptr;
  n.lib = lib;
  return &n;
}

int nccl_err(const Nccl* n, const char* what, ncclResult_t r) {
  return fe_internal_error(FE_ERR_CUDA, (std::string(what) + ": " + n->errorString(r)).c_str());
}
}  // namespace

extern "C" int fe_comm_unique_id(void* out, size_t bytes) {
  if (!out || bytes < sizeof(ncclUniqueId)) return fe_internal_error(FE_ERR_ARG, "unique-id buffer too small");
  const Nccl* n = nccl();
  if (!n) return fe_internal_error(FE_ERR_CUDA, "NCCL (libnccl.so.2) not found");
  ncclUniqueId id;
  ncclResult_t r = n->getUniqueId(&id);
  if (r != ncclSuccess) return nccl_err(n, "ncclGetUniqueId", r);
  std::memcpy(out, &id, sizeof(id));
  return FE_OK;
}

extern "C" size_t fe_comm_unique_id_bytes(void) { return sizeof(ncclUniqueId); }

extern "C" int fe_comm_create(const void* uid, int nranks, int rank, int device, fe_comm** out) {
  if (!uid || !out || nranks < 1 || rank < 0 || rank >= nranks) return fe_internal_error(FE_ERR_ARG, "bad argument");
  *out = nullptr;
  const Nccl* n = nccl();
  if (!n) return fe_internal_error(FE_ERR_CUDA, "NCCL (libnccl.so.2) not found");
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return fe_internal_error(FE_ERR_CUDA, "cannot select the device");
  }
  fe_comm* c = new fe_comm();
  c->nranks = nranks;
  c->rank = rank;
  c->device = device;
  if (cudaMalloc(&c->flag, sizeof(float)) != cudaSuccess || cudaMemset(c->flag, 0, sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(c->flag);
    delete c;
    return fe_internal_error(FE_ERR_NOMEM, "barrier element allocation failed");
  }
  ncclUniqueId id;
  std::memcpy(&id, uid, sizeof(id));
  ncclResult_t r = n->commInitRank(&c->comm, nranks, id, rank);
  if (r != ncclSuccess) {
    cudaFree(c->flag);
    delete c;
    return nccl_err(n, "ncclCommInitRank", r);
  }
  *out = c;
  return FE_OK;
}

extern "C" int fe_comm_destroy(fe_comm* c) {
  if (!c) return FE_OK;
  const Nccl* n = nccl();
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  if (n && c->comm) n->commDestroy(c->comm);
  cudaFree(c->flag);
  delete c;
  return FE_OK;
}

void fe_comm_barrier(fe_comm* c, cudaStream_t s) {
  const Nccl* n = nccl();
  if (c && n) n->allReduce(c->flag, c->flag, 1, ncclFloat32, ncclSum, c->comm, s);
}
