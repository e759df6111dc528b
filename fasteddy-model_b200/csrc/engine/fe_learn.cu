// fe_learn.cu -- the learned SGS closure (no counterpart in the reference; it replaces the
// stresses of cudaDevice_hydroCoreCalcTaus_PrognosticTKE_DeviatoricTerm,
// cuda_sgsTurbDevice.cu:308-367, where cudaDevice_hydroCoreCalcTurbMixing consumes them,
// cuda_hydroCoreDevice.cu:759-768).
//
// Owns the FP32 master parameters, the Adam moments, the standardisation and a device copy
// of a training set; evaluates gradients and predictions with the tensor-core kernels of
// fe_mlp.cuh and trains with Adam. The time-step hook launches the inference kernel on the
// stress points of a domain after the TKE closure has run, so the network's stresses feed the
// SGS divergence and the TKE shear production of the same stage.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "fasteddy_b200.h"
#include "fe_learn.h"
#include "fe_mlp.cuh"

struct fe_mlp {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // MP_TOTAL FP32 master parameters
  float* grad = nullptr;
  float* mom1 = nullptr;
  float* mom2 = nullptr;
  fe::MlpNorm* norm = nullptr;
  fe::MlpNorm hnorm;
  float* X = nullptr;       // data set: n x 11 inputs, n x 9 targets (tau/rho)
  float* T = nullptr;
  int* order = nullptr;     // shuffled sample order
  long long n = 0;
  double* loss = nullptr;
  int* err = nullptr;
  long long adamStep = 0;
};

namespace {

#define LCU(call)                                                                                   \
  do {                                                                                              \
    cudaError_t e__ = (call);                                                                       \
    if (e__ != cudaSuccess)                                                                         \
      return fe_internal_error(FE_ERR_CUDA, (std::string(#call) + ": " + cudaGetErrorString(e__)).c_str()); \
  } while (0)

int attrs_set(void) {
  cudaError_t e = cudaFuncSetAttribute(fe::k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       fe::MlpTrainSmem::BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fe::k_mlp_infer<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, fe::MlpInferSmem::BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fe::k_mlp_infer<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, fe::MlpInferSmem::BYTES);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fe::k_mlp_infer<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, fe::MlpInferSmem::BYTES);
  if (e != cudaSuccess) return fe_internal_error(FE_ERR_CUDA, cudaGetErrorString(e));
  return FE_OK;
}

int check_err(fe_mlp* m) {
  int h = 0;
  LCU(cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  if (h) {
    cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    return fe_internal_error(FE_ERR_CUDA, "learned closure: a tensor-core completion wait expired");
  }
  return FE_OK;
}

int grid_for(const fe_mlp* m, long long tiles, int perSm) {
  return (int)std::max(1LL, std::min(tiles, (long long)m->nsm * perSm));
}

// gradient of the mean squared standardised error over samples [first, first+count) into m->grad
int launch_grad(fe_mlp* m, long long first, long long count) {
  LCU(cudaMemsetAsync(m->grad, 0, sizeof(float) * fe::MP_TOTAL, m->stream));
  LCU(cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream));
  const long long tiles = (count + fe::MLP_M - 1) / fe::MLP_M;
  fe::k_mlp_train<<<grid_for(m, tiles, 1), 128, fe::MlpTrainSmem::BYTES, m->stream>>>(
      m->params, m->norm, m->X, m->T, m->order, m->n, first, count, m->grad, m->loss, m->err);
  LCU(cudaGetLastError());
  return FE_OK;
}

}  // namespace

int* fe_learn_err_flag(const fe_mlp* m) { return m ? m->err : nullptr; }
int fe_learn_device(const fe_mlp* m) { return m ? m->device : -1; }

cudaError_t fe_learn_enqueue_tau(const fe_mlp* m, const fe::Phys& P, const fe::Ptrs& Q, const float* st, cudaStream_t s,
                                 bool fromState) {
  const long long cells = (long long)(P.Nx + 2) * (P.Ny + 2) * (P.Nz + 1);
  const long long tiles = (cells + fe::MLP_M - 1) / fe::MLP_M;
  if (Q.feat && !fromState)
    fe::k_mlp_infer<2><<<grid_for(m, tiles, 5), 128, fe::MlpInferSmem::BYTES, s>>>(P, Q, st, m->params, m->norm, nullptr,
                                                                                      nullptr, 0, m->err);
  else
    fe::k_mlp_infer<1><<<grid_for(m, tiles, 5), 128, fe::MlpInferSmem::BYTES, s>>>(P, Q, st, m->params, m->norm, nullptr,
                                                                                      nullptr, 0, m->err);
  return cudaGetLastError();
}

extern "C" long long fe_mlp_param_count(void) { return fe::MP_TOTAL; }

extern "C" int fe_mlp_create(int device, unsigned long long seed, fe_mlp** out) {
  if (!out) return fe_internal_error(FE_ERR_ARG, "NULL argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    cudaGetLastError();
    return fe_internal_error(FE_ERR_NO_DEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= ndev) return fe_internal_error(FE_ERR_ARG, "device index out of range");
  LCU(cudaSetDevice(device));
  int major = 0;
  LCU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  if (major != 10) return fe_internal_error(FE_ERR_NO_DEVICE, "the learned closure needs an sm_100 (B200) device");
  int rc = attrs_set();
  if (rc) return rc;
  fe_mlp* m = new fe_mlp();
  m->device = device;
  cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device);
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->params, sizeof(float) * fe::MP_TOTAL);
  if (e == cudaSuccess) e = cudaMalloc(&m->grad, sizeof(float) * fe::MP_TOTAL);
  if (e == cudaSuccess) e = cudaMalloc(&m->mom1, sizeof(float) * fe::MP_TOTAL);
  if (e == cudaSuccess) e = cudaMalloc(&m->mom2, sizeof(float) * fe::MP_TOTAL);
  if (e == cudaSuccess) e = cudaMalloc(&m->norm, sizeof(fe::MlpNorm));
  if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&m->err, sizeof(int));
  if (e != cudaSuccess) {
    fe_mlp_destroy(m);
    return fe_internal_error(FE_ERR_NOMEM, cudaGetErrorString(e));
  }
  cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
  // Glorot-uniform weights, zero biases; padded entries zero
  std::vector<float> p(fe::MP_TOTAL, 0.0f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int ofs, int nout, int nin, int useOut, int useIn) {
    const double a = std::sqrt(6.0 / (double)(useIn + useOut));
    std::uniform_real_distribution<double> U(-a, a);
    for (int o = 0; o < nout; o++)
      for (int i = 0; i < nin; i++) p[ofs + o * nin + i] = (o < useOut && i < useIn) ? (float)U(rng) : 0.0f;
  };
  fill(fe::MP_W1, 64, 16, 64, fe::SGS_NIN);
  fill(fe::MP_W2, 64, 64, 64, 64);
  fill(fe::MP_W3, 64, 64, 64, 64);
  fill(fe::MP_W4, 16, 64, fe::SGS_NOUT, 64);
  rc = fe_mlp_set_params(m, p.data());
  if (!rc) {
    float mu[16] = {0}, sg[16], omu[16] = {0}, osg[16];
    for (int q = 0; q < 16; q++) sg[q] = osg[q] = 1.0f;
    rc = fe_mlp_set_norm(m, mu, sg, omu, osg);
  }
  if (rc) {
    fe_mlp_destroy(m);
    return rc;
  }
  *out = m;
  return FE_OK;
}

extern "C" int fe_mlp_destroy(fe_mlp* m) {
  if (!m) return FE_OK;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  cudaFree(m->params);
  cudaFree(m->grad);
  cudaFree(m->mom1);
  cudaFree(m->mom2);
  cudaFree(m->norm);
  cudaFree(m->X);
  cudaFree(m->T);
  cudaFree(m->order);
  cudaFree(m->loss);
  cudaFree(m->err);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return FE_OK;
}

extern "C" int fe_mlp_set_params(fe_mlp* m, const float* params) {
  if (!m || !params) return fe_internal_error(FE_ERR_ARG, "NULL argument");
  LCU(cudaSetDevice(m->device));
  LCU(cudaMemcpyAsync(m->params, params, sizeof(float) * fe::MP_TOTAL, cudaMemcpyHostToDevice, m->stream));
  LCU(cudaMemsetAsync(m->mom1, 0, sizeof(float) * fe::MP_TOTAL, m->stream));
  LCU(cudaMemsetAsync(m->mom2, 0, sizeof(float) * fe::MP_TOTAL, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  m->adamStep = 0;
  return FE_OK;
}

extern "C" int fe_mlp_get_params(fe_mlp* m, float* params) {
  if (!m || !params) return fe_internal_error(FE_ERR_ARG, "NULL argument");
  LCU(cudaSetDevice(m->device));
  LCU(cudaMemcpyAsync(params, m->params, sizeof(float) * fe::MP_TOTAL, cudaMemcpyDeviceToHost, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  return FE_OK;
}

extern "C" int fe_mlp_set_norm(fe_mlp* m, const float* in_mu, const float* in_sig, const float* out_mu,
                               const float* out_sig) {
  if (!m || !in_mu || !in_sig || !out_mu || !out_sig) return fe_internal_error(FE_ERR_ARG, "NULL argument");
  fe::MlpNorm h;
  for (int q = 0; q < 16; q++) {
    h.in_mu[q] = q < fe::SGS_NIN ? in_mu[q] : 0.0f;
    h.in_sig[q] = q < fe::SGS_NIN ? in_sig[q] : 1.0f;
    h.out_mu[q] = q < fe::SGS_NOUT ? out_mu[q] : 0.0f;
    h.out_sig[q] = q < fe::SGS_NOUT ? out_sig[q] : 1.0f;
    if (!(h.in_sig[q] > 0.0f) || !(h.out_sig[q] > 0.0f))
      return fe_internal_error(FE_ERR_ARG, "standard deviations must be positive");
  }
  LCU(cudaSetDevice(m->device));
  LCU(cudaMemcpyAsync(m->norm, &h, sizeof(h), cudaMemcpyHostToDevice, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  m->hnorm = h;
  return FE_OK;
}

extern "C" int fe_mlp_get_norm(fe_mlp* m, float* in_mu, float* in_sig, float* out_mu, float* out_sig) {
  if (!m) return fe_internal_error(FE_ERR_ARG, "NULL handle");
  for (int q = 0; q < fe::SGS_NIN; q++) {
    if (in_mu) in_mu[q] = m->hnorm.in_mu[q];
    if (in_sig) in_sig[q] = m->hnorm.in_sig[q];
  }
  for (int q = 0; q < fe::SGS_NOUT; q++) {
    if (out_mu) out_mu[q] = m->hnorm.out_mu[q];
    if (out_sig) out_sig[q] = m->hnorm.out_sig[q];
  }
  return FE_OK;
}

extern "C" int fe_mlp_set_data(fe_mlp* m, const float* X, const float* T, long long n, unsigned long long seed,
                               int fit_norm) {
  if (!m || !X || !T || n <= 0) return fe_internal_error(FE_ERR_ARG, "bad argument");
  if (n >= (1LL << 31)) return fe_internal_error(FE_ERR_ARG, "data set too large");
  LCU(cudaSetDevice(m->device));
  cudaFree(m->X);
  cudaFree(m->T);
  cudaFree(m->order);
  m->X = m->T = nullptr;
  m->order = nullptr;
  m->n = 0;
  LCU(cudaMalloc(&m->X, sizeof(float) * n * fe::SGS_NIN));
  LCU(cudaMalloc(&m->T, sizeof(float) * n * fe::SGS_NOUT));
  LCU(cudaMalloc(&m->order, sizeof(int) * n));
  std::vector<int> ord((size_t)n);
  for (long long i = 0; i < n; i++) ord[i] = (int)i;
  std::mt19937_64 rng(seed);
  std::shuffle(ord.begin(), ord.end(), rng);
  LCU(cudaMemcpyAsync(m->X, X, sizeof(float) * n * fe::SGS_NIN, cudaMemcpyHostToDevice, m->stream));
  LCU(cudaMemcpyAsync(m->T, T, sizeof(float) * n * fe::SGS_NOUT, cudaMemcpyHostToDevice, m->stream));
  LCU(cudaMemcpyAsync(m->order, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  m->n = n;
  if (fit_norm) {
    float imu[fe::SGS_NIN], isg[fe::SGS_NIN], omu[fe::SGS_NOUT], osg[fe::SGS_NOUT];
    auto stats = [&](const float* A, int w, int q, float& mu, float& sg) {
      double s = 0.0, s2 = 0.0;
      for (long long i = 0; i < n; i++) s += A[i * w + q];
      const double mean = s / (double)n;
      for (long long i = 0; i < n; i++) {
        const double d = A[i * w + q] - mean;
        s2 += d * d;
      }
      const double sd = std::sqrt(s2 / (double)n);
      mu = (float)mean;
      sg = (float)(sd > 0.0 ? sd : 1.0);
    };
    for (int q = 0; q < fe::SGS_NIN; q++) stats(X, fe::SGS_NIN, q, imu[q], isg[q]);
    for (int q = 0; q < fe::SGS_NOUT; q++) stats(T, fe::SGS_NOUT, q, omu[q], osg[q]);
    return fe_mlp_set_norm(m, imu, isg, omu, osg);
  }
  return FE_OK;
}

extern "C" int fe_mlp_gradient(fe_mlp* m, long long first, long long count, float* grad, double* loss) {
  if (!m || count <= 0 || first < 0) return fe_internal_error(FE_ERR_ARG, "bad argument");
  if (!m->n) return fe_internal_error(FE_ERR_STATE, "no data set");
  LCU(cudaSetDevice(m->device));
  // gradients are taken in data-set order (no shuffling) so callers can reproduce them
  int* saved = m->order;
  m->order = nullptr;
  int rc = launch_grad(m, first, count);
  m->order = saved;
  if (rc) return rc;
  if (grad) LCU(cudaMemcpyAsync(grad, m->grad, sizeof(float) * fe::MP_TOTAL, cudaMemcpyDeviceToHost, m->stream));
  if (loss) LCU(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
  LCU(cudaStreamSynchronize(m->stream));
  return check_err(m);
}

extern "C" int fe_mlp_train(fe_mlp* m, int steps, long long batch, float lr, double* loss_hist) {
  if (!m || steps < 0 || batch <= 0 || !(lr > 0.0f)) return fe_internal_error(FE_ERR_ARG, "bad argument");
  if (!m->n) return fe_internal_error(FE_ERR_STATE, "no data set");
  LCU(cudaSetDevice(m->device));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  std::vector<double> hist;
  double* dl = nullptr;
  if (loss_hist && steps > 0) LCU(cudaMalloc(&dl, sizeof(double) * steps));
  long long pos = 0;
  for (int s = 0; s < steps; s++) {
    const long long cnt = std::min(batch, m->n);
    int rc = launch_grad(m, pos, cnt);
    if (rc) { cudaFree(dl); return rc; }
    pos = (pos + cnt) % m->n;
    m->adamStep++;
    const float c1 = 1.0f - (float)std::pow((double)b1, (double)m->adamStep);
    const float c2 = 1.0f - (float)std::pow((double)b2, (double)m->adamStep);
    fe::k_adam<<<(fe::MP_TOTAL + 255) / 256, 256, 0, m->stream>>>(m->params, m->grad, m->mom1, m->mom2, lr, b1, b2, eps, c1,
                                                                   c2);
    if (dl) cudaMemcpyAsync(dl + s, m->loss, sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
  }
  LCU(cudaGetLastError());
  if (dl) {
    cudaError_t e = cudaMemcpyAsync(loss_hist, dl, sizeof(double) * steps, cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(dl);
    if (e != cudaSuccess) return fe_internal_error(FE_ERR_CUDA, cudaGetErrorString(e));
  }
  LCU(cudaStreamSynchronize(m->stream));
  return check_err(m);
}

extern "C" int fe_mlp_predict(fe_mlp* m, const float* X, long long n, float* Y) {
  if (!m || !X || !Y || n <= 0) return fe_internal_error(FE_ERR_ARG, "bad argument");
  LCU(cudaSetDevice(m->device));
  float *dX = nullptr, *dY = nullptr;
  LCU(cudaMalloc(&dX, sizeof(float) * n * fe::SGS_NIN));
  cudaError_t e = cudaMalloc(&dY, sizeof(float) * n * fe::SGS_NOUT);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dX, X, sizeof(float) * n * fe::SGS_NIN, cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) {
    const long long tiles = (n + fe::MLP_M - 1) / fe::MLP_M;
    fe::Phys P;
    std::memset(&P, 0, sizeof(P));
    fe::Ptrs Q;
    std::memset(&Q, 0, sizeof(Q));
    fe::k_mlp_infer<0><<<grid_for(m, tiles, 5), 128, fe::MlpInferSmem::BYTES, m->stream>>>(P, Q, nullptr, m->params, m->norm,
                                                                                            dX, dY, n, m->err);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(Y, dY, sizeof(float) * n * fe::SGS_NOUT, cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  cudaFree(dX);
  cudaFree(dY);
  if (e != cudaSuccess) return fe_internal_error(FE_ERR_CUDA, cudaGetErrorString(e));
  return check_err(m);
}

// Mean device time of `reps` gradient evaluations over `batch` samples (training) or of
// inference over the first `batch` samples of the data set (FP32 inputs/outputs in HBM).
extern "C" int fe_mlp_time(fe_mlp* m, int train, long long batch, int reps, float* ms) {
  if (!m || !ms || reps <= 0 || batch <= 0) return fe_internal_error(FE_ERR_ARG, "bad argument");
  if (!m->n) return fe_internal_error(FE_ERR_STATE, "no data set");
  LCU(cudaSetDevice(m->device));
  batch = std::min(batch, m->n);
  float* dY = nullptr;
  if (!train) LCU(cudaMalloc(&dY, sizeof(float) * batch * fe::SGS_NOUT));
  cudaEvent_t e0, e1;
  LCU(cudaEventCreate(&e0));
  LCU(cudaEventCreate(&e1));
  const long long tiles = (batch + fe::MLP_M - 1) / fe::MLP_M;
  fe::Phys P;
  std::memset(&P, 0, sizeof(P));
  fe::Ptrs Q;
  std::memset(&Q, 0, sizeof(Q));
  for (int r = -1; r < reps; r++) {
    if (r == 0) cudaEventRecord(e0, m->stream);
    if (train)
      fe::k_mlp_train<<<grid_for(m, tiles, 1), 128, fe::MlpTrainSmem::BYTES, m->stream>>>(
          m->params, m->norm, m->X, m->T, nullptr, m->n, 0, batch, m->grad, m->loss, m->err);
    else
      fe::k_mlp_infer<0><<<grid_for(m, tiles, 5), 128, fe::MlpInferSmem::BYTES, m->stream>>>(P, Q, nullptr, m->params,
                                                                                              m->norm, m->X, dY, batch, m->err);
  }
  cudaEventRecord(e1, m->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(dY);
  if (e != cudaSuccess) return fe_internal_error(FE_ERR_CUDA, cudaGetErrorString(e));
  *ms = t / reps;
  return check_err(m);
}

extern "C" int fe_mlp_check(fe_mlp* m) {
  if (!m) return fe_internal_error(FE_ERR_ARG, "NULL handle");
  LCU(cudaSetDevice(m->device));
  return check_err(m);
}
