// fe_mlp.cuh -- the learned SGS closure on the 5th-generation tensor cores (sm_100a).
//
// Network: 11 -> 64 -> 64 -> 64 -> 9, tanh on the hidden layers (hardware tanh.approx: bf16x2 on
// the BF16-rounded pre-activations for inference, f32 for training; see epi_tanh); inputs standardised ((x - mu) times the
// FP32 reciprocal of sig), outputs tau/rho = out_mu + out_sig * y. Every layer is one 128-row tile of tcgen05.mma
// (kind::f16, BF16 A and B operands from shared memory, FP32 accumulators in tensor memory),
// issued by one thread; the epilogue (tcgen05.ld, bias, tanh, BF16 pack) runs on all 128
// threads, one tile row (one cell) per thread. Operand tiles use the canonical K-major,
// no-swizzle layout: 8-row x 16-byte core matrices, element (r, k) of an R x K tile at byte
//   (r/8)*(K/8)*128 + (k/8)*128 + (r%8)*16 + (k%8)*2
// (leading byte offset 128 between K chunks, stride byte offset (K/8)*128 between row groups).
//
// Training (k_mlp_train) keeps the forward activations of the tile in shared memory and runs
// the backward pass on the same tensor cores: dH(l-1) = dZ(l) W(l) (A = dZ, B = W^T) and the
// weight gradient dW(l)^T = [H(l-1)^T; 1] dZ(l) with the batch as the reduction dimension
// (A = activations transposed plus a row of ones, whose output row is the bias gradient),
// accumulated in tensor memory over all tiles of the CTA and flushed once with atomics.
//
// Every wait on an mbarrier is bounded (about a second of clock); on expiry the kernel
// raises an error flag, releases its tensor memory and returns.
#pragma once
#include <cuda_bf16.h>

#include "fe_sgs.cuh"

namespace fe {

constexpr int MLP_H = 64;    // hidden width
constexpr int MLP_K0 = 16;   // padded input width (11 used)
constexpr int MLP_N4 = 16;   // padded output width (9 used)
constexpr int MLP_M = 128;   // cells per tile (MMA M)
constexpr int MP_W1 = 0;
constexpr int MP_B1 = MP_W1 + MLP_H * MLP_K0;
constexpr int MP_W2 = MP_B1 + MLP_H;
constexpr int MP_B2 = MP_W2 + MLP_H * MLP_H;
constexpr int MP_W3 = MP_B2 + MLP_H;
constexpr int MP_B3 = MP_W3 + MLP_H * MLP_H;
constexpr int MP_W4 = MP_B3 + MLP_H;
constexpr int MP_B4 = MP_W4 + MLP_N4 * MLP_H;
constexpr int MP_TOTAL = MP_B4 + MLP_N4;

struct MlpNorm {
  float in_mu[16], in_sig[16];
  float out_mu[16], out_sig[16];
};

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle, version 1 (sm_100)
__device__ __forceinline__ uint64_t umma_sdesc(const void* p, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_u32(p);
  uint64_t d = (uint64_t)((a >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accum));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bounded wait for the completion of phase `phase`; false when about a second passed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > 4000000000LL) return false;
  }
}

// ------------------------------------------------------------------ canonical tiles
__device__ __forceinline__ int canon(int r, int k, int K) { return (r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

__device__ __forceinline__ void st_chunk(char* base, int r, int q, int K, const float* v) {
  uint4 u;
  __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]), p1 = __floats2bfloat162_rn(v[2], v[3]);
  __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]), p3 = __floats2bfloat162_rn(v[6], v[7]);
  u.x = *reinterpret_cast<uint32_t*>(&p0);
  u.y = *reinterpret_cast<uint32_t*>(&p1);
  u.z = *reinterpret_cast<uint32_t*>(&p2);
  u.w = *reinterpret_cast<uint32_t*>(&p3);
  *reinterpret_cast<uint4*>(base + (r >> 3) * (K >> 3) * 128 + q * 128 + (r & 7) * 16) = u;
}
__device__ __forceinline__ void st_chunk_u(char* base, int r, int q, int K, uint4 u) {
  *reinterpret_cast<uint4*>(base + (r >> 3) * (K >> 3) * 128 + q * 128 + (r & 7) * 16) = u;
}
__device__ __forceinline__ void ld_chunk(const char* base, int r, int q, int K, float* v) {
  const uint4 u = *reinterpret_cast<const uint4*>(base + (r >> 3) * (K >> 3) * 128 + q * 128 + (r & 7) * 16);
  const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
  for (int t = 0; t < 4; t++) {
    __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[t]);
    v[2 * t] = __bfloat162float(p.x);
    v[2 * t + 1] = __bfloat162float(p.y);
  }
}
__device__ __forceinline__ void st_elem(char* base, int r, int k, int K, float v) {
  *reinterpret_cast<__nv_bfloat16*>(base + canon(r, k, K)) = __float2bfloat16_rn(v);
}

// Weights of the CTA into shared memory: W (N x K row-major, FP32) as an N x K tile, and if
// `wt` its transpose as a K x N tile.
__device__ __forceinline__ void stage_weight(const float* __restrict__ W, int N, int K, char* w, char* wt, int tid,
                                             int nthr) {
  for (int e = tid; e < N * K; e += nthr) {
    const int r = e / K, k = e - (e / K) * K;
    const float v = W[e];
    st_elem(w, r, k, K, v);
    if (wt) st_elem(wt, k, r, N, v);
  }
}

// ------------------------------------------------------------------ shared-memory plans
// inference: weights, one input tile, one activation tile (reused layer to layer)
struct MlpInferSmem {
  static constexpr int W1 = 0, W2 = W1 + 64 * 16 * 2, W3 = W2 + 64 * 64 * 2, W4 = W3 + 64 * 64 * 2;
  static constexpr int X0 = W4 + 16 * 64 * 2, H = X0 + 128 * 16 * 2, BIAS = H + 128 * 64 * 2;
  static constexpr int NORM = BIAS + (64 * 3 + 16) * 4, ISIG = NORM + 64 * 4, BAR = ISIG + 16 * 4, TADDR = BAR + 8;
  static constexpr int FLAG = TADDR + 4;
  static constexpr int BYTES = FLAG + 4;
};
// training: also the transposed weights, all forward activations and the backward tiles
struct MlpTrainSmem {
  static constexpr int W1 = 0, W2 = W1 + 64 * 16 * 2, W3 = W2 + 64 * 64 * 2, W4 = W3 + 64 * 64 * 2;
  static constexpr int W4T = W4 + 16 * 64 * 2, W3T = W4T + 64 * 16 * 2, W2T = W3T + 64 * 64 * 2;
  static constexpr int X0 = W2T + 64 * 64 * 2, H1 = X0 + 128 * 16 * 2, H2 = H1 + 128 * 64 * 2, H3 = H2 + 128 * 64 * 2;
  static constexpr int DZK = H3 + 128 * 64 * 2, DZT = DZK + 128 * 64 * 2, ATH = DZT + 64 * 128 * 2;
  static constexpr int BIAS = ATH + 128 * 128 * 2, NORM = BIAS + (64 * 3 + 16) * 4, ISIG = NORM + 64 * 4;
  static constexpr int RED = ISIG + 16 * 4;
  static constexpr int BAR = RED + 4 * 8, TADDR = BAR + 8, FLAG = TADDR + 4;
  static constexpr int BYTES = FLAG + 4;
};

// tensor-memory columns
constexpr int TM_INFER_COLS = 64;
constexpr int TM_TRAIN_COLS = 512;
constexpr int TC_DF = 0, TC_DB = 64, TC_G4 = 128, TC_G3 = 192, TC_G2 = 256, TC_G1 = 320;

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void stage_isig(const MlpNorm* nmp, float* isig, int tid) {
  if (tid < 16) isig[tid] = 1.0f / nmp->in_sig[tid];
}
// standardised input row -> 2 BF16 chunks of the X0 tile
// (isig: the FP32 reciprocals of in_sig, formed once per CTA by stage_isig)
__device__ __forceinline__ void put_inputs(char* x0, int r, const float* x, const MlpNorm& nm, const float* isig,
                                           bool valid) {
  float v[16];
#pragma unroll
  for (int q = 0; q < 16; q++) v[q] = (valid && q < SGS_NIN) ? (x[q] - nm.in_mu[q]) * isig[q] : 0.0f;
  st_chunk(x0, r, 0, 16, v);
  st_chunk(x0, r, 1, 16, v + 8);
}

// tanh of a hidden unit for training: the hardware tanh.approx.f32 (relative error about
// 2^-11, below the BF16 resolution of the activation tile it feeds)
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
// tanh of two hidden units for inference: the pre-activations rounded to BF16 (the precision of
// the activation tile they end up in) and the hardware tanh.approx.bf16x2, two values per
// special-function instruction; the result is the packed BF16 pair of the tile. The rounding
// is integer arithmetic (add half a BF16 ulp to the FP32 bits, keep the high halves: round to
// nearest, ties away from zero in magnitude) so that the special-function pipe, which the tanh
// saturates, does not also carry a conversion per pair.
__device__ __forceinline__ uint32_t tanh2_bf16(float a, float b) {
  const uint32_t ua = __float_as_uint(a) + 0x8000u, ub = __float_as_uint(b) + 0x8000u;
  const uint32_t p = __byte_perm(ua, ub, 0x7632);  // a's high half low, b's high half high
  uint32_t r;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(r) : "r"(p));
  return r;
}

// hidden-layer epilogue: accumulator row + bias -> tanh -> BF16 tile row. PAIRED (inference):
// tanh2_bf16; otherwise (training, whose gradients are checked tightly) tanh_hw per unit.
template <bool PAIRED>
__device__ __forceinline__ void epi_tanh(uint32_t tacc, const float* bias, char* out, int r) {
#pragma unroll
  for (int g = 0; g < 4; g += 2) {
    float v2[32];
    tmem_ld16(tacc + g * 16, v2);
    tmem_ld16(tacc + g * 16 + 16, v2 + 16);
    tmem_wait_ld();
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const float* v = v2 + 16 * h;
    const float* b = bias + (g + h) * 16;
    if (PAIRED) {
      uint4 lo, hi;
      lo.x = tanh2_bf16(v[0] + b[0], v[1] + b[1]);
      lo.y = tanh2_bf16(v[2] + b[2], v[3] + b[3]);
      lo.z = tanh2_bf16(v[4] + b[4], v[5] + b[5]);
      lo.w = tanh2_bf16(v[6] + b[6], v[7] + b[7]);
      hi.x = tanh2_bf16(v[8] + b[8], v[9] + b[9]);
      hi.y = tanh2_bf16(v[10] + b[10], v[11] + b[11]);
      hi.z = tanh2_bf16(v[12] + b[12], v[13] + b[13]);
      hi.w = tanh2_bf16(v[14] + b[14], v[15] + b[15]);
      st_chunk_u(out, r, 2 * (g + h), 64, lo);
      st_chunk_u(out, r, 2 * (g + h) + 1, 64, hi);
    } else {
      float t[16];
#pragma unroll
      for (int q = 0; q < 16; q++) t[q] = tanh_hw(v[q] + b[q]);
      st_chunk(out, r, 2 * (g + h), 64, t);
      st_chunk(out, r, 2 * (g + h) + 1, 64, t + 8);
    }
  }
  }
}

// make generic shared-memory writes visible to the tensor cores and order tensor-memory reads
// before the next MMA
__device__ __forceinline__ void sync_for_mma() {
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
}

// ------------------------------------------------------------------ inference
// SRC 0: inputs from X[n][11], outputs tau/rho to Y[n][9].
// SRC 1: inputs from the state at the stress points of the +1 ring (levels kMin..kMax), the
//        9 stress/flux fields tau = rho (out_mu + out_sig y) written to Q.tau; the surface
//        layer's tau31, tau32, tauTH3 at kMin are kept.
// SRC 2: as SRC 1 with the inputs read from Q.feat (written by the last-stage SGS kernel).
template <int SRC>
__global__ void __launch_bounds__(128) k_mlp_infer(Phys P, Ptrs Q, const float* __restrict__ st,
                                                   const float* __restrict__ params, const MlpNorm* __restrict__ nmp,
                                                   const float* __restrict__ X, float* __restrict__ Y, long long n,
                                                   int* __restrict__ err) {
  using S = MlpInferSmem;
  extern __shared__ __align__(1024) char sm[];
  const int tid = threadIdx.x, warp = tid >> 5;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::BAR);
  uint32_t* taddrSlot = reinterpret_cast<uint32_t*>(sm + S::TADDR);
  float* bias = reinterpret_cast<float*>(sm + S::BIAS);
  int* flag = reinterpret_cast<int*>(sm + S::FLAG);
  MlpNorm& nm = *reinterpret_cast<MlpNorm*>(sm + S::NORM);
  if (tid < 64) reinterpret_cast<float*>(&nm)[tid] = reinterpret_cast<const float*>(nmp)[tid];
  float* isig = reinterpret_cast<float*>(sm + S::ISIG);
  stage_isig(nmp, isig, tid);
  stage_weight(params + MP_W1, 64, 16, sm + S::W1, nullptr, tid, 128);
  stage_weight(params + MP_W2, 64, 64, sm + S::W2, nullptr, tid, 128);
  stage_weight(params + MP_W3, 64, 64, sm + S::W3, nullptr, tid, 128);
  stage_weight(params + MP_W4, 16, 64, sm + S::W4, nullptr, tid, 128);
  for (int e = tid; e < 64; e += 128) {
    bias[e] = params[MP_B1 + e];
    bias[64 + e] = params[MP_B2 + e];
    bias[128 + e] = params[MP_B3 + e];
  }
  if (tid < 16) bias[192 + tid] = params[MP_B4 + tid];
  if (tid == 0) { mbar_init(bar); *flag = 0; }
  if (warp == 0) tmem_alloc(taddrSlot, TM_INFER_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *taddrSlot;
  const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;

  // ring geometry (SRC 1)
  const int rj = P.Ny + 2, rk = P.Nz + 1;
  const long long ntot = SRC == 0 ? n : (long long)(P.Nx + 2) * rj * rk;
  const long long ntiles = (ntot + MLP_M - 1) / MLP_M;
  const uint32_t id64 = umma_idesc(128, 64), id16 = umma_idesc(128, 16);

  // inputs of one row of a tile (a thread's cell), loaded one tile ahead of its MMA chain
  struct Row {
    float x[SGS_NIN];
    long long c;
    float rho;
    int i, j, k;
    bool valid;
  };
  auto fetch = [&](long long tile, Row& r) {
    const long long row = tile * MLP_M + tid;
    r.valid = tile < ntiles && row < ntot;
    r.c = 0;
    r.rho = 0.0f;
    r.i = r.j = r.k = 0;
#pragma unroll
    for (int q = 0; q < SGS_NIN; q++) r.x[q] = 0.0f;
    if (!r.valid) return;
    if (SRC == 0) {
#pragma unroll
      for (int q = 0; q < SGS_NIN; q++) r.x[q] = X[row * SGS_NIN + q];
    } else {
      r.k = P.kMin + (int)(row % rk);
      r.j = P.jMin - 1 + (int)((row / rk) % rj);
      r.i = P.iMin - 1 + (int)(row / ((long long)rk * rj));
      r.c = (long long)r.i * P.si + (long long)r.j * P.sj + r.k;
      if (SRC == 2) {
#pragma unroll
        for (int q = 0; q < SGS_NIN; q++) r.x[q] = Q.feat[q * P.n + r.c];
      } else {
        sgs_inputs(P, Q, st, r.c, r.x);
      }
      r.rho = st[r.c];
    }
  };
  Row nxt;
  fetch(blockIdx.x, nxt);
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long row = tile * MLP_M + tid;
    const Row cur = nxt;
    const bool valid = cur.valid;
    const long long c = cur.c;
    const float rho = cur.rho;
    const int i = cur.i, j = cur.j, k = cur.k;
    put_inputs(sm + S::X0, tid, cur.x, nm, isig, valid);
    sync_for_mma();
    bool ok = true;
    // layer 1, then the next tile's inputs (loads and, from the state, their arithmetic) while it runs
    if (tid == 0) {
      tc_fence_after();
      umma_bf16(tbase + TC_DF, umma_sdesc(sm + S::X0, 128, 256), umma_sdesc(sm + S::W1, 128, 256), id64, 0);
      umma_commit(bar);
    }
    fetch(tile + gridDim.x, nxt);
    ok = ok && mbar_wait(bar, phase);
    phase ^= 1;
    tc_fence_after();
    epi_tanh<true>(tlane + TC_DF, bias, sm + S::H, tid);
    sync_for_mma();
    // layers 2 and 3 (the MMA has finished reading H before the epilogue overwrites it)
#pragma unroll 1
    for (int l = 0; l < 2; l++) {
      if (tid == 0) {
        tc_fence_after();
        const char* w = sm + (l == 0 ? S::W2 : S::W3);
#pragma unroll
        for (int s = 0; s < 4; s++)
          umma_bf16(tbase + TC_DF, umma_sdesc(sm + S::H + s * 256, 128, 1024), umma_sdesc(w + s * 256, 128, 1024), id64,
                    s > 0);
        umma_commit(bar);
      }
      ok = ok && mbar_wait(bar, phase);
      phase ^= 1;
      tc_fence_after();
      epi_tanh<true>(tlane + TC_DF, bias + 64 * (l + 1), sm + S::H, tid);
      sync_for_mma();
    }
    // layer 4
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < 4; s++)
        umma_bf16(tbase + TC_DF, umma_sdesc(sm + S::H + s * 256, 128, 1024), umma_sdesc(sm + S::W4 + s * 256, 128, 1024),
                  id16, s > 0);
      umma_commit(bar);
    }
    ok = ok && mbar_wait(bar, phase);
    phase ^= 1;
    tc_fence_after();
    float y[16];
    tmem_ld16(tlane + TC_DF, y);
    tmem_wait_ld();
    if (!ok) *flag = 1;
    if (valid && ok) {
      if (SRC == 0) {
#pragma unroll
        for (int q = 0; q < SGS_NOUT; q++) Y[row * SGS_NOUT + q] = nm.out_mu[q] + nm.out_sig[q] * (y[q] + bias[192 + q]);
      } else {
        const bool sfc = P.surf > 0 && k == P.kMin && i >= P.iMin && j >= P.jMin;
#pragma unroll
        for (int q = 0; q < SGS_NOUT; q++) {
          if (sfc && (q == 2 || q == 3 || q == 8)) continue;
          Q.tau[q * P.n + c] = rho * (nm.out_mu[q] + nm.out_sig[q] * (y[q] + bias[192 + q]));
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    if (*flag) break;
  }
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && *flag) atomicExch(err, 1);
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, TM_INFER_COLS);
  }
}

// ------------------------------------------------------------------ training
// Gradient of L = sum over samples [first, first+count) and the 9 outputs of (y - t)^2,
// t = (T/1 - out_mu)/out_sig, divided by count*9; accumulated into grad[] (FP32 atomics) and
// the loss into loss[0] (FP64 atomic). `order` (optional) maps sample slots to rows of X/T.
__global__ void __launch_bounds__(128, 1) k_mlp_train(const float* __restrict__ params, const MlpNorm* __restrict__ nmp,
                                                      const float* __restrict__ X, const float* __restrict__ T,
                                                      const int* __restrict__ order, long long nrows, long long first,
                                                      long long count, float* __restrict__ grad, double* __restrict__ loss,
                                                      int* __restrict__ err) {
  using S = MlpTrainSmem;
  extern __shared__ __align__(1024) char sm[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + S::BAR);
  uint32_t* taddrSlot = reinterpret_cast<uint32_t*>(sm + S::TADDR);
  float* bias = reinterpret_cast<float*>(sm + S::BIAS);
  double* red = reinterpret_cast<double*>(sm + S::RED);
  int* flag = reinterpret_cast<int*>(sm + S::FLAG);
  MlpNorm& nm = *reinterpret_cast<MlpNorm*>(sm + S::NORM);
  if (tid < 64) reinterpret_cast<float*>(&nm)[tid] = reinterpret_cast<const float*>(nmp)[tid];
  float* isig = reinterpret_cast<float*>(sm + S::ISIG);
  stage_isig(nmp, isig, tid);
  stage_weight(params + MP_W1, 64, 16, sm + S::W1, nullptr, tid, 128);
  stage_weight(params + MP_W2, 64, 64, sm + S::W2, sm + S::W2T, tid, 128);
  stage_weight(params + MP_W3, 64, 64, sm + S::W3, sm + S::W3T, tid, 128);
  stage_weight(params + MP_W4, 16, 64, sm + S::W4, sm + S::W4T, tid, 128);
  for (int e = tid; e < 64; e += 128) {
    bias[e] = params[MP_B1 + e];
    bias[64 + e] = params[MP_B2 + e];
    bias[128 + e] = params[MP_B3 + e];
  }
  if (tid < 16) bias[192 + tid] = params[MP_B4 + tid];
  // rows 64..127 of the transposed-activation tile: a row of ones (bias gradient), then zeros
  for (int e = tid; e < 64 * 128; e += 128) {
    const int r = 64 + e / 128, b = e % 128;
    st_elem(sm + S::ATH, r, b, 128, r == 64 ? 1.0f : 0.0f);
  }
  if (tid == 0) { mbar_init(bar); *flag = 0; }
  if (warp == 0) tmem_alloc(taddrSlot, TM_TRAIN_COLS);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *taddrSlot;
  const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  const uint32_t id64 = umma_idesc(128, 64), id16 = umma_idesc(128, 16);
  const long long ntiles = (count + MLP_M - 1) / MLP_M;
  const float gscale = 1.0f;  // dZ4 = 2 (y - t); the 1/(count*9) is applied at the flush
  double lsum = 0.0;
  bool firstTile = true;
  bool ok = true;

  auto mma_wait = [&]() {
    ok = ok && mbar_wait(bar, phase);
    if (!ok) *flag = 1;
    phase ^= 1;
    tc_fence_after();
  };

  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long slot = tile * MLP_M + tid;
    const bool valid = slot < count;
    long long row = 0;
    if (valid) {
      row = (first + slot) % nrows;
      if (order) row = order[row];
    }
    float x[SGS_NIN];
#pragma unroll
    for (int q = 0; q < SGS_NIN; q++) x[q] = valid ? X[row * SGS_NIN + q] : 0.0f;
    put_inputs(sm + S::X0, tid, x, nm, isig, valid);
    sync_for_mma();
    // ---- forward
    if (tid == 0) {
      tc_fence_after();
      umma_bf16(tbase + TC_DF, umma_sdesc(sm + S::X0, 128, 256), umma_sdesc(sm + S::W1, 128, 256), id64, 0);
      umma_commit(bar);
    }
    mma_wait();
    epi_tanh<false>(tlane + TC_DF, bias, sm + S::H1, tid);
    sync_for_mma();
#pragma unroll 1
    for (int l = 0; l < 2; l++) {
      const char* hin = sm + (l == 0 ? S::H1 : S::H2);
      const char* w = sm + (l == 0 ? S::W2 : S::W3);
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < 4; s++)
          umma_bf16(tbase + TC_DF, umma_sdesc(hin + s * 256, 128, 1024), umma_sdesc(w + s * 256, 128, 1024), id64, s > 0);
        umma_commit(bar);
      }
      mma_wait();
      epi_tanh<false>(tlane + TC_DF, bias + 64 * (l + 1), sm + (l == 0 ? S::H2 : S::H3), tid);
      sync_for_mma();
    }
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < 4; s++)
        umma_bf16(tbase + TC_DF, umma_sdesc(sm + S::H3 + s * 256, 128, 1024), umma_sdesc(sm + S::W4 + s * 256, 128, 1024),
                  id16, s > 0);
      umma_commit(bar);
    }
    mma_wait();
    float dz[64];
    {
      float y[16];
      tmem_ld16(tlane + TC_DF, y);
      tmem_wait_ld();
#pragma unroll
      for (int q = 0; q < 16; q++) {
        float e = 0.0f;
        if (valid && q < SGS_NOUT) {
          const float t = (T[row * SGS_NOUT + q] - nm.out_mu[q]) / nm.out_sig[q];
          e = (y[q] + bias[192 + q]) - t;
          lsum += (double)e * (double)e;
        }
        dz[q] = gscale * 2.0f * e;
      }
    }
    // ---- backward, layer 4: dZ4 (K = 16) and its transpose; [H3^T; 1]
    st_chunk(sm + S::DZK, tid, 0, 16, dz);
    st_chunk(sm + S::DZK, tid, 1, 16, dz + 8);
#pragma unroll
    for (int q = 0; q < 16; q++) st_elem(sm + S::DZT, q, tid, 128, dz[q]);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      float h[8];
      ld_chunk(sm + S::H3, tid, q, 64, h);
#pragma unroll
      for (int t = 0; t < 8; t++) st_elem(sm + S::ATH, q * 8 + t, tid, 128, h[t]);
    }
    sync_for_mma();
    if (tid == 0) {
      tc_fence_after();
      umma_bf16(tbase + TC_DB, umma_sdesc(sm + S::DZK, 128, 256), umma_sdesc(sm + S::W4T, 128, 256), id64, 0);
#pragma unroll
      for (int s = 0; s < 8; s++)
        umma_bf16(tbase + TC_G4, umma_sdesc(sm + S::ATH + s * 256, 128, 2048), umma_sdesc(sm + S::DZT + s * 256, 128, 2048),
                  id16, (firstTile && s == 0) ? 0u : 1u);
      umma_commit(bar);
    }
    mma_wait();
    // ---- layers 3, 2, 1
#pragma unroll 1
    for (int l = 3; l >= 1; l--) {
      const char* hl = sm + (l == 3 ? S::H3 : (l == 2 ? S::H2 : S::H1));  // activation whose dZ this is
      // dZ(l) = dH(l) * (1 - h(l)^2)
#pragma unroll
      for (int g = 0; g < 4; g++) {
        float v[16];
        tmem_ld16(tlane + TC_DB + g * 16, v);
        tmem_wait_ld();
        float h[16];
        ld_chunk(hl, tid, 2 * g, 64, h);
        ld_chunk(hl, tid, 2 * g + 1, 64, h + 8);
#pragma unroll
        for (int q = 0; q < 16; q++) dz[g * 16 + q] = v[q] * (1.0f - h[q] * h[q]);
      }
      if (l > 1) {
#pragma unroll
        for (int q = 0; q < 8; q++) st_chunk(sm + S::DZK, tid, q, 64, dz + 8 * q);
      }
#pragma unroll
      for (int q = 0; q < 64; q++) st_elem(sm + S::DZT, q, tid, 128, dz[q]);
      // [H(l-1)^T; 1]: H2, H1 or the inputs
      if (l > 1) {
        const char* hp = sm + (l == 3 ? S::H2 : S::H1);
#pragma unroll
        for (int q = 0; q < 8; q++) {
          float h[8];
          ld_chunk(hp, tid, q, 64, h);
#pragma unroll
          for (int t = 0; t < 8; t++) st_elem(sm + S::ATH, q * 8 + t, tid, 128, h[t]);
        }
      } else {
#pragma unroll
        for (int q = 0; q < 2; q++) {
          float h[8];
          ld_chunk(sm + S::X0, tid, q, 16, h);
#pragma unroll
          for (int t = 0; t < 8; t++) st_elem(sm + S::ATH, q * 8 + t, tid, 128, h[t]);
        }
      }
      sync_for_mma();
      if (tid == 0) {
        tc_fence_after();
        if (l > 1) {
          const char* wt = sm + (l == 3 ? S::W3T : S::W2T);
#pragma unroll
          for (int s = 0; s < 4; s++)
            umma_bf16(tbase + TC_DB, umma_sdesc(sm + S::DZK + s * 256, 128, 1024), umma_sdesc(wt + s * 256, 128, 1024), id64,
                      s > 0);
        }
        const uint32_t g = tbase + (l == 3 ? TC_G3 : (l == 2 ? TC_G2 : TC_G1));
#pragma unroll
        for (int s = 0; s < 8; s++)
          umma_bf16(g, umma_sdesc(sm + S::ATH + s * 256, 128, 2048), umma_sdesc(sm + S::DZT + s * 256, 128, 2048), id64,
                    (firstTile && s == 0) ? 0u : 1u);
        umma_commit(bar);
      }
      mma_wait();
    }
    firstTile = false;
    tc_fence_before();
    __syncthreads();
    if (*flag) break;
  }
  // ---- flush: rows r < K_in of G(l) hold dW(l)[c][r], row 64 the bias gradient
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const bool anyTile = !firstTile;
  if (*flag == 0 && anyTile && warp < 3) {
    const float inv = 1.0f / ((float)count * (float)SGS_NOUT);
    const int r = tid;
    const bool isB = (r == 64), isW = r < 64;
    // layer 4 (16 columns, 9 used)
    {
      float v[16];
      tmem_ld16(tlane + TC_G4, v);
      tmem_wait_ld();
      if (isW || isB)
        for (int c = 0; c < SGS_NOUT; c++) atomicAdd(&grad[isB ? MP_B4 + c : MP_W4 + c * 64 + r], v[c] * inv);
    }
#pragma unroll 1
    for (int l = 3; l >= 1; l--) {
      const uint32_t g = tlane + (l == 3 ? TC_G3 : (l == 2 ? TC_G2 : TC_G1));
      const int kin = l == 1 ? 16 : 64;
      const int wofs = l == 3 ? MP_W3 : (l == 2 ? MP_W2 : MP_W1), bofs = l == 3 ? MP_B3 : (l == 2 ? MP_B2 : MP_B1);
      for (int gq = 0; gq < 4; gq++) {
        float v[16];
        tmem_ld16(g + gq * 16, v);
        tmem_wait_ld();
        const bool useW = isW && r < (l == 1 ? SGS_NIN : 64);
        if (useW || isB)
          for (int q = 0; q < 16; q++) {
            const int c = gq * 16 + q;
            atomicAdd(&grad[isB ? bofs + c : wofs + c * kin + r], v[q] * inv);
          }
      }
    }
  }
  // loss
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if (lane == 0) red[warp] = lsum;
  tc_fence_before();
  __syncthreads();
  if (tid == 0) {
    const double s = red[0] + red[1] + red[2] + red[3];
    if (s != 0.0) atomicAdd(loss, s / ((double)count * SGS_NOUT));
    if (*flag) atomicExch(err, 1);
  }
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, TM_TRAIN_COLS);
  }
}

// Adam on the FP32 master parameters; padded entries (W1 columns >= 11, W4 rows and b4
// entries >= 9) stay zero.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= MP_TOTAL) return;
  bool pad = false;
  if (e < MP_B1) pad = (e % MLP_K0) >= SGS_NIN;
  else if (e >= MP_W4 && e < MP_B4) pad = ((e - MP_W4) / MLP_H) >= SGS_NOUT;
  else if (e >= MP_B4) pad = (e - MP_B4) >= SGS_NOUT;
  if (pad) { p[e] = 0.0f; return; }
  const float gi = g[e];
  const float mi = b1 * m[e] + (1.0f - b1) * gi;
  const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
  m[e] = mi;
  v[e] = vi;
  p[e] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace fe
