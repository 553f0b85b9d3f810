// Learned proposal network: training-data features, inference, training
// (forward + backward on the tensor cores) and the Adam update.
//
// Training step of one CTA (128 rows, thread t = row t = TMEM lane t):
//   forward   X0 -> H1 -> H2 -> H3 -> out (4 MMA chains into TMEM columns
//             [0,128)), keeping H_l^T (features x rows, K-major) in shared
//             memory for the weight gradients and the ReLU masks in
//             registers;
//   loss      NLL of the target displacement under the output mixture and
//             dL/dout (FP32), scaled by 1/R_total;
//   backward  for l = 4..1: dH_{l-1} = dZ_l W_l (A = dZ_l, B = W_l^T) into
//             columns [0,128) and dW_l^T = H_{l-1}^T dZ_l (A = H^T,
//             B = dZ_l^T) into columns [128,256) (layer 1: dW_1 = dZ_1^T X0);
//             dZ_{l-1} = dH_{l-1} * ReLU'(Z_{l-1}) overwrites H_{l-1}^T in
//             place once its MMA has read it; bias gradients are the row sums
//             of dZ^T.  Gradients are added to the global FP32 buffer with
//             atomics (one add per parameter per CTA).
// Every MMA operand is BF16 (as the oracle emulates), every accumulation
// FP32.  Waits on the MMA mbarrier are bounded; a timeout sets
// OQ_FLAG_TIMEOUT, stops the CTA's work and frees its TMEM.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "oqmc_mlp.cuh"
#include "oqmc_ctx.h"
#include "oqmc_mlp_host.h"
#include "../../include/oqmc_b200.h"

// training smem map (bytes)
#define TR_ACT 0
#define TR_HT0 32768
#define TR_HT1 40960
#define TR_HT2 73728
#define TR_HT3 106496
#define TR_W 139264
#define TR_BIAS (TR_W + OQ_MLP_SM_WEIGHTS)
#define TR_BAR (TR_BIAS + OQ_MLP_SM_BIAS)
#define TR_SMEM (TR_BAR + 64)
// forward-only smem map
#define FW_ACT 0
#define FW_W 32768
#define FW_BIAS (FW_W + OQ_MLP_SM_WEIGHTS)
#define FW_BAR (FW_BIAS + OQ_MLP_SM_BIAS)
#define FW_SMEM (FW_BAR + 64)

static_assert(TR_SMEM <= 232448, "training tile exceeds shared memory");

// Sum of row n (128 BF16 values) of a [rows x 128] K-major buffer.
__device__ __forceinline__ float oq_mlp_rowsum(const unsigned char* buf, int n) {
  float s = 0.0f;
#pragma unroll 4
  for (int c = 0; c < 16; ++c) {
    const uint4 q = *reinterpret_cast<const uint4*>(buf + (((n >> 3) * 16 + c) << 7) + ((n & 7) << 4));
    s += oq_bf16_lo(q.x) + oq_bf16_hi(q.x) + oq_bf16_lo(q.y) + oq_bf16_hi(q.y) +
         oq_bf16_lo(q.z) + oq_bf16_hi(q.z) + oq_bf16_lo(q.w) + oq_bf16_hi(q.w);
  }
  return s;
}

// dZ = dH (TMEM row r) * ReLU mask; BF16 into act (KC = 16, may be null) and
// transposed into ht.
__device__ __forceinline__ void oq_mlp_dz_epilogue(uint32_t trow, const uint32_t* mask,
                                                   unsigned char* act, int r, unsigned char* ht) {
#pragma unroll 1
  for (int c0 = 0; c0 < OQ_MLP_H; c0 += 16) {
    float v[16];
    oq_tmem_ld16(trow + (uint32_t)c0, v);
    const uint32_t mb = mask[c0 >> 5] >> (c0 & 16);
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = ((mb >> j) & 1u) ? v[j] : 0.0f;
    if (act) oq_mlp_store_row16(act, r, c0, 16, v);
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const uint32_t p = oq_bf16x2(v[j], v[j + 1]);
      *reinterpret_cast<unsigned short*>(ht + oq_kmajor_off2(c0 + j, r, 16)) =
          (unsigned short)(p & 0xFFFFu);
      *reinterpret_cast<unsigned short*>(ht + oq_kmajor_off2(c0 + j + 1, r, 16)) =
          (unsigned short)(p >> 16);
    }
  }
}

// Read ncol columns of TMEM row r (a weight-gradient row) and add them to
// grad[base + col * stride].
__device__ __forceinline__ void oq_mlp_flush_grad(uint32_t trow, int ncol, float* grad,
                                                  int base, int stride) {
#pragma unroll 1
  for (int c0 = 0; c0 < ncol; c0 += 16) {
    float v[16];
    oq_tmem_ld16(trow + (uint32_t)c0, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) atomicAdd(grad + base + (c0 + j) * stride, v[j]);
  }
}

__global__ void __launch_bounds__(128, 1)
k_mlp_train(const unsigned short* __restrict__ feat, const float* __restrict__ target, int R,
            float scale, const unsigned short* __restrict__ wbf,
            const unsigned short* __restrict__ wtbf, const float* __restrict__ theta,
            float* __restrict__ grad, double* __restrict__ loss_sum, unsigned* flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* act = smem + TR_ACT;
  unsigned char* ht0 = smem + TR_HT0;
  unsigned char* ht1 = smem + TR_HT1;
  unsigned char* ht2 = smem + TR_HT2;
  unsigned char* ht3 = smem + TR_HT3;
  unsigned char* wreg = smem + TR_W;
  unsigned char* z4t = wreg + 32768;
  float* bias = reinterpret_cast<float*>(smem + TR_BIAS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + TR_BAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + TR_BAR + 8);
  const int t = threadIdx.x, warp = t >> 5;
  const int row = blockIdx.x * 128 + t;
  const bool valid = row < R;
  if (warp == 0) oq_tmem_alloc(slot, 256);
  if (t == 0) oq_mbar_init(bar, 1);
  {
    uint4 q[4] = {};
    if (valid) {
      const uint4* s = reinterpret_cast<const uint4*>(feat + (size_t)row * OQ_MLP_K0);
      for (int k = 0; k < 4; ++k) q[k] = s[k];
    }
    for (int c = 0; c < 4; ++c)
      *reinterpret_cast<uint4*>(act + (((t >> 3) * 4 + c) << 7) + ((t & 7) << 4)) = q[c];
    const unsigned short* h = reinterpret_cast<const unsigned short*>(q);
    for (int k = 0; k < OQ_MLP_K0; ++k)
      *reinterpret_cast<unsigned short*>(ht0 + oq_kmajor_off2(k, t, 16)) = h[k];
  }
  float dtg[3] = {0.0f, 0.0f, 0.0f};
  if (valid) {
    dtg[0] = target[(size_t)row * 3];
    dtg[1] = target[(size_t)row * 3 + 1];
    dtg[2] = target[(size_t)row * 3 + 2];
  }
  oq_mlp_load_weights(wreg, wbf);
  oq_mlp_load_bias(bias, theta);
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
  const uint32_t tmem = *slot;
  const uint32_t lane = (uint32_t)(warp * 32) << 16;
  const uint32_t t1 = tmem + lane, t2 = tmem + 128 + lane;
  OqMlpSync sy{bar, 0u};
  uint32_t mask[12];
  for (int i = 0; i < 12; ++i) mask[i] = 0u;
  float out[OQ_MLP_NOUT];
  unsigned char* hts[3] = {ht1, ht2, ht3};
  bool ok = oq_mlp_forward_tile(act, wreg, bias, tmem, sy, out, hts, mask);
  if (ok) {
    float g[OQ_MLP_NOUT];
    double nl = 0.0;
    if (valid) {
      nl = oq_mix_nll_grad(out, dtg, scale, g);
    } else {
      for (int j = 0; j < OQ_MLP_NOUT; ++j) g[j] = 0.0f;
    }
    double s = nl;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((t & 31) == 0 && loss_sum) atomicAdd(loss_sum, s);
    // dZ4 (rows x 48) and its transpose; W4^T into the weight region
    for (int c0 = 0; c0 < OQ_MLP_NOUT; c0 += 16) oq_mlp_store_row16(act, t, c0, 6, g + c0);
    for (int j = 0; j < OQ_MLP_NOUT; j += 2) {
      const uint32_t p = oq_bf16x2(g[j], g[j + 1]);
      *reinterpret_cast<unsigned short*>(z4t + oq_kmajor_off2(j, t, 16)) = (unsigned short)(p & 0xFFFFu);
      *reinterpret_cast<unsigned short*>(z4t + oq_kmajor_off2(j + 1, t, 16)) = (unsigned short)(p >> 16);
    }
    oq_mlp_load_kmajor(wreg, wtbf + OQ_MLP_OFF_W4, OQ_MLP_H, OQ_MLP_NOUT);
    oq_mlp_pre_issue();
    if (t == 0) {
      const uint32_t a0 = oq_smem_addr(act), b0 = oq_smem_addr(wreg);
      for (int ks = 0; ks < OQ_MLP_NOUT / 16; ++ks)
        oq_mma_bf16(tmem, oq_desc_kmajor(a0 + ks * 256u, 128u, 6u * 128u),
                    oq_desc_kmajor(b0 + ks * 256u, 128u, 6u * 128u), oq_idesc_bf16(128, 128),
                    ks > 0 ? 1u : 0u);
      const uint32_t h0 = oq_smem_addr(ht3), z0 = oq_smem_addr(z4t);
      for (int ks = 0; ks < 8; ++ks)
        oq_mma_bf16(tmem + 128, oq_desc_kmajor(h0 + ks * 256u, 128u, 2048u),
                    oq_desc_kmajor(z0 + ks * 256u, 128u, 2048u), oq_idesc_bf16(128, OQ_MLP_NOUT),
                    ks > 0 ? 1u : 0u);
      oq_mma_commit(bar);
    }
    ok = oq_mlp_wait(sy);
  }
  if (ok) {
    if (t < OQ_MLP_NOUT) {
      // row t of dZ4^T, 128 rows of the tile
      float sb = 0.0f;
      for (int c = 0; c < 16; ++c) {
        const uint4 q = *reinterpret_cast<const uint4*>(z4t + (((t >> 3) * 16 + c) << 7) + ((t & 7) << 4));
        sb += oq_bf16_lo(q.x) + oq_bf16_hi(q.x) + oq_bf16_lo(q.y) + oq_bf16_hi(q.y) +
              oq_bf16_lo(q.z) + oq_bf16_hi(q.z) + oq_bf16_lo(q.w) + oq_bf16_hi(q.w);
      }
      atomicAdd(grad + OQ_MLP_OFF_B4 + t, sb);
    }
    oq_mlp_flush_grad(t2, OQ_MLP_NOUT, grad, OQ_MLP_OFF_W4 + t, OQ_MLP_H);   // dW4[n][t]
    oq_mlp_dz_epilogue(t1, mask + 8, act, t, ht3);                          // dZ3
    oq_tc_fence_before();
    __syncthreads();
    oq_mlp_load_kmajor(wreg, wtbf + OQ_MLP_OFF_W3, OQ_MLP_H, OQ_MLP_H);
    oq_mlp_pre_issue();
    if (t == 0) {
      oq_mlp_mma(tmem, act, wreg, OQ_MLP_H, OQ_MLP_H, nullptr);
      oq_mlp_mma(tmem + 128, ht2, ht3, OQ_MLP_H, OQ_MLP_H, bar);
    }
    ok = oq_mlp_wait(sy);
  }
  if (ok) {
    atomicAdd(grad + OQ_MLP_OFF_B3 + t, oq_mlp_rowsum(ht3, t));
    oq_mlp_flush_grad(t2, OQ_MLP_H, grad, OQ_MLP_OFF_W3 + t, OQ_MLP_H);
    oq_mlp_dz_epilogue(t1, mask + 4, act, t, ht2);                          // dZ2
    oq_tc_fence_before();
    __syncthreads();
    oq_mlp_load_kmajor(wreg, wtbf + OQ_MLP_OFF_W2, OQ_MLP_H, OQ_MLP_H);
    oq_mlp_pre_issue();
    if (t == 0) {
      oq_mlp_mma(tmem, act, wreg, OQ_MLP_H, OQ_MLP_H, nullptr);
      oq_mlp_mma(tmem + 128, ht1, ht2, OQ_MLP_H, OQ_MLP_H, bar);
    }
    ok = oq_mlp_wait(sy);
  }
  if (ok) {
    atomicAdd(grad + OQ_MLP_OFF_B2 + t, oq_mlp_rowsum(ht2, t));
    oq_mlp_flush_grad(t2, OQ_MLP_H, grad, OQ_MLP_OFF_W2 + t, OQ_MLP_H);
    oq_mlp_dz_epilogue(t1, mask, nullptr, t, ht1);                          // dZ1^T
    oq_mlp_pre_issue();
    if (t == 0) oq_mlp_mma(tmem, ht1, ht0, OQ_MLP_K0, OQ_MLP_H, bar);       // dW1 [128 x 32]
    ok = oq_mlp_wait(sy);
  }
  if (ok) {
    atomicAdd(grad + OQ_MLP_OFF_B1 + t, oq_mlp_rowsum(ht1, t));
    oq_mlp_flush_grad(t1, OQ_MLP_K0, grad, OQ_MLP_OFF_W1 + t * OQ_MLP_K0, 1);
  }
  oq_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    oq_tc_fence_after();
    if (!ok) oq_mbar_wait(bar, sy.phase ^ 1u);   // let an outstanding MMA drain
    oq_tmem_dealloc(tmem, 256);
  }
  if (!ok && t == 0) atomicOr(flags, OQ_FLAG_TIMEOUT);
}

__global__ void __launch_bounds__(128, 1)
k_mlp_forward(const unsigned short* __restrict__ feat, int R,
              const unsigned short* __restrict__ wbf, const float* __restrict__ theta,
              float* __restrict__ out_g, unsigned* flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* act = smem + FW_ACT;
  unsigned char* wreg = smem + FW_W;
  float* bias = reinterpret_cast<float*>(smem + FW_BIAS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + FW_BAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + FW_BAR + 8);
  const int t = threadIdx.x, warp = t >> 5;
  const int row = blockIdx.x * 128 + t;
  const bool valid = row < R;
  (void)act;
  // TMEM: accumulator in columns [0, 128), BF16 activations in [128, 192)
  if (warp == 0) oq_tmem_alloc(slot, 256);
  if (t == 0) oq_mbar_init(bar, 1);
  oq_mlp_load_weights(wreg, wbf);
  oq_mlp_load_bias(bias, theta);
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
  const uint32_t tmem = *slot;
  {
    uint32_t f2[16] = {};
    if (valid) {
      const uint4* s = reinterpret_cast<const uint4*>(feat + (size_t)row * OQ_MLP_K0);
      for (int k = 0; k < 4; ++k) {
        const uint4 q = s[k];
        f2[4 * k] = q.x; f2[4 * k + 1] = q.y; f2[4 * k + 2] = q.z; f2[4 * k + 3] = q.w;
      }
    }
    oq_mlp_store_features_ta(tmem + ((uint32_t)((t >> 5) * 32) << 16), f2);
    oq_tmem_wait_st();
  }
  OqMlpSync sy{bar, 0u};
  float out[OQ_MLP_NOUT];
  const bool ok = oq_mlp_forward_tile_ta(wreg, bias, tmem, sy, out);
  if (ok && valid)
    for (int j = 0; j < OQ_MLP_NOUT; ++j) out_g[(size_t)row * OQ_MLP_NOUT + j] = out[j];
  oq_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    oq_tc_fence_after();
    if (!ok) oq_mbar_wait(bar, sy.phase ^ 1u);
    oq_tmem_dealloc(tmem, 256);
  }
  if (!ok && t == 0) atomicOr(flags, OQ_FLAG_TIMEOUT);
}

// Features of every (walker, electron) row (row = w * n_e + e) of walkers X0
// (W, n_e, 3) and, when X1 is given, the displacement X1 - X0 as the target.
__global__ void k_mlp_features(const OqSystem* __restrict__ S, const double* __restrict__ X0,
                               const double* __restrict__ X1, int W, int ne,
                               unsigned short* __restrict__ feat, float* __restrict__ target) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= W * ne) return;
  const int w = q / ne, e = q - w * ne;
  const double* x = X0 + (size_t)w * ne * 3;
  auto P = [&](int j, int c) { return x[j * 3 + c]; };
  float f[OQ_MLP_K0];
  oq_mlp_features(*S, P, ne, e, x[e * 3], x[e * 3 + 1], x[e * 3 + 2], f);
  uint4* dst = reinterpret_cast<uint4*>(feat + (size_t)q * OQ_MLP_K0);
  for (int k = 0; k < 4; ++k) {
    uint4 v;
    v.x = oq_bf16x2(f[8 * k], f[8 * k + 1]);
    v.y = oq_bf16x2(f[8 * k + 2], f[8 * k + 3]);
    v.z = oq_bf16x2(f[8 * k + 4], f[8 * k + 5]);
    v.w = oq_bf16x2(f[8 * k + 6], f[8 * k + 7]);
    dst[k] = v;
  }
  if (X1 && target) {
    const double* y = X1 + (size_t)w * ne * 3;
    for (int c = 0; c < 3; ++c) target[(size_t)q * 3 + c] = (float)(y[e * 3 + c] - x[e * 3 + c]);
  }
}

// Layer, row, column and fan-out of a weight entry (false for biases).
__device__ __forceinline__ bool oq_mlp_weight_of(int i, int& off, int& n, int& k, int& N, int& K) {
  if (i < OQ_MLP_OFF_B1) { off = OQ_MLP_OFF_W1; N = OQ_MLP_H; K = OQ_MLP_K0; }
  else if (i >= OQ_MLP_OFF_W2 && i < OQ_MLP_OFF_B2) { off = OQ_MLP_OFF_W2; N = OQ_MLP_H; K = OQ_MLP_H; }
  else if (i >= OQ_MLP_OFF_W3 && i < OQ_MLP_OFF_B3) { off = OQ_MLP_OFF_W3; N = OQ_MLP_H; K = OQ_MLP_H; }
  else if (i >= OQ_MLP_OFF_W4 && i < OQ_MLP_OFF_B4) { off = OQ_MLP_OFF_W4; N = OQ_MLP_NOUT; K = OQ_MLP_H; }
  else return false;
  n = (i - off) / K;
  k = (i - off) - n * K;
  return true;
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; lr = 0 only
// refreshes the BF16 copies.  Gradients are cleared for the next step.
__global__ void k_mlp_adam(float* __restrict__ theta, float* __restrict__ m, float* __restrict__ v,
                           float* __restrict__ grad, unsigned short* __restrict__ wbf,
                           unsigned short* __restrict__ wtbf, float lr, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= OQ_MLP_NPARAM) return;
  float p = theta[i];
  if (lr > 0.0f) {
    const float gi = grad[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    theta[i] = p;
  }
  grad[i] = 0.0f;
  int off, n, k, N, K;
  if (oq_mlp_weight_of(i, off, n, k, N, K)) {
    const unsigned short b = (unsigned short)(oq_bf16x2(p, 0.0f) & 0xFFFFu);
    wbf[i] = b;
    wtbf[off + k * N + n] = b;
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static thread_local char g_mlp_err[512] = "";

static int merr(oqmc_mlp* m, int code, const std::string& msg) {
  snprintf(m ? m->err : g_mlp_err, 512, "%s", msg.c_str());
  return code;
}

#define OQ_MCUDA(m, call)                                                                \
  do {                                                                                   \
    cudaError_t _e = (call);                                                             \
    if (_e != cudaSuccess) return merr(m, OQ_ERR_CUDA, std::string("CUDA error: ") +    \
                                                           cudaGetErrorString(_e));      \
  } while (0)

static int cast_weights(oqmc_mlp* m, cudaStream_t s) {
  k_mlp_adam<<<(OQ_MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->theta, m->m, m->v, m->grad, m->wbf,
                                                         m->wtbf, 0.0f, 1.0f, 1.0f);
  OQ_MCUDA(m, cudaGetLastError());
  return OQ_OK;
}

static int train_kernel(oqmc_mlp* m, const unsigned short* feat, const float* target, int R,
                        float* grad, double* loss, cudaStream_t s) {
  static bool attr = false;
  if (!attr) {
    OQ_MCUDA(m, cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     TR_SMEM));
    attr = true;
  }
  k_mlp_train<<<(R + 127) / 128, 128, TR_SMEM, s>>>(feat, target, R, 1.0f / (float)R, m->wbf,
                                                    m->wtbf, m->theta, grad, loss, m->d_flags);
  OQ_MCUDA(m, cudaGetLastError());
  return OQ_OK;
}

int oq_mlp_check_flags(oqmc_mlp* m, cudaStream_t s) {
  unsigned f = 0;
  OQ_MCUDA(m, cudaMemcpyAsync(&f, m->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  OQ_MCUDA(m, cudaStreamSynchronize(s));
  if (f & OQ_FLAG_TIMEOUT) return merr(m, OQ_ERR_TIMEOUT, "tensor-core wait timed out");
  return OQ_OK;
}

extern "C" {

const char* oqmc_mlp_last_error(const oqmc_mlp* m) { return m ? m->err : g_mlp_err; }

int oqmc_mlp_destroy(oqmc_mlp* m) {
  if (!m) return OQ_OK;
  cudaFree(m->theta);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->grad);
  cudaFree(m->wbf);
  cudaFree(m->wtbf);
  cudaFree(m->d_flags);
  delete m;
  return OQ_OK;
}

int oqmc_mlp_create(oqmc_mlp** out, uint64_t seed) {
  if (!out) return merr(nullptr, OQ_ERR_ARG, "null argument");
  *out = nullptr;
  oqmc_mlp* m = new oqmc_mlp();
  cudaGetDevice(&m->device);
  const size_t nb = OQ_MLP_NPARAM * sizeof(float);
  cudaError_t e = cudaMalloc(&m->theta, nb);
  e = e == cudaSuccess ? cudaMalloc(&m->m, nb) : e;
  e = e == cudaSuccess ? cudaMalloc(&m->v, nb) : e;
  e = e == cudaSuccess ? cudaMalloc(&m->grad, nb) : e;
  e = e == cudaSuccess ? cudaMalloc(&m->wbf, OQ_MLP_NPARAM * 2) : e;
  e = e == cudaSuccess ? cudaMalloc(&m->wtbf, OQ_MLP_NPARAM * 2) : e;
  e = e == cudaSuccess ? cudaMalloc(&m->d_flags, sizeof(unsigned)) : e;
  if (e != cudaSuccess) {
    oqmc_mlp_destroy(m);
    return merr(nullptr, OQ_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
  }
  // He-uniform hidden layers, output layer scaled by 0.1 (splitmix64 stream)
  std::vector<float> th(OQ_MLP_NPARAM, 0.0f);
  uint64_t st = seed;
  auto uni = [&]() {
    st += 0x9E3779B97F4A7C15ull;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  struct Blk { int off, n, fan; double gain; };
  const Blk blk[4] = {{OQ_MLP_OFF_W1, OQ_MLP_H * OQ_MLP_K0, OQ_MLP_K0, 1.0},
                      {OQ_MLP_OFF_W2, OQ_MLP_H * OQ_MLP_H, OQ_MLP_H, 1.0},
                      {OQ_MLP_OFF_W3, OQ_MLP_H * OQ_MLP_H, OQ_MLP_H, 1.0},
                      {OQ_MLP_OFF_W4, OQ_MLP_NOUT * OQ_MLP_H, OQ_MLP_H, 0.1}};
  for (const Blk& b : blk) {
    const double lim = sqrt(6.0 / b.fan) * b.gain;
    for (int i = 0; i < b.n; ++i) th[b.off + i] = (float)((2.0 * uni() - 1.0) * lim);
  }
  e = cudaMemcpy(m->theta, th.data(), nb, cudaMemcpyHostToDevice);
  e = e == cudaSuccess ? cudaMemset(m->m, 0, nb) : e;
  e = e == cudaSuccess ? cudaMemset(m->v, 0, nb) : e;
  e = e == cudaSuccess ? cudaMemset(m->grad, 0, nb) : e;
  e = e == cudaSuccess ? cudaMemset(m->d_flags, 0, sizeof(unsigned)) : e;
  if (e != cudaSuccess) {
    oqmc_mlp_destroy(m);
    return merr(nullptr, OQ_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e));
  }
  if (cast_weights(m, 0) != OQ_OK || cudaDeviceSynchronize() != cudaSuccess) {
    oqmc_mlp_destroy(m);
    return merr(nullptr, OQ_ERR_CUDA, "weight cast failed");
  }
  *out = m;
  return OQ_OK;
}

int oqmc_mlp_get_params(oqmc_mlp* m, float* theta_host) {
  if (!m || !theta_host) return merr(m, OQ_ERR_ARG, "null argument");
  OQ_MCUDA(m, cudaMemcpy(theta_host, m->theta, OQ_MLP_NPARAM * sizeof(float),
                         cudaMemcpyDeviceToHost));
  return OQ_OK;
}

int oqmc_mlp_set_params(oqmc_mlp* m, const float* theta_host) {
  if (!m || !theta_host) return merr(m, OQ_ERR_ARG, "null argument");
  OQ_MCUDA(m, cudaMemcpy(m->theta, theta_host, OQ_MLP_NPARAM * sizeof(float),
                         cudaMemcpyHostToDevice));
  OQ_MCUDA(m, cudaMemset(m->m, 0, OQ_MLP_NPARAM * sizeof(float)));
  OQ_MCUDA(m, cudaMemset(m->v, 0, OQ_MLP_NPARAM * sizeof(float)));
  m->t = 0;
  const int rc = cast_weights(m, 0);
  if (rc != OQ_OK) return rc;
  OQ_MCUDA(m, cudaDeviceSynchronize());
  return OQ_OK;
}

int oqmc_mlp_num_params(void) { return OQ_MLP_NPARAM; }

int oqmc_mlp_features(oqmc_ctx* ctx, const double* X0, const double* X1, int W,
                      unsigned short* feat, float* target, void* stream) {
  if (!ctx || W < 0 || (W > 0 && (!X0 || !feat)) || (X1 && !target))
    return oq_ctx_set_error(ctx, OQ_ERR_ARG, "bad arguments");
  if (ctx->n_e > 32) return oq_ctx_set_error(ctx, OQ_ERR_UNSUPPORTED, "more than 32 electrons");
  if (W == 0) return OQ_OK;
  const int rows = W * ctx->n_e;
  k_mlp_features<<<(rows + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
      ctx->d_sys, X0, X1, W, ctx->n_e, feat, target);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return oq_ctx_set_error(ctx, OQ_ERR_CUDA, cudaGetErrorString(e));
  return OQ_OK;
}

int oqmc_mlp_forward(oqmc_mlp* m, const unsigned short* feat, int R, float* out, void* stream) {
  if (!m || R < 0 || (R > 0 && (!feat || !out))) return merr(m, OQ_ERR_ARG, "bad arguments");
  if (R == 0) return OQ_OK;
  static bool attr = false;
  if (!attr) {
    OQ_MCUDA(m, cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     FW_SMEM));
    attr = true;
  }
  cudaStream_t s = (cudaStream_t)stream;
  k_mlp_forward<<<(R + 127) / 128, 128, FW_SMEM, s>>>(feat, R, m->wbf, m->theta, out, m->d_flags);
  OQ_MCUDA(m, cudaGetLastError());
  return oq_mlp_check_flags(m, s);
}

int oqmc_mlp_backward(oqmc_mlp* m, const unsigned short* feat, const float* target, int R,
                      float* grad, double* loss_sum, void* stream) {
  if (!m || R < 1 || !feat || !target || !grad) return merr(m, OQ_ERR_ARG, "bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  OQ_MCUDA(m, cudaMemsetAsync(grad, 0, OQ_MLP_NPARAM * sizeof(float), s));
  if (loss_sum) OQ_MCUDA(m, cudaMemsetAsync(loss_sum, 0, sizeof(double), s));
  const int rc = train_kernel(m, feat, target, R, grad, loss_sum, s);
  if (rc != OQ_OK) return rc;
  return oq_mlp_check_flags(m, s);
}

int oqmc_mlp_step(oqmc_mlp* m, const unsigned short* feat, const float* target, int R, float lr,
                  double* loss_sum, void* stream) {
  if (!m || R < 1 || !feat || !target || !(lr >= 0.0f)) return merr(m, OQ_ERR_ARG, "bad arguments");
  cudaStream_t s = (cudaStream_t)stream;
  if (loss_sum) OQ_MCUDA(m, cudaMemsetAsync(loss_sum, 0, sizeof(double), s));
  int rc = train_kernel(m, feat, target, R, m->grad, loss_sum, s);
  if (rc != OQ_OK) return rc;
  m->t += 1;
  const float bc1 = 1.0f - powf(0.9f, (float)m->t), bc2 = 1.0f - powf(0.999f, (float)m->t);
  k_mlp_adam<<<(OQ_MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->theta, m->m, m->v, m->grad, m->wbf,
                                                         m->wtbf, lr, bc1, bc2);
  OQ_MCUDA(m, cudaGetLastError());
  return OQ_OK;
}

int oqmc_mlp_get_flags(oqmc_mlp* m, unsigned* flags, int clear, void* stream) {
  if (!m || !flags) return OQ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  OQ_MCUDA(m, cudaMemcpyAsync(flags, m->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  if (clear) OQ_MCUDA(m, cudaMemsetAsync(m->d_flags, 0, sizeof(unsigned), s));
  OQ_MCUDA(m, cudaStreamSynchronize(s));
  return OQ_OK;
}

}  // extern "C"
