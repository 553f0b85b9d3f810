// Learned Metropolis proposal: a per-electron MLP (32 -> 128 -> 128 -> 128
// -> 48, ReLU, BF16 operands, FP32 accumulation) whose outputs define an
// 8-component isotropic Gaussian mixture for the electron's displacement.
//
// Tensor-core layout.  A CTA evaluates the network for 128 rows (walkers or
// training samples) at once: thread t owns row t, which is TMEM lane t of
// the accumulators.  Each layer is one chain of tcgen05.mma (kind::f16, BF16
// A and B, M = 128, N = out width, K = in width in steps of 16) issued by
// thread 0 from shared-memory operands in the K-major no-swizzle canonical
// layout (oqmc_tc.cuh), committed to an mbarrier that every thread waits on
// (bounded); the epilogue reads the thread's accumulator row with
// tcgen05.ld, adds the bias, applies ReLU, rounds to BF16 and writes the row
// back as the next layer's A operand.
//
// Mixture outputs: logits 0..7, means 8..31 (component c at 8+3c), sigma_c =
// 0.02 + softplus(out[32+c]); outputs 40..47 are unused padding to N = 48.
#pragma once
#include "oqmc_tc.cuh"

#define OQ_MLP_K0 32
#define OQ_MLP_H 128
#define OQ_MLP_NOUT 48
#define OQ_MLP_NMIX 8
#define OQ_MLP_SIGMIN 0.02
// flat FP32 parameter vector (row-major weights [out][in])
#define OQ_MLP_OFF_W1 0
#define OQ_MLP_OFF_B1 4096
#define OQ_MLP_OFF_W2 4224
#define OQ_MLP_OFF_B2 20608
#define OQ_MLP_OFF_W3 20736
#define OQ_MLP_OFF_B3 37120
#define OQ_MLP_OFF_W4 37248
#define OQ_MLP_OFF_B4 43392
#define OQ_MLP_NPARAM 43440

// shared-memory sizes (bytes) of the canonical operand buffers
#define OQ_MLP_SM_W1 (OQ_MLP_H * OQ_MLP_K0 * 2)      // 8 KB
#define OQ_MLP_SM_WH (OQ_MLP_H * OQ_MLP_H * 2)       // 32 KB
#define OQ_MLP_SM_W4 (OQ_MLP_NOUT * OQ_MLP_H * 2)    // 12 KB
#define OQ_MLP_SM_WEIGHTS (OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH + OQ_MLP_SM_W4)   // 84 KB
#define OQ_MLP_SM_ACT (128 * OQ_MLP_H * 2)           // 32 KB
#define OQ_MLP_SM_BIAS 1792                           // 3*128 + 48 floats, padded

// Two FP32 values as packed BF16 (round to nearest even): lo in bits 0..15.
__device__ __forceinline__ uint32_t oq_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
  return r;
}
__device__ __forceinline__ float oq_bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float oq_bf16_hi(uint32_t v) { return __uint_as_float(v & 0xFFFF0000u); }

// Copy a row-major BF16 matrix [N][K] from global memory into the canonical
// K-major layout (16-byte chunks; K a multiple of 8).
__device__ __forceinline__ void oq_mlp_load_kmajor(unsigned char* dst,
                                                   const unsigned short* __restrict__ src,
                                                   int N, int K) {
  const int KC = K / 8;
  const uint4* s4 = reinterpret_cast<const uint4*>(src);
  for (int i = threadIdx.x; i < N * KC; i += blockDim.x) {
    const int n = i / KC, c = i - n * KC;
    *reinterpret_cast<uint4*>(dst + (((n >> 3) * KC + c) << 7) + ((n & 7) << 4)) = s4[i];
  }
}

// Store 16 FP32 values (columns c0..c0+15 of row r) as BF16 into a K-major
// canonical buffer with KC chunks per row.
__device__ __forceinline__ void oq_mlp_store_row16(unsigned char* buf, int r, int c0, int KC,
                                                   const float v[16]) {
  uint4 a, b;
  a.x = oq_bf16x2(v[0], v[1]);   a.y = oq_bf16x2(v[2], v[3]);
  a.z = oq_bf16x2(v[4], v[5]);   a.w = oq_bf16x2(v[6], v[7]);
  b.x = oq_bf16x2(v[8], v[9]);   b.y = oq_bf16x2(v[10], v[11]);
  b.z = oq_bf16x2(v[12], v[13]); b.w = oq_bf16x2(v[14], v[15]);
  const int c = c0 >> 3;
  unsigned char* p = buf + (((r >> 3) * KC + c) << 7) + ((r & 7) << 4);
  *reinterpret_cast<uint4*>(p) = a;
  *reinterpret_cast<uint4*>(p + 128) = b;
}

// Issue D[128 x N] = A[128 x K] B[N x K]^T (both K-major canonical, BF16)
// from one thread; commit to bar unless it is null (a later commit covers
// these MMAs too).
__device__ __forceinline__ void oq_mlp_mma(uint32_t tmem_d, const unsigned char* A,
                                           const unsigned char* Bm, int N, int K, uint64_t* bar) {
  const uint32_t a0 = oq_smem_addr(A), b0 = oq_smem_addr(Bm);
  const uint32_t sbo = (uint32_t)(K / 8) * 128u;
  const uint32_t idesc = oq_idesc_bf16(128, N);
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t ad = oq_desc_kmajor(a0 + (uint32_t)ks * 256u, 128u, sbo);
    const uint64_t bd = oq_desc_kmajor(b0 + (uint32_t)ks * 256u, 128u, sbo);
    oq_mma_bf16(tmem_d, ad, bd, idesc, ks > 0 ? 1u : 0u);
  }
  if (bar) oq_mma_commit(bar);
}

// One CTA-wide step: make the generic-proxy smem writes visible, order them
// before the MMA, issue from thread 0 and wait (bounded) for completion.
// Returns false (for every thread) when the wait timed out.
struct OqMlpSync {
  uint64_t* bar;
  uint32_t phase;
};

__device__ __forceinline__ bool oq_mlp_wait(OqMlpSync& s) {
  const bool ok = oq_mbar_wait(s.bar, s.phase);
  s.phase ^= 1u;
  oq_tc_fence_after();
  return !__syncthreads_or(!ok);
}

__device__ __forceinline__ void oq_mlp_pre_issue() {
  oq_fence_async_smem();
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
}

// Hidden-layer epilogue: columns [c_begin, c_end) of row r of D (TMEM lane
// r) + bias, ReLU, BF16 into the K-major buffer `act` (KC = 16).  Optionally
// also into the transposed buffer `ht` ([128 features x 128 rows], KC = 16)
// and a 128-bit ReLU mask.  Columns are read 64 at a time (four loads in
// flight, one wait).
__device__ __forceinline__ void oq_mlp_hidden_epilogue(uint32_t tmem_row, const float* bias,
                                                       unsigned char* act, int r,
                                                       unsigned char* ht, uint32_t* mask,
                                                       int c_begin = 0, int c_end = OQ_MLP_H) {
#pragma unroll 1
  for (int h0 = c_begin; h0 < c_end; h0 += 64) {
    uint32_t raw[64];
#pragma unroll
    for (int q = 0; q < 4; ++q) oq_tmem_ld16_nw(tmem_row + (uint32_t)(h0 + 16 * q), raw + 16 * q);
    oq_tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int c0 = h0 + 16 * q;
      float v[16];
      uint32_t mbits = 0;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const float z = __uint_as_float(raw[16 * q + j]) + bias[c0 + j];
        v[j] = z > 0.0f ? z : 0.0f;
        mbits |= (z > 0.0f ? 1u : 0u) << j;
      }
      oq_mlp_store_row16(act, r, c0, 16, v);
      if (mask) mask[c0 >> 5] |= mbits << (c0 & 16);
      if (ht) {
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
  }
}

// Output epilogue: 48 FP32 outputs of row r.
__device__ __forceinline__ void oq_mlp_out_epilogue(uint32_t tmem_row, const float* bias,
                                                    float out[OQ_MLP_NOUT]) {
  uint32_t raw[OQ_MLP_NOUT];
#pragma unroll
  for (int q = 0; q < OQ_MLP_NOUT / 16; ++q) oq_tmem_ld16_nw(tmem_row + (uint32_t)(16 * q), raw + 16 * q);
  oq_tmem_wait_ld();
  const float4* b4 = reinterpret_cast<const float4*>(bias);   // 16-byte aligned
#pragma unroll
  for (int j = 0; j < OQ_MLP_NOUT / 4; ++j) {
    const float4 bb = b4[j];
    out[4 * j] = __uint_as_float(raw[4 * j]) + bb.x;
    out[4 * j + 1] = __uint_as_float(raw[4 * j + 1]) + bb.y;
    out[4 * j + 2] = __uint_as_float(raw[4 * j + 2]) + bb.z;
    out[4 * j + 3] = __uint_as_float(raw[4 * j + 3]) + bb.w;
  }
}

// Load biases b1..b3 (128 each) and b4 (48) from the FP32 parameter vector.
__device__ __forceinline__ void oq_mlp_load_bias(float* bias, const float* __restrict__ theta) {
  for (int i = threadIdx.x; i < 3 * OQ_MLP_H + OQ_MLP_NOUT; i += blockDim.x) {
    const int l = i / OQ_MLP_H, j = i - l * OQ_MLP_H;
    const int off = l == 0 ? OQ_MLP_OFF_B1 : l == 1 ? OQ_MLP_OFF_B2 : l == 2 ? OQ_MLP_OFF_B3
                                                                       : OQ_MLP_OFF_B4;
    bias[i] = theta[off + j];
  }
}

// Load W1..W4 (BF16, row-major) into the canonical weight region.
__device__ __forceinline__ void oq_mlp_load_weights(unsigned char* wreg,
                                                    const unsigned short* __restrict__ wbf) {
  oq_mlp_load_kmajor(wreg, wbf + OQ_MLP_OFF_W1, OQ_MLP_H, OQ_MLP_K0);
  oq_mlp_load_kmajor(wreg + OQ_MLP_SM_W1, wbf + OQ_MLP_OFF_W2, OQ_MLP_H, OQ_MLP_H);
  oq_mlp_load_kmajor(wreg + OQ_MLP_SM_W1 + OQ_MLP_SM_WH, wbf + OQ_MLP_OFF_W3, OQ_MLP_H, OQ_MLP_H);
  oq_mlp_load_kmajor(wreg + OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH, wbf + OQ_MLP_OFF_W4, OQ_MLP_NOUT,
                     OQ_MLP_H);
}

// Forward pass of the 128 rows whose BF16 inputs are in `act` (K = 32,
// KC = 4); leaves row r's 48 outputs in `out` of thread r (r < 128).
// With 256 threads, threads 128-255 (warps 4-7, the same TMEM lane quarters
// as warps 0-3) write columns 64-127 of every hidden layer and threads
// 0-127 columns 0-63.  `ht`/`mask` (training, 128 threads) receive the
// transposed hidden activations and ReLU masks of layers 1..3.  Returns
// false when an MMA wait timed out (uniform over the CTA).
__device__ __forceinline__ bool oq_mlp_forward_tile(unsigned char* act, const unsigned char* wreg,
                                                    const float* bias, uint32_t tmem,
                                                    OqMlpSync& sy, float out[OQ_MLP_NOUT],
                                                    unsigned char* const* ht, uint32_t* mask) {
  const int r = threadIdx.x & 127;
  const bool pair = blockDim.x == 256;
  const int c_begin = pair ? (threadIdx.x >= 128 ? 64 : 0) : 0;
  const int c_end = pair ? c_begin + 64 : OQ_MLP_H;
  const uint32_t trow = tmem + ((uint32_t)((r >> 5) * 32) << 16);
  const unsigned char* W[4] = {wreg, wreg + OQ_MLP_SM_W1, wreg + OQ_MLP_SM_W1 + OQ_MLP_SM_WH,
                               wreg + OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH};
  for (int l = 0; l < 4; ++l) {
    oq_mlp_pre_issue();
    if (threadIdx.x == 0)
      oq_mlp_mma(tmem, act, W[l], l == 3 ? OQ_MLP_NOUT : OQ_MLP_H, l == 0 ? OQ_MLP_K0 : OQ_MLP_H,
                 sy.bar);
    if (!oq_mlp_wait(sy)) return false;
    if (l < 3)
      oq_mlp_hidden_epilogue(trow, bias + l * OQ_MLP_H, act, r, ht ? ht[l] : nullptr,
                             mask ? mask + 4 * l : nullptr, c_begin, c_end);
    else if (threadIdx.x < 128)
      oq_mlp_out_epilogue(trow, bias + 3 * OQ_MLP_H, out);
  }
  oq_tc_fence_before();
  return true;
}

// ---------------------------------------------------------------------------
// Forward pass with the activations in tensor memory.  Each group of 128
// rows owns 192 TMEM columns from `tmem`: the FP32 accumulator D in
// columns [0, 128) and the BF16 A operand (the layer input, two elements per
// column) in [128, 192).  Thread r writes its row's features, and after each
// hidden layer its ReLU outputs, into its own lane of the A columns with
// tcgen05.st, so no activation tile sits in shared memory and the MMA reads
// A straight from TMEM.
#define OQ_MLP_TA_COL 128u

__device__ __forceinline__ void oq_mlp_mma_ta(uint32_t tmem_d, uint32_t tmem_a,
                                              const unsigned char* Bm, int N, int K,
                                              uint64_t* bar) {
  const uint32_t b0 = oq_smem_addr(Bm);
  const uint32_t sbo = (uint32_t)(K / 8) * 128u;
  const uint32_t idesc = oq_idesc_bf16(128, N);
  for (int ks = 0; ks < K / 16; ++ks) {
    const uint64_t bd = oq_desc_kmajor(b0 + (uint32_t)ks * 256u, 128u, sbo);
    oq_mma_bf16_ta(tmem_d, tmem_a + (uint32_t)ks * 8u, bd, idesc, ks > 0 ? 1u : 0u);
  }
  if (bar) oq_mma_commit(bar);
}

// Row r's 32 BF16 features (16 packed words, the lower half the even
// feature) into its lane of the A columns.
__device__ __forceinline__ void oq_mlp_store_features_ta(uint32_t trow, const uint32_t f2[16]) {
  oq_tmem_st16(trow + OQ_MLP_TA_COL, f2);
}

// Hidden-layer epilogue into the A columns: D + bias, ReLU, BF16 pairs.
__device__ __forceinline__ void oq_mlp_hidden_epilogue_ta(uint32_t trow, const float* bias) {
#pragma unroll 1
  for (int h0 = 0; h0 < OQ_MLP_H; h0 += 64) {
    uint32_t raw[64];
#pragma unroll
    for (int q = 0; q < 4; ++q) oq_tmem_ld16_nw(trow + (uint32_t)(h0 + 16 * q), raw + 16 * q);
    oq_tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      // the biases as 16-byte shared-memory loads (the same words for every
      // thread: broadcasts)
      const float4* b4 = reinterpret_cast<const float4*>(bias + h0 + 32 * q);
      uint32_t pk[16];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float4 bb = b4[j];
        const uint32_t* rw = raw + 32 * q + 4 * j;
        pk[2 * j] = oq_bf16x2(fmaxf(__uint_as_float(rw[0]) + bb.x, 0.0f),
                              fmaxf(__uint_as_float(rw[1]) + bb.y, 0.0f));
        pk[2 * j + 1] = oq_bf16x2(fmaxf(__uint_as_float(rw[2]) + bb.z, 0.0f),
                                  fmaxf(__uint_as_float(rw[3]) + bb.w, 0.0f));
      }
      oq_tmem_st16(trow + OQ_MLP_TA_COL + (uint32_t)((h0 + 32 * q) >> 1), pk);
    }
  }
  oq_tmem_wait_st();
}

// Forward pass of a 128-thread CTA's 128 rows with the activations in TMEM
// (features already stored in the A columns, oq_tmem_wait_st done); leaves
// row r's 48 outputs in `out` of thread r.  Returns false when an MMA wait
// timed out (uniform over the CTA).
__device__ __forceinline__ bool oq_mlp_forward_tile_ta(const unsigned char* wreg,
                                                       const float* bias, uint32_t tmem,
                                                       OqMlpSync& sy, float out[OQ_MLP_NOUT]) {
  const int r = threadIdx.x & 127;
  const uint32_t trow = tmem + ((uint32_t)((r >> 5) * 32) << 16);
  const unsigned char* W[4] = {wreg, wreg + OQ_MLP_SM_W1, wreg + OQ_MLP_SM_W1 + OQ_MLP_SM_WH,
                               wreg + OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH};
  for (int l = 0; l < 4; ++l) {
    oq_tc_fence_before();
    __syncthreads();
    oq_tc_fence_after();
    if (threadIdx.x == 0)
      oq_mlp_mma_ta(tmem, tmem + OQ_MLP_TA_COL, W[l], l == 3 ? OQ_MLP_NOUT : OQ_MLP_H,
                    l == 0 ? OQ_MLP_K0 : OQ_MLP_H, sy.bar);
    if (!oq_mlp_wait(sy)) return false;
    if (l < 3)
      oq_mlp_hidden_epilogue_ta(trow, bias + l * OQ_MLP_H);
    else
      oq_mlp_out_epilogue(trow, bias + 3 * OQ_MLP_H, out);
  }
  oq_tc_fence_before();
  return true;
}

// ---------------------------------------------------------------------------
// Mixture density (double precision on the FP32 network outputs)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double oq_softplus(double x) {
  return x > 30.0 ? x : log1p(exp(x));
}

// log q(d) of the mixture defined by out.
__device__ __forceinline__ double oq_mix_logq(const float out[OQ_MLP_NOUT], double dx, double dy,
                                              double dz) {
  double amax = -1e300;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) amax = fmax(amax, (double)out[c]);
  double zs = 0.0;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) zs += exp((double)out[c] - amax);
  const double lz = amax + log(zs);
  double L[OQ_MLP_NMIX], lmax = -1e300;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    const double sg = OQ_MLP_SIGMIN + oq_softplus((double)out[32 + c]);
    const double ex = dx - out[8 + 3 * c], ey = dy - out[9 + 3 * c], ez = dz - out[10 + 3 * c];
    L[c] = (double)out[c] - lz - 3.0 * log(sg) - 2.7568155996140185 -
           0.5 * (ex * ex + ey * ey + ez * ez) / (sg * sg);
    lmax = fmax(lmax, L[c]);
  }
  double s = 0.0;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) s += exp(L[c] - lmax);
  return lmax + log(s);
}

// Draw a displacement: component = first c with CDF(c) > uc, then
// mu_c + sigma_c * n3.
__device__ __forceinline__ void oq_mix_sample(const float out[OQ_MLP_NOUT], double uc,
                                              const double n3[3], double d[3]) {
  double amax = -1e300;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) amax = fmax(amax, (double)out[c]);
  double zs = 0.0;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) zs += exp((double)out[c] - amax);
  double cdf = 0.0;
  int sel = OQ_MLP_NMIX - 1;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    cdf += exp((double)out[c] - amax) / zs;
    if (cdf > uc) { sel = c; break; }
  }
  const double sg = OQ_MLP_SIGMIN + oq_softplus((double)out[32 + sel]);
  d[0] = out[8 + 3 * sel] + sg * n3[0];
  d[1] = out[9 + 3 * sel] + sg * n3[1];
  d[2] = out[10 + 3 * sel] + sg * n3[2];
}

// FP32 versions for the sampler (fast exponentials; the proposal density is
// evaluated by the same function that defines the draw's mixture, so the
// rounding enters the acceptance ratio at the 1e-6 level only).
__device__ __forceinline__ float oq_softplus_f(float x) {
  return x > 20.0f ? x : __logf(1.0f + __expf(x));
}

__device__ __forceinline__ float oq_mix_logq_f(const float out[OQ_MLP_NOUT], float dx, float dy,
                                               float dz) {
  float amax = out[0];
#pragma unroll
  for (int c = 1; c < OQ_MLP_NMIX; ++c) amax = fmaxf(amax, out[c]);
  float zs = 0.0f;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c) zs += __expf(out[c] - amax);
  const float lz = amax + __logf(zs);
  float L[OQ_MLP_NMIX], lmax = -3.0e38f;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    const float sg = (float)OQ_MLP_SIGMIN + oq_softplus_f(out[32 + c]);
    const float ex = dx - out[8 + 3 * c], ey = dy - out[9 + 3 * c], ez = dz - out[10 + 3 * c];
    const float is = 1.0f / sg;
    L[c] = out[c] - lz + 3.0f * __logf(is) - 2.7568156f - 0.5f * (ex * ex + ey * ey + ez * ez) * is * is;
    lmax = fmaxf(lmax, L[c]);
  }
  float s = 0.0f;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c) s += __expf(L[c] - lmax);
  return lmax + __logf(s);
}

__device__ __forceinline__ void oq_mix_sample_f(const float out[OQ_MLP_NOUT], float uc,
                                                const double n3[3], double d[3]) {
  float amax = out[0];
#pragma unroll
  for (int c = 1; c < OQ_MLP_NMIX; ++c) amax = fmaxf(amax, out[c]);
  float w[OQ_MLP_NMIX], zs = 0.0f;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    w[c] = __expf(out[c] - amax);
    zs += w[c];
  }
  // component: first c whose cumulative weight exceeds uc (branch-free scan)
  const float thr = uc * zs;
  int sel = OQ_MLP_NMIX - 1;
  float acc = 0.0f;
  bool found = false;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    acc += w[c];
    const bool hit = !found && acc > thr;
    sel = hit ? c : sel;
    found = found || hit;
  }
  float sg = 0.0f, mx = 0.0f, my = 0.0f, mz = 0.0f;
#pragma unroll
  for (int c = 0; c < OQ_MLP_NMIX; ++c)
    if (c == sel) {
      sg = (float)OQ_MLP_SIGMIN + oq_softplus_f(out[32 + c]);
      mx = out[8 + 3 * c]; my = out[9 + 3 * c]; mz = out[10 + 3 * c];
    }
  d[0] = (double)(mx + sg * (float)n3[0]);
  d[1] = (double)(my + sg * (float)n3[1]);
  d[2] = (double)(mz + sg * (float)n3[2]);
}

// Negative log-likelihood of target d and its gradient with respect to the
// 48 outputs (times scale); unused outputs get 0.
__device__ __forceinline__ double oq_mix_nll_grad(const float out[OQ_MLP_NOUT], const float d[3],
                                                  float scale, float g[OQ_MLP_NOUT]) {
  double amax = -1e300;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) amax = fmax(amax, (double)out[c]);
  double zs = 0.0;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) zs += exp((double)out[c] - amax);
  const double lz = amax + log(zs);
  double L[OQ_MLP_NMIX], sg[OQ_MLP_NMIX], r2[OQ_MLP_NMIX], lmax = -1e300;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    sg[c] = OQ_MLP_SIGMIN + oq_softplus((double)out[32 + c]);
    const double ex = d[0] - out[8 + 3 * c], ey = d[1] - out[9 + 3 * c], ez = d[2] - out[10 + 3 * c];
    r2[c] = ex * ex + ey * ey + ez * ez;
    L[c] = (double)out[c] - lz - 3.0 * log(sg[c]) - 2.7568155996140185 - 0.5 * r2[c] / (sg[c] * sg[c]);
    lmax = fmax(lmax, L[c]);
  }
  double s = 0.0;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) s += exp(L[c] - lmax);
  const double lq = lmax + log(s);
  for (int j = 0; j < OQ_MLP_NOUT; ++j) g[j] = 0.0f;
  for (int c = 0; c < OQ_MLP_NMIX; ++c) {
    const double gam = exp(L[c] - lq);
    const double w = exp((double)out[c] - lz);
    g[c] = (float)(scale * (w - gam));
    const double is2 = 1.0 / (sg[c] * sg[c]);
    g[8 + 3 * c] = (float)(scale * (-gam * (d[0] - out[8 + 3 * c]) * is2));
    g[9 + 3 * c] = (float)(scale * (-gam * (d[1] - out[9 + 3 * c]) * is2));
    g[10 + 3 * c] = (float)(scale * (-gam * (d[2] - out[10 + 3 * c]) * is2));
    const double dsig = -gam * (r2[c] * is2 / sg[c] - 3.0 / sg[c]);
    const double sigm = 1.0 / (1.0 + exp(-(double)out[32 + c]));
    g[32 + c] = (float)(scale * dsig * sigm);
  }
  return -lq;
}

// ---------------------------------------------------------------------------
// Features of electron e at (xe, ye, ze): position relative to the nearest
// and second-nearest nucleus, displacements to the 8 nearest other electrons
// (nearest first, ties to the lower index, zeros when fewer), spin (+1 for
// even e) and a constant 1.  P(j, c) returns coordinate c of electron j.
// ---------------------------------------------------------------------------
template <class SJ, class PosF>
__device__ __forceinline__ void oq_mlp_features(const SJ& J, PosF P, int ne, int e, double xe,
                                                double ye, double ze, float f[OQ_MLP_K0]) {
  double d0 = 1e300, d1 = 1e300;
  int i0 = 0, i1 = 0;
  for (int I = 0; I < J.natm; ++I) {
    const double ax = xe - J.nuc[I][0], ay = ye - J.nuc[I][1], az = ze - J.nuc[I][2];
    const double r2 = ax * ax + ay * ay + az * az;
    if (r2 < d0) {
      d1 = d0; i1 = i0; d0 = r2; i0 = I;
    } else if (r2 < d1) {
      d1 = r2; i1 = I;
    }
  }
  if (J.natm == 1) i1 = i0;
  f[0] = (float)(xe - J.nuc[i0][0]); f[1] = (float)(ye - J.nuc[i0][1]); f[2] = (float)(ze - J.nuc[i0][2]);
  f[3] = (float)(xe - J.nuc[i1][0]); f[4] = (float)(ye - J.nuc[i1][1]); f[5] = (float)(ze - J.nuc[i1][2]);
  uint32_t used = 1u << e;
  for (int k = 0; k < 8; ++k) {
    double best = 1e300;
    int bj = -1;
    for (int j = 0; j < ne; ++j) {
      if (used & (1u << j)) continue;
      const double ax = P(j, 0) - xe, ay = P(j, 1) - ye, az = P(j, 2) - ze;
      const double r2 = ax * ax + ay * ay + az * az;
      if (r2 < best) { best = r2; bj = j; }
    }
    if (bj < 0) {
      f[6 + 3 * k] = 0.0f; f[7 + 3 * k] = 0.0f; f[8 + 3 * k] = 0.0f;
    } else {
      used |= 1u << bj;
      f[6 + 3 * k] = (float)(P(bj, 0) - xe);
      f[7 + 3 * k] = (float)(P(bj, 1) - ye);
      f[8 + 3 * k] = (float)(P(bj, 2) - ze);
    }
  }
  f[30] = (e & 1) ? -1.0f : 1.0f;
  f[31] = 1.0f;
}

// The same features for a compile-time electron count (the sweep's): the
// squared distances to the other electrons are computed once in FP32 and
// kept in registers, the 8 nearest are selected with branch-free
// compare/selects (same order and tie rule as oq_mlp_features, which ranks
// FP64 distances, so two nearly equidistant electrons can swap places) and
// only their coordinates are read again.
template <int NE, class SJ, class PosF>
__device__ __forceinline__ void oq_mlp_features_ne(const SJ& J, PosF P, int e, double xe,
                                                   double ye, double ze, float f[OQ_MLP_K0]) {
  double d0 = 1e300, d1 = 1e300;
  int i0 = 0, i1 = 0;
  for (int I = 0; I < J.natm; ++I) {
    const double ax = xe - J.nuc[I][0], ay = ye - J.nuc[I][1], az = ze - J.nuc[I][2];
    const double r2 = ax * ax + ay * ay + az * az;
    if (r2 < d0) {
      d1 = d0; i1 = i0; d0 = r2; i0 = I;
    } else if (r2 < d1) {
      d1 = r2; i1 = I;
    }
  }
  if (J.natm == 1) i1 = i0;
  f[0] = (float)(xe - J.nuc[i0][0]); f[1] = (float)(ye - J.nuc[i0][1]); f[2] = (float)(ze - J.nuc[i0][2]);
  f[3] = (float)(xe - J.nuc[i1][0]); f[4] = (float)(ye - J.nuc[i1][1]); f[5] = (float)(ze - J.nuc[i1][2]);
  // squared distances in FP32 from the FP64 coordinate differences: the
  // ranking only has to be a fixed function of the configuration
  float r2[NE];
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    const float ax = (float)(P(j, 0) - xe), ay = (float)(P(j, 1) - ye),
                az = (float)(P(j, 2) - ze);
    r2[j] = (j == e) ? 3.0e38f : ax * ax + ay * ay + az * az;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float best = 3.0e38f;
    int bj = -1;
#pragma unroll
    for (int j = 0; j < NE; ++j) {
      const bool c = r2[j] < best;
      best = c ? r2[j] : best;
      bj = c ? j : bj;
    }
#pragma unroll
    for (int j = 0; j < NE; ++j) r2[j] = (j == bj) ? 3.0e38f : r2[j];
    if (bj < 0) {
      f[6 + 3 * k] = 0.0f; f[7 + 3 * k] = 0.0f; f[8 + 3 * k] = 0.0f;
    } else {
      f[6 + 3 * k] = (float)(P(bj, 0) - xe);
      f[7 + 3 * k] = (float)(P(bj, 1) - ye);
      f[8 + 3 * k] = (float)(P(bj, 2) - ze);
    }
  }
  f[30] = (e & 1) ? -1.0f : 1.0f;
  f[31] = 1.0f;
}

// Write the 32 features of row r as BF16 into a K-major buffer (KC = 4).
__device__ __forceinline__ void oq_mlp_store_features(unsigned char* act, int r,
                                                      const float f[OQ_MLP_K0]) {
  oq_mlp_store_row16(act, r, 0, 4, f);
  oq_mlp_store_row16(act, r, 16, 4, f + 16);
}
