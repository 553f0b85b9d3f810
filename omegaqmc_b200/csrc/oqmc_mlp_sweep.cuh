// Metropolis sweeps with the learned proposal (mixed precision).
//
// A CTA runs G independent groups of 128 walkers; group g is warps
// 4g..4g+3, thread r of the group owns walker r of its tile and row r of the
// group's network evaluations (TMEM lane r).  The BF16 weights (canonical
// tensor-core layout) are shared by the groups in shared memory; each group
// has its own mbarrier and named barrier, so the groups advance
// independently and one group's network latency overlaps the others'
// CUDA-core work.  For up to two groups (the default) each group's
// activations live in its own 256 TMEM columns (the FP32 accumulator and
// the BF16 layer input that the next MMA reads from TMEM), which leaves the
// shared memory for the groups' FP64 positions: the features and the move
// read them there.  The inverse Slater matrices and log|det| stay in global
// memory, walker-minor (L2-resident).  With four groups the activations are
// shared-memory tiles and the positions stay in global memory.
//
// For each electron e of a sweep:
//   1. the group writes the features of its walkers' electron e and runs the
//      network on the tensor cores -> mixture q(. | x);
//   2. each thread draws the displacement d (component from a uniform, then
//      mu + sigma * N(0, 1)) and evaluates log q(d | x) (FP32 mixture math);
//   3. features at x' = x + d -> network -> log q(-d | x');
//   4. oq_try_move accepts with |psi(x')/psi(x)|^2 q(x|x') / q(x'|x)
//      (Sherman-Morrison update on acceptance).
// Random numbers: Philox counters (walker, sweep, electron, stream 0) for
// the normals and the acceptance uniform, stream 2 for the component.
#pragma once
#include "oqmc_batch.cuh"
#include "oqmc_mlp.cuh"

#define OQ_MLPS_BIAS 1024
#define OQ_MLPS_BAR (OQ_MLPS_BIAS + OQ_MLP_SM_BIAS)
#define OQ_MLPS_ACT 3072
#define OQ_MLPS_MAXG 4

// Shared memory of k_moves_mlp with G walker groups of ne-electron walkers:
// header, the groups' activation tiles and the weights, plus, where it fits
// in a CTA's 227 KB, an FP32 copy of each group's walker positions
// ([3 ne][128] floats per group) that the features read instead of the
// FP64 state in global memory.
__host__ __device__ constexpr size_t oq_mlp_sweep_base(int groups) {
  return (size_t)OQ_MLPS_ACT + (size_t)groups * OQ_MLP_SM_ACT + OQ_MLP_SM_WEIGHTS;
}
__host__ __device__ constexpr size_t oq_mlp_posf_bytes(int groups, int ne) {
  return (size_t)groups * 3 * ne * 128 * sizeof(float);
}
__host__ __device__ constexpr bool oq_mlp_posf_fits(int groups, int ne) {
  return oq_mlp_sweep_base(groups) + oq_mlp_posf_bytes(groups, ne) <= (size_t)227 * 1024;
}
// Activations in TMEM and FP64 positions in shared memory (the default
// layout): for up to two groups, where the groups' positions fit beside the
// weights.  The shared memory then holds the header, the weights and
// [G][3 ne][128] doubles; TMEM gives each group 256 columns (its FP32
// accumulator and its BF16 activations).
__host__ __device__ constexpr size_t oq_mlp_ta_bytes(int groups, int ne) {
  return (size_t)OQ_MLPS_ACT + OQ_MLP_SM_WEIGHTS + (size_t)groups * 3 * ne * 128 * sizeof(double);
}
__host__ __device__ constexpr bool oq_mlp_ta_fits(int groups, int ne) {
  return groups <= 2 && oq_mlp_ta_bytes(groups, ne) <= (size_t)227 * 1024;
}
__host__ __device__ constexpr size_t oq_mlp_sweep_smem(int groups, int ne) {
  return oq_mlp_ta_fits(groups, ne)
             ? oq_mlp_ta_bytes(groups, ne)
             : oq_mlp_sweep_base(groups) +
                   (oq_mlp_posf_fits(groups, ne) ? oq_mlp_posf_bytes(groups, ne) : 0);
}

struct OqMlpWeights {
  const unsigned short* wbf;   // BF16 weights, row-major
  const float* theta;          // FP32 parameters (biases read from here)
};

// Named barrier `id` over n threads, and its OR-reduction of a predicate.
__device__ __forceinline__ void oq_group_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ bool oq_group_or(bool v, int id, int n) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n"
      " selp.u32 %0, 1, 0, q;\n}"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}

// Network forward pass of one group's 128 rows (inputs already in `act`),
// synchronising only the group's 128 threads (named barrier bar_id).
// Returns false (for every thread of the group) when an MMA wait timed out.
__device__ __forceinline__ bool oq_mlp_forward_group(unsigned char* act, const unsigned char* wreg,
                                                     const float* bias, uint32_t tmem_cols,
                                                     uint64_t* bar, uint32_t& phase, int r,
                                                     int bar_id, float out[OQ_MLP_NOUT]) {
  const uint32_t trow = tmem_cols + ((uint32_t)((r >> 5) * 32) << 16);
  const unsigned char* W[4] = {wreg, wreg + OQ_MLP_SM_W1, wreg + OQ_MLP_SM_W1 + OQ_MLP_SM_WH,
                               wreg + OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH};
  for (int l = 0; l < 4; ++l) {
    oq_fence_async_smem();
    oq_tc_fence_before();
    oq_group_sync(bar_id, 128);
    oq_tc_fence_after();
    if (r == 0)
      oq_mlp_mma(tmem_cols, act, W[l], l == 3 ? OQ_MLP_NOUT : OQ_MLP_H,
                 l == 0 ? OQ_MLP_K0 : OQ_MLP_H, bar);
    const bool ok = oq_mbar_wait(bar, phase);
    phase ^= 1u;
    oq_tc_fence_after();
    if (oq_group_or(!ok, bar_id, 128)) return false;
    if (l < 3)
      oq_mlp_hidden_epilogue(trow, bias + l * OQ_MLP_H, act, r, nullptr, nullptr);
    else
      oq_mlp_out_epilogue(trow, bias + 3 * OQ_MLP_H, out);
  }
  oq_tc_fence_before();
  return true;
}

// The same pass with the group's activations in TMEM (group columns from
// tmem: accumulator [0, 128), BF16 activations [128, 192)); the features are
// already in the activation columns.
__device__ __forceinline__ bool oq_mlp_forward_group_ta(const unsigned char* wreg,
                                                        const float* bias, uint32_t tmem_cols,
                                                        uint64_t* bar, uint32_t& phase, int r,
                                                        int bar_id, float out[OQ_MLP_NOUT]) {
  const uint32_t trow = tmem_cols + ((uint32_t)((r >> 5) * 32) << 16);
  const unsigned char* W[4] = {wreg, wreg + OQ_MLP_SM_W1, wreg + OQ_MLP_SM_W1 + OQ_MLP_SM_WH,
                               wreg + OQ_MLP_SM_W1 + 2 * OQ_MLP_SM_WH};
  for (int l = 0; l < 4; ++l) {
    oq_tc_fence_before();
    oq_group_sync(bar_id, 128);
    oq_tc_fence_after();
    if (r == 0)
      oq_mlp_mma_ta(tmem_cols, tmem_cols + OQ_MLP_TA_COL, W[l],
                    l == 3 ? OQ_MLP_NOUT : OQ_MLP_H, l == 0 ? OQ_MLP_K0 : OQ_MLP_H, bar);
    const bool ok = oq_mbar_wait(bar, phase);
    phase ^= 1u;
    oq_tc_fence_after();
    if (oq_group_or(!ok, bar_id, 128)) return false;
    if (l < 3)
      oq_mlp_hidden_epilogue_ta(trow, bias + l * OQ_MLP_H);
    else
      oq_mlp_out_epilogue(trow, bias + 3 * OQ_MLP_H, out);
  }
  oq_tc_fence_before();
  return true;
}

// Row r's features as BF16 pairs into its lane of the group's activation
// columns (the rounding of oq_mlp_store_features).
__device__ __forceinline__ void oq_mlp_features_to_tmem(uint32_t tmem_cols, int r,
                                                        const float f[OQ_MLP_K0]) {
  uint32_t f2[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) f2[j] = oq_bf16x2(f[2 * j], f[2 * j + 1]);
  oq_mlp_store_features_ta(tmem_cols + ((uint32_t)((r >> 5) * 32) << 16), f2);
  oq_tmem_wait_st();
}

template <int NOCC, class B, int G>
__global__ void __launch_bounds__(128 * G, 1)
k_moves_mlp(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
            const void* __restrict__ gC, OqMoveArgs a, OqMlpWeights nw) {
  constexpr int NE = 2 * NOCC;
  static_assert(G >= 1 && G <= OQ_MLPS_MAXG, "1..4 walker groups");
  extern __shared__ __align__(16) unsigned char smem[];
  OqJas& J = *reinterpret_cast<OqJas*>(smem);
  float* bias = reinterpret_cast<float*>(smem + OQ_MLPS_BIAS);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + OQ_MLPS_BAR);     // [G]
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + OQ_MLPS_BAR + 8 * OQ_MLPS_MAXG);
  // TA: activations in TMEM, the group's FP64 positions in shared memory;
  // otherwise activation tiles in shared memory and the positions in global
  // memory, with an FP32 copy for the features where it fits
  constexpr bool TA = oq_mlp_ta_fits(G, NE);
  constexpr bool POSF = !TA && oq_mlp_posf_fits(G, NE);
  unsigned char* wreg = smem + OQ_MLPS_ACT + (TA ? 0 : G * OQ_MLP_SM_ACT);
  const OqSystem& S = *gsys;
  const OqSplit& SP = *gsplit;
  const float* C = reinterpret_cast<const float*>(gC);
  const int g = threadIdx.x >> 7, r = threadIdx.x & 127, warp = threadIdx.x >> 5;
  unsigned char* act = smem + OQ_MLPS_ACT + g * OQ_MLP_SM_ACT;
  // FP32 copy of the group's positions, [3 NE][128]: row r's walker only
  float* posf = reinterpret_cast<float*>(smem + oq_mlp_sweep_base(G)) + (size_t)g * 3 * NE * 128;
  // FP64 positions of the group (TA), [3 NE][128]
  double* posd = reinterpret_cast<double*>(smem + OQ_MLPS_ACT + OQ_MLP_SM_WEIGHTS) +
                 (size_t)g * 3 * NE * 128;
  const int W = a.W;
  const int w = (blockIdx.x * G + g) * 128 + r;
  const bool live = w < W;
  const int wr = live ? w : W - 1;          // rows past the end read a valid walker
  constexpr uint32_t TCOLS = TA ? 256u * G : (G == 1 ? 128u : G == 2 ? 256u : 512u);
  if (warp == 0) oq_tmem_alloc(slot, TCOLS);
  if (threadIdx.x < G) oq_mbar_init(bars + threadIdx.x, 1);
  oq_jas_load(J, S);
  oq_mlp_load_weights(wreg, nw.wbf);
  oq_mlp_load_bias(bias, nw.theta);
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
  const uint32_t tbase = *slot;
  const uint32_t tmem = tbase + (uint32_t)((TA ? 256 : 128) * g);
  uint64_t* bar = bars + g;
  const int bar_id = 1 + g;
  uint32_t phase = 0u;
  double* pos = a.pos;
  float* Ai = reinterpret_cast<float*>(a.ainv);
  double logdet = a.logdet[wr];
  int nacc = 0;
  bool ok = true;
  auto P = [&](int j, int c) { return pos[(size_t)(3 * j + c) * W + wr]; };
  // the features read the other electrons from the FP32 copy where it fits
  // (a fixed function of the state, so the proposal density of every state
  // is well defined and the Metropolis-Hastings ratio stays exact)
  auto PF = [&](int j, int c) { return (double)posf[(3 * j + c) * 128 + r]; };
  auto PD = [&](int j, int c) { return posd[(3 * j + c) * 128 + r]; };
  if (POSF)
    for (int k = 0; k < 3 * NE; ++k) posf[k * 128 + r] = (float)pos[(size_t)k * W + wr];
  if (TA)
    for (int k = 0; k < 3 * NE; ++k) posd[k * 128 + r] = pos[(size_t)k * W + wr];
  for (int t = 0; t < a.n_steps && ok; ++t) {
    const uint32_t gstep = (uint32_t)(a.step_base + t);
    for (int e = 0; e < NE; ++e) {
      double n3[3], u;
      oq_move_randoms(a.seed, (uint32_t)w, gstep, (uint32_t)e, n3, u);
      const OqU4 c2 = {(uint32_t)w, gstep, (uint32_t)e, 2u};
      const OqU4 rc = oq_philox(c2, (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
      const float uc = ((float)rc.x + 0.5f) * 2.3283064365386963e-10f;
      const double ox = TA ? PD(e, 0) : P(e, 0), oy = TA ? PD(e, 1) : P(e, 1),
                   oz = TA ? PD(e, 2) : P(e, 2);
      float f[OQ_MLP_K0], out[OQ_MLP_NOUT];
      if (TA) {
        oq_mlp_features_ne<NE>(J, PD, e, ox, oy, oz, f);
        oq_mlp_features_to_tmem(tmem, r, f);
        ok = oq_mlp_forward_group_ta(wreg, bias, tmem, bar, phase, r, bar_id, out);
      } else {
        if (POSF) oq_mlp_features_ne<NE>(J, PF, e, ox, oy, oz, f);
        else oq_mlp_features_ne<NE>(J, P, e, ox, oy, oz, f);
        oq_mlp_store_features(act, r, f);
        ok = oq_mlp_forward_group(act, wreg, bias, tmem, bar, phase, r, bar_id, out);
      }
      if (!ok) break;
      double d[3];
      oq_mix_sample_f(out, uc, n3, d);
      const float lqf = oq_mix_logq_f(out, (float)d[0], (float)d[1], (float)d[2]);
      const double nx = ox + d[0], ny = oy + d[1], nz = oz + d[2];
      if (TA) {
        oq_mlp_features_ne<NE>(J, PD, e, nx, ny, nz, f);
        oq_mlp_features_to_tmem(tmem, r, f);
        ok = oq_mlp_forward_group_ta(wreg, bias, tmem, bar, phase, r, bar_id, out);
      } else {
        if (POSF) oq_mlp_features_ne<NE>(J, PF, e, nx, ny, nz, f);
        else oq_mlp_features_ne<NE>(J, P, e, nx, ny, nz, f);
        oq_mlp_store_features(act, r, f);
        ok = oq_mlp_forward_group(act, wreg, bias, tmem, bar, phase, r, bar_id, out);
      }
      if (!ok) break;
      const float lqr = oq_mix_logq_f(out, (float)(ox - nx), (float)(oy - ny), (float)(oz - nz));
      if (live) {
        bool acc;
        if (TA)
          acc = oq_try_move_s<NOCC, float, float, B>(J, S, SP, C, posd + r, 128, Ai + w, W, e,
                                                     nx, ny, nz, lqr - lqf, 1.0f, (float)u,
                                                     logdet);
        else
          acc = oq_try_move<NOCC, float, float, B>(J, S, SP, C, pos, Ai, W, w, e, nx, ny, nz,
                                                   lqr - lqf, 1.0f, (float)u, logdet);
        nacc += acc;
        if (POSF && acc) {
          posf[(3 * e) * 128 + r] = (float)nx;
          posf[(3 * e + 1) * 128 + r] = (float)ny;
          posf[(3 * e + 2) * 128 + r] = (float)nz;
        }
      }
    }
  }
  if (TA && live)
    for (int k = 0; k < 3 * NE; ++k) pos[(size_t)k * W + w] = posd[k * 128 + r];
  if (live) a.logdet[w] = logdet;
  if (a.acc_sum) {
    double v = (double)nacc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(a.acc_sum, v);
  }
  if (!ok && r == 0) {
    oq_mbar_wait(bar, phase ^ 1u);          // let the group's outstanding MMA drain
    atomicOr(a.flags, OQ_FLAG_TIMEOUT);
  }
  oq_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    oq_tc_fence_after();
    oq_tmem_dealloc(tbase, TCOLS);
  }
}
