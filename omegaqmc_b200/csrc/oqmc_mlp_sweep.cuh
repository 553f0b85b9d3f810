// Metropolis sweeps with the learned proposal (mixed precision).
//
// One CTA = 128 walkers = the 128 rows of every network evaluation, run by
// 256 threads: thread t < 128 owns walker t; threads 128-255 only share the
// hidden-layer epilogues (columns 64-127).  The walkers' positions and inverse Slater matrices stay in
// shared memory for the whole launch (as in k_moves), next to the BF16
// weights in the canonical tensor-core layout.  For each electron e of a
// sweep:
//   1. every thread writes the features of its walker's electron e and the
//      CTA runs the network on the tensor cores -> mixture q(. | x);
//   2. the thread draws the displacement d (component from a uniform, then
//      mu + sigma * N(0, 1)) and evaluates log q(d | x) (FP32 mixture math);
//   3. features at x' = x + d -> network -> log q(-d | x');
//   4. oq_try_move accepts with |psi(x')/psi(x)|^2 q(x|x') / q(x'|x)
//      (Sherman-Morrison update on acceptance).
// Random numbers: Philox counters (walker, sweep, electron, stream 0/1) for
// the normals and the acceptance uniform, stream 2 for the component.
#pragma once
#include "oqmc_batch.cuh"
#include "oqmc_mlp.cuh"

#define OQ_MLPS_BIAS 1024
#define OQ_MLPS_BAR (OQ_MLPS_BIAS + OQ_MLP_SM_BIAS)
#define OQ_MLPS_ACT 3072
#define OQ_MLPS_W (OQ_MLPS_ACT + OQ_MLP_SM_ACT)
#define OQ_MLPS_POS (OQ_MLPS_W + OQ_MLP_SM_WEIGHTS)

// Shared memory of k_moves_mlp for NOCC occupied orbitals per spin.
__host__ __device__ constexpr size_t oq_mlp_sweep_smem(int nocc) {
  return (size_t)OQ_MLPS_POS + (size_t)6 * nocc * 128 * 8 + (size_t)2 * nocc * nocc * 128 * 4;
}

struct OqMlpWeights {
  const unsigned short* wbf;   // BF16 weights, row-major
  const float* theta;          // FP32 parameters (biases read from here)
};

template <int NOCC, class B>
__global__ void __launch_bounds__(256, 1)
k_moves_mlp(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
            const void* __restrict__ gC, OqMoveArgs a, OqMlpWeights nw) {
  constexpr int NE = 2 * NOCC;
  constexpr int NN = NOCC * NOCC;
  constexpr int WT = 128;
  extern __shared__ __align__(16) unsigned char smem[];
  OqJas& J = *reinterpret_cast<OqJas*>(smem);
  float* bias = reinterpret_cast<float*>(smem + OQ_MLPS_BIAS);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + OQ_MLPS_BAR);
  uint32_t* slot = reinterpret_cast<uint32_t*>(smem + OQ_MLPS_BAR + 8);
  unsigned char* act = smem + OQ_MLPS_ACT;
  unsigned char* wreg = smem + OQ_MLPS_W;
  double* pos = reinterpret_cast<double*>(smem + OQ_MLPS_POS);   // [3 NE][128]
  float* Ai = reinterpret_cast<float*>(pos + 3 * NE * WT);        // [2 NN][128]
  const OqSystem& S = *gsys;
  const OqSplit& SP = *gsplit;
  const float* C = reinterpret_cast<const float*>(gC);
  const int tid = threadIdx.x & 127, warp = threadIdx.x >> 5;
  const bool owner = threadIdx.x < 128;     // owns walker tid
  const int W = a.W;
  const int w = blockIdx.x * WT + tid;
  const bool live = owner && w < W;
  if (warp == 0) oq_tmem_alloc(slot, 128);
  if (tid == 0) oq_mbar_init(bar, 1);
  oq_jas_load(J, S);
  oq_mlp_load_weights(wreg, nw.wbf);
  oq_mlp_load_bias(bias, nw.theta);
  const float* gA = reinterpret_cast<const float*>(a.ainv);
  if (owner) {
    for (int k = 0; k < 3 * NE; ++k) pos[k * WT + tid] = live ? a.pos[(size_t)k * W + w] : 0.0;
    for (int k = 0; k < 2 * NN; ++k) Ai[k * WT + tid] = live ? gA[(size_t)k * W + w] : 0.0f;
  }
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
  const uint32_t tmem = *slot;
  OqMlpSync sy{bar, 0u};
  double logdet = live ? a.logdet[w] : 0.0;
  int nacc = 0;
  bool ok = true;
  auto P = [&](int j, int c) { return pos[(3 * j + c) * WT + tid]; };
  for (int t = 0; t < a.n_steps && ok; ++t) {
    const uint32_t gstep = (uint32_t)(a.step_base + t);
    for (int e = 0; e < NE; ++e) {
      double n3[3], u;
      oq_move_randoms(a.seed, (uint32_t)w, gstep, (uint32_t)e, n3, u);
      const OqU4 c2 = {(uint32_t)w, gstep, (uint32_t)e, 2u};
      const OqU4 rc = oq_philox(c2, (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
      const float uc = ((float)rc.x + 0.5f) * 2.3283064365386963e-10f;
      const double ox = P(e, 0), oy = P(e, 1), oz = P(e, 2);
      float f[OQ_MLP_K0], out[OQ_MLP_NOUT];
      if (owner) {
        oq_mlp_features(J, P, NE, e, ox, oy, oz, f);
        oq_mlp_store_features(act, tid, f);
      }
      ok = oq_mlp_forward_tile(act, wreg, bias, tmem, sy, out, nullptr, nullptr);
      if (!ok) break;
      double d[3] = {0.0, 0.0, 0.0};
      float lqf = 0.0f;
      if (owner) {
        oq_mix_sample_f(out, uc, n3, d);
        lqf = oq_mix_logq_f(out, (float)d[0], (float)d[1], (float)d[2]);
      }
      const double nx = ox + d[0], ny = oy + d[1], nz = oz + d[2];
      if (owner) {
        oq_mlp_features(J, P, NE, e, nx, ny, nz, f);
        oq_mlp_store_features(act, tid, f);
      }
      ok = oq_mlp_forward_tile(act, wreg, bias, tmem, sy, out, nullptr, nullptr);
      if (!ok) break;
      const float lqr = owner ? oq_mix_logq_f(out, (float)(ox - nx), (float)(oy - ny),
                                             (float)(oz - nz))
                              : 0.0f;
      if (live)
        nacc += oq_try_move<NOCC, float, float, B>(J, S, SP, C, pos, Ai, WT, tid, e, nx, ny, nz,
                                                   (double)(lqr - lqf), u, logdet);
    }
  }
  if (live) {
    for (int k = 0; k < 3 * NE; ++k) a.pos[(size_t)k * W + w] = pos[k * WT + tid];
    float* gAw = reinterpret_cast<float*>(a.ainv);
    for (int k = 0; k < 2 * NN; ++k) gAw[(size_t)k * W + w] = Ai[k * WT + tid];
    a.logdet[w] = logdet;
  }
  if (a.acc_sum) {
    double v = (double)nacc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) atomicAdd(a.acc_sum, v);
  }
  oq_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    oq_tc_fence_after();
    if (!ok) oq_mbar_wait(bar, sy.phase ^ 1u);
    oq_tmem_dealloc(tmem, 128);
  }
  if (!ok && tid == 0) atomicOr(a.flags, OQ_FLAG_TIMEOUT);
}
