// Local energy with the MO contraction on the tensor cores (mixed build).
//
// A CTA of 128 threads owns 128 rows = (walker, electron) pairs, electron-
// major (row r: electron r / Wb, walker r % Wb, Wb = 128 / n_e).  Each thread
// evaluates the AO value, gradient and Laplacian of its row and writes them
// to shared memory as the A operand of five GEMMs (one per component):
//   MO[c](128 x 16) = AO[c](128 x K) * C(K x 16),  K = nbf padded to 16.
// FP32 accuracy from split operands: A = A_hi + A_lo with A_hi rounded to
// TF32 and A_lo = A - A_hi stored as BF16; C = C_hi + C_lo (TF32 each), so
//   D = A_hi C_hi + A_hi C_lo  (kind::tf32)  +  A_lo C_hi  (kind::f16, BF16)
// leaves an error of order 2^-19 relative per product.  One thread issues
// the MMAs into TMEM (five 16-column FP32 accumulators), commits to an
// mbarrier, and every warp reads its 32 rows back with tcgen05.ld; the
// Slater gradient/Laplacian, Jastrow VGL and Coulomb terms follow as in
// k_eloc (OmegaQMC/psi/gto.py:728-778, 1575-1649, 2406-2451, 2506-2579).
#pragma once
#include "oqmc_sweep.cuh"
#include "oqmc_tc.cuh"

// Shared-memory plan of k_eloc_tc.  K4: nbf padded to a multiple of 8 (the
// TF32 MMA K step), K2: padded to 16 (the BF16 step).  B operands are packed
// on the host in the same canonical layout: C_hi, C_lo (TF32), C_hi (BF16).
struct OqTcPlan {
  uint32_t K4, K2, a_hi, a_lo, b_hi, b_lo, b_bf, b_end, red, bar, slot, total;
};

__host__ __device__ inline OqTcPlan oq_tc_plan(int nbf) {
  OqTcPlan p;
  p.K4 = (uint32_t)((nbf + 7) / 8 * 8);
  p.K2 = (uint32_t)((nbf + 15) / 16 * 16);
  uint32_t o = 0;
  p.a_hi = o; o += 5u * 128u * p.K4 * 4u;
  p.a_lo = o; o += 5u * 128u * p.K2 * 2u;
  p.b_hi = o; o += 16u * p.K4 * 4u;
  p.b_lo = o; o += 16u * p.K4 * 4u;
  p.b_bf = o; o += 16u * p.K2 * 2u;
  p.b_end = o;
  o = (o + 15u) & ~15u;
  p.red = o; o += 128u * 4u * 8u;
  p.bar = o; o += 16u;
  p.slot = o; o += 16u;
  p.total = o;
  return p;
}

// Store one AO's five components (value, d/dx, d/dy, d/dz, Laplacian) of
// row r at column k into the split A operands (the BF16 low part truncated).
__device__ __forceinline__ void oq_tc_store_ao(unsigned char* sm, const OqTcPlan& P, int r, int k,
                                               const float v[5]) {
  const uint32_t o4 = oq_kmajor_off4(r, k, (int)(P.K4 >> 2));
  const uint32_t o2 = oq_kmajor_off2(r, k, (int)(P.K2 >> 3));
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    const float hi = oq_tf32(v[c]);
    *reinterpret_cast<float*>(sm + P.a_hi + (uint32_t)c * 128u * P.K4 * 4u + o4) = hi;
    *reinterpret_cast<unsigned short*>(sm + P.a_lo + (uint32_t)c * 128u * P.K2 * 2u + o2) =
        (unsigned short)(__float_as_uint(v[c] - hi) >> 16);
  }
}

// Zero the BF16 low part of column k (K4 <= k < K2: no TF32 column there).
__device__ __forceinline__ void oq_tc_zero_lo(unsigned char* sm, const OqTcPlan& P, int r, int k) {
  const uint32_t o2 = oq_kmajor_off2(r, k, (int)(P.K2 >> 3));
#pragma unroll
  for (int c = 0; c < 5; ++c)
    *reinterpret_cast<unsigned short*>(sm + P.a_lo + (uint32_t)c * 128u * P.K2 * 2u + o2) = 0;
}

// AO VGL of one position written into the A operands (table-driven basis;
// FP64 radial sums for tight groups near their nucleus and cusp shells).
__device__ __forceinline__ void oq_tc_ao_rows(const OqSystem& S, const OqSplit& SP,
                                              unsigned char* sm, const OqTcPlan& P, int r,
                                              double x, double y, double z) {
  for (int g = 0; g < S.ngroup; ++g) {
    const int ia = S.g_iat[g];
    const double dxd = x - S.nuc[ia][0], dyd = y - S.nuc[ia][1], dzd = z - S.nuc[ia][2];
    const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
    const float dx = (float)dxd, dy = (float)dyd, dz = (float)dzd;
    const int ncol = S.g_ncol[g], np = S.g_n[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    float R[OQ_MAX_COL], Rp[OQ_MAX_COL], Rl[OQ_MAX_COL];
    if ((r2d < SP.r2[g]) || S.s_cusp[sh0]) {
      double Rd[OQ_MAX_COL] = {0, 0, 0, 0}, Rpd[OQ_MAX_COL] = {0, 0, 0, 0},
             Rld[OQ_MAX_COL] = {0, 0, 0, 0};
      for (int p = 0; p < np; ++p) {
        const double a = S.alpha[off + p];
        const double e = exp(-a * r2d);
        const double fp = -2.0 * a * e, fl = (4.0 * a * a * r2d - 6.0 * a) * e;
#pragma unroll
        for (int k = 0; k < OQ_MAX_COL; ++k)
          if (k < ncol) {
            const double n = S.norm[S.s_norm[sh0 + k] + p];
            Rd[k] += n * e; Rpd[k] += n * fp; Rld[k] += n * fl;
          }
      }
      if (S.g_am[g] == 0) {
#pragma unroll
        for (int k = 0; k < OQ_MAX_COL; ++k)
          if (k < ncol && S.s_cusp[sh0 + k]) oq_cusp_vgl(S, ia, sqrt(r2d), Rd[k], Rpd[k], Rld[k]);
      }
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k) { R[k] = (float)Rd[k]; Rp[k] = (float)Rpd[k]; Rl[k] = (float)Rld[k]; }
    } else {
      const float r2 = (float)r2d;
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k) R[k] = Rp[k] = Rl[k] = 0.0f;
      for (int p = 0; p < np; ++p) {
        const float a = (float)S.alpha[off + p];
        const float e = __expf(-a * r2);
        const float fp = -2.0f * a * e, fl = (4.0f * a * a * r2 - 6.0f * a) * e;
#pragma unroll
        for (int k = 0; k < OQ_MAX_COL; ++k)
          if (k < ncol) {
            const float n = (float)S.norm[S.s_norm[sh0 + k] + p];
            R[k] += n * e; Rp[k] += n * fp; Rl[k] += n * fl;
          }
      }
    }
    const int am = S.g_am[g];
#pragma unroll
    for (int k = 0; k < OQ_MAX_COL; ++k) {
      if (k >= ncol) break;
      const int ao = S.s_ao[sh0 + k];
      if (am == 0) {
        const float v[5] = {R[k], Rp[k] * dx, Rp[k] * dy, Rp[k] * dz, Rl[k]};
        oq_tc_store_ao(sm, P, r, ao, v);
      } else {
        float Yd[5], dYd[5][3];
        if (am == 2) oq_harm_d<float>(dx, dy, dz, Yd, dYd);
        const float lfac = Rl[k] + (float)(2 * am) * Rp[k];
        for (int c = 0; c < 2 * am + 1; ++c) {
          float Y, dY[3];
          if (am == 1) {
            Y = (c == 0) ? dx : (c == 1) ? dy : dz;
            dY[0] = (float)(c == 0); dY[1] = (float)(c == 1); dY[2] = (float)(c == 2);
          } else if (am == 2) {
            Y = Yd[c]; dY[0] = dYd[c][0]; dY[1] = dYd[c][1]; dY[2] = dYd[c][2];
          } else {
            oq_harm_table<float>(S.harm, am, c, dx, dy, dz, Y, dY);
          }
          const float v[5] = {R[k] * Y, Rp[k] * dx * Y + R[k] * dY[0],
                              Rp[k] * dy * Y + R[k] * dY[1], Rp[k] * dz * Y + R[k] * dY[2],
                              lfac * Y};
          oq_tc_store_ao(sm, P, r, ao + c, v);
        }
      }
    }
  }
}

template <int NOCC>
__global__ void __launch_bounds__(128)
k_eloc_tc(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
          const unsigned char* __restrict__ gB, OqElocArgs a) {
  constexpr int NE = 2 * NOCC;
  constexpr int WB = 128 / NE;
  extern __shared__ __align__(1024) unsigned char sm[];
  // the system tables are read through L1 (uniform loads); shared memory
  // holds only the MMA operands, the reduction buffer and the barrier
  const OqSystem& S = *gsys;
  const OqSplit& SP = *gsplit;
  const OqTcPlan P = oq_tc_plan(S.nbf);
  double* red = reinterpret_cast<double*>(sm + P.red);        // [4][128]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + P.bar);
  uint32_t* slot = reinterpret_cast<uint32_t*>(sm + P.slot);
  const int t = threadIdx.x, warp = t >> 5;
  {
    const int nb4 = (int)((P.b_end - P.b_hi) / 16);
    const int4* b4 = reinterpret_cast<const int4*>(gB);
    int4* sb = reinterpret_cast<int4*>(sm + P.b_hi);
    for (int i = t; i < nb4; i += 128) sb[i] = b4[i];
  }
  if (warp == 0) oq_tmem_alloc(slot, 128);
  if (t == 0) oq_mbar_init(bar, 1);
  oq_tc_fence_before();
  __syncthreads();
  oq_tc_fence_after();
  const uint32_t tmem = *slot;
  const int W = a.W;
  const int e = t / WB, wl = t % WB;
  const int w = blockIdx.x * WB + wl;
  const bool live = (e < NE) && (w < W);
  // ---- AO VGL rows -> shared-memory A operands ----
  double xe = 0, ye = 0, ze = 0;
  const float zero[5] = {0, 0, 0, 0, 0};
  if (live) {
    xe = a.pos[(size_t)(3 * e) * W + w];
    ye = a.pos[(size_t)(3 * e + 1) * W + w];
    ze = a.pos[(size_t)(3 * e + 2) * W + w];
    oq_tc_ao_rows(S, SP, sm, P, t, xe, ye, ze);
    for (int k = S.nbf; k < (int)P.K4; ++k) oq_tc_store_ao(sm, P, t, k, zero);
  } else {
    for (int k = 0; k < (int)P.K4; ++k) oq_tc_store_ao(sm, P, t, k, zero);
  }
  for (int k = (int)P.K4; k < (int)P.K2; ++k) oq_tc_zero_lo(sm, P, t, k);
  oq_fence_async_smem();
  __syncthreads();
  if (t == 0) {
    oq_tc_fence_after();
    const uint32_t idt = oq_idesc_tf32(128, 16), idb = oq_idesc_bf16(128, 16);
    const uint32_t base = oq_smem_addr(sm);
    const uint32_t KC4 = P.K4 >> 2, KC2 = P.K2 >> 3;
    for (int c = 0; c < 5; ++c) {
      const uint32_t d = tmem + (uint32_t)(16 * c);
      const uint32_t ahi = base + P.a_hi + (uint32_t)c * 128u * P.K4 * 4u;
      const uint32_t alo = base + P.a_lo + (uint32_t)c * 128u * P.K2 * 2u;
      for (int s = 0; s < (int)P.K4 / 8; ++s) {
        const uint64_t ad = oq_desc_kmajor(ahi + 256u * s, 128u, KC4 * 128u);
        const uint64_t bh = oq_desc_kmajor(base + P.b_hi + 256u * s, 128u, KC4 * 128u);
        const uint64_t bl = oq_desc_kmajor(base + P.b_lo + 256u * s, 128u, KC4 * 128u);
        oq_mma_tf32(d, ad, bh, idt, s > 0 ? 1u : 0u);
        oq_mma_tf32(d, ad, bl, idt, 1u);
      }
      for (int s = 0; s < (int)P.K2 / 16; ++s) {
        const uint64_t ad = oq_desc_kmajor(alo + 256u * s, 128u, KC2 * 128u);
        const uint64_t bb = oq_desc_kmajor(base + P.b_bf + 256u * s, 128u, KC2 * 128u);
        oq_mma_bf16(d, ad, bb, idb, 1u);
      }
    }
    oq_mma_commit(bar);
  }
  __syncwarp();
  const bool ok_wait = oq_mbar_wait(bar, 0);
  oq_tc_fence_after();
  // ---- MO VGL of this row from TMEM (lane = row = t) ----
  float mv[16], mgx[16], mgy[16], mgz[16], ml[16];
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  oq_tmem_ld16(lane_base + 0, mv);
  oq_tmem_ld16(lane_base + 16, mgx);
  oq_tmem_ld16(lane_base + 32, mgy);
  oq_tmem_ld16(lane_base + 48, mgz);
  oq_tmem_ld16(lane_base + 64, ml);
  double ee = 0.0, en = 0.0, lp_tot = 0.0, g2 = 0.0;
  if (live && ok_wait) {
    const int s = e & 1, i = e >> 1;
    const float* A = reinterpret_cast<const float*>(a.ainv);
    float gx = 0, gy = 0, gz = 0, lp = 0;
#pragma unroll
    for (int m = 0; m < NOCC; ++m) {
      const float am = A[(size_t)((s * NOCC + m) * NOCC + i) * W + w];
      gx += am * mgx[m]; gy += am * mgy[m]; gz += am * mgz[m]; lp += am * ml[m];
    }
    float jx = 0, jy = 0, jz = 0, jl = 0;
    for (int j = 0; j < NE; ++j) {
      if (j == e) continue;
      const double dx = xe - a.pos[(size_t)(3 * j) * W + w],
                   dy = ye - a.pos[(size_t)(3 * j + 1) * W + w],
                   dz = ze - a.pos[(size_t)(3 * j + 2) * W + w];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (j > e) ee += rsqrt(r2 + OQ_EPS);
      if (S.has_j2) {
        const int o = ((e & 1) == (j & 1)) ? 0 : 2;
        const float r2t = (float)r2, rinv = rsqrtf(r2t);
        float upr, l;
        oq_pade_vgl_q((float)S.j2[o], (float)S.j2[o + 1], r2t * rinv, rinv, upr, l);
        jx += upr * (float)dx; jy += upr * (float)dy; jz += upr * (float)dz; jl += l;
      }
    }
    for (int I = 0; I < S.natm; ++I) {
      const double dx = xe - S.nuc[I][0], dy = ye - S.nuc[I][1], dz = ze - S.nuc[I][2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      en -= S.Z[I] * rsqrt(r2 + OQ_EPS);
      if (S.has_j1) {
        const float r2t = (float)r2, rinv = rsqrtf(r2t);
        float upr, l;
        oq_pade_vgl_q((float)S.j1a[I], (float)S.j1b[I], r2t * rinv, rinv, upr, l);
        jx += upr * (float)dx; jy += upr * (float)dy; jz += upr * (float)dz; jl += l;
      }
    }
    const double sgx = gx, sgy = gy, sgz = gz;
    const double Gx = sgx + jx, Gy = sgy + jy, Gz = sgz + jz;
    lp_tot = (double)lp - (sgx * sgx + sgy * sgy + sgz * sgz) + (double)jl;
    g2 = Gx * Gx + Gy * Gy + Gz * Gz;
  }
  red[0 * 128 + t] = ee;
  red[1 * 128 + t] = en;
  red[2 * 128 + t] = lp_tot;
  red[3 * 128 + t] = g2;
  oq_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    oq_tc_fence_after();
    if (!ok_wait) oq_mbar_wait(bar, 0);   // let the MMAs drain before freeing TMEM
    oq_tmem_dealloc(tmem, 128);
  }
  if (!ok_wait && t == 0) atomicOr(a.flags, OQ_FLAG_TIMEOUT);
  // per-walker sums over its NE rows (threads t < WB), then over walkers
  if (t < 64) {
    const int ww = blockIdx.x * WB + t;
    const bool wlive = (t < WB) && (ww < W) && ok_wait;
    double see = 0, sen = 0, slp = 0, sg2 = 0;
    if (wlive) {
      for (int k = 0; k < NE; ++k) {
        see += red[0 * 128 + k * WB + t];
        sen += red[1 * 128 + k * WB + t];
        slp += red[2 * 128 + k * WB + t];
        sg2 += red[3 * 128 + k * WB + t];
      }
    }
    const double ke = -0.5 * (slp + sg2);
    const double el = see + sen + ke + S.e_nn;
    const bool ok = wlive && isfinite(el);
    if (wlive) {
      if (a.el_trace) a.el_trace[ww] = el;
      if (a.eparts) {
        double* ep = a.eparts + (size_t)ww * 4;
        ep[0] = see; ep[1] = sen; ep[2] = ke; ep[3] = el;
      }
      if (!ok) atomicOr(a.flags, OQ_FLAG_NAN);
    }
    double vals[6] = {ok ? see : 0.0, ok ? sen : 0.0, ok ? ke : 0.0, ok ? el : 0.0,
                      ok ? el * el : 0.0, ok ? 1.0 : 0.0};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double v = vals[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      vals[k] = v;
    }
    if ((t & 31) == 0) {
#pragma unroll
      for (int k = 0; k < 5; ++k) atomicAdd(a.sums + k, vals[k]);
      atomicAdd(a.sums + 6, vals[5]);
    }
  }
}
