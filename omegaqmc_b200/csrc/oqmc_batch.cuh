// Batched sampling of several molecules in one persistent launch.
//
// The launch owns a list of tiles (system, first walker); every CTA pulls
// tiles from a global counter until the list is exhausted.  A tile of WT
// walkers of one system is processed start to finish by one CTA:
//   1. its positions are read from the system's (W, n_e, 3) walker array
//      (one contiguous block, coalesced) into shared memory, walker-minor;
//   2. the Slater inverses are rebuilt in FP64 (MO values from the tables,
//      Gauss-Jordan with partial pivoting), stored in shared memory as Real;
//   3. n_sweeps single-electron sweeps run with the walkers' state resident
//      in shared memory (threads 0..WT-1, one walker each), and every
//      measure_every sweeps all NT threads evaluate the local energy, NT/WT
//      threads per walker splitting its electrons;
//   4. the positions are written back.
// Tiles of different systems carry different electron counts, so the CTA's
// shared memory is sized for the largest tile of the batch.  The kernel that
// dispatches on the tile's system (a switch over per-system basis policies)
// is generated at run time together with those policies.
//
// Random numbers use the same Philox counters (walker, sweep, electron) as
// the per-system move kernel, so a batched run reproduces the per-system
// path (refresh, then sweeps) walker by walker for the same seed.
//
// The launch keeps its own bookkeeping in OqBatchCtl: the tile counter, a
// count of finished CTAs, the sweep counter of the next launch and the next
// measurement slot.  The last CTA to finish resets the tile counter and
// advances the sweep and slot counters, so consecutive launches (for example
// the nodes of a captured CUDA graph) continue the Markov chains without any
// host work in between.
#pragma once
#include "oqmc_sweep.cuh"

// Nuclei and Jastrow constants of one system (the fields the move and
// local-energy code read), copied to shared memory per tile.
struct OqJas {
  int natm, has_j1, has_j2, pad;
  double e_nn;
  double nuc[OQ_MAX_NUC][3];
  double Z[OQ_MAX_NUC];
  double j1a[OQ_MAX_NUC], j1b[OQ_MAX_NUC];
  double j2[4];
};

// One system of the batch (device copy; filled by the host).
struct OqBatchSys {
  const OqSystem* sys;      // system tables (global memory)
  const OqSplit* split;
  const double* C64;        // MO coefficients (nbf x nocc), FP64 and FP32
  const float* C32;
  double* walkers;          // (W, n_e, 3) positions, updated in place
  double* sums;             // [cap][OQ_NSUM] measurement sums (accumulated)
  unsigned long long* busy_ns;   // += tile time (ns), per system
  int W, n_e, wt;           // walkers, electrons, walkers per tile
  int proposal;             // 0 fixed-width, 1 nucleus-scaled Gaussian
  int cap;                  // measurement slots in sums
  int pad;
  double step, scale_r0, scale_fmin;
};

struct OqBatchTile {
  int sys, w0;
};

struct OqBatchCtl {
  unsigned next;            // next tile
  unsigned done;            // finished CTAs
  unsigned long long step;  // sweep counter at the start of the next launch
  unsigned long long slot;  // measurement slot of the next launch's first measurement
};

struct OqBatchArgs {
  const OqBatchSys* systems;
  const OqBatchTile* tiles;
  OqBatchCtl* ctl;
  unsigned* flags;
  int n_tiles;
  int n_sweeps;
  int measure_every;
  int write_sums;           // 0: local energies evaluated but not accumulated
  uint64_t seed;
};

#define OQ_BATCH_HDR 1024   // bytes reserved for OqJas + the tile broadcast

__device__ __forceinline__ unsigned long long oq_globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void oq_jas_load(OqJas& J, const OqSystem& S) {
  const int t = threadIdx.x;
  if (t == 0) {
    J.natm = S.natm; J.has_j1 = S.has_j1; J.has_j2 = S.has_j2; J.e_nn = S.e_nn;
  }
  if (t < 4) J.j2[t] = S.j2[t];
  for (int I = t; I < S.natm; I += blockDim.x) {
    J.nuc[I][0] = S.nuc[I][0]; J.nuc[I][1] = S.nuc[I][1]; J.nuc[I][2] = S.nuc[I][2];
    J.Z[I] = S.Z[I]; J.j1a[I] = S.j1a[I]; J.j1b[I] = S.j1b[I];
  }
}

// Shared memory of one tile: [reduction [NT/WT][4][WT] doubles, only when
// several threads share a walker's local energy][positions [3 NE][WT]
// doubles][inverses [2 NOCC^2][WT] Real].  The nuclei and Jastrow constants
// (J) are the system's OqJas in constant memory, written into the generated
// module, so every lane of a warp reads the same word (a broadcast) and the
// tile's shared memory holds walker state only.
template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ void oq_batch_tile(const OqBatchArgs& a, const OqBatchSys& d,
                                              const SJ& J, int w0, uint64_t step0,
                                              uint64_t slot0, unsigned char* smem) {
  constexpr int NE = 2 * NOCC;
  const int NT = blockDim.x, tid = threadIdx.x, WT = d.wt;
  const int parts = NT / WT, part = tid / WT, wl = tid - part * WT;
  double* red = reinterpret_cast<double*>(smem);                    // [parts][4][WT]
  double* pos = red + (parts > 1 ? 4 * NT : 0);                     // [3 NE][WT]
  Real* Ai = reinterpret_cast<Real*>(pos + 3 * NE * WT);           // [2 NOCC^2][WT]
  const OqSystem& S = *d.sys;
  const OqSplit& SP = *d.split;
  const Real* C = sizeof(Real) == 4 ? reinterpret_cast<const Real*>(d.C32)
                                    : reinterpret_cast<const Real*>(d.C64);
  unsigned long long t_start = 0;
  if (tid == 0) t_start = oq_globaltimer();
  const int cnt = min(WT, d.W - w0);
  {
    const double* src = d.walkers + (size_t)w0 * 3 * NE;
    for (int q = tid; q < cnt * 3 * NE; q += NT) {
      const int wl = q / (3 * NE), k = q - wl * 3 * NE;
      pos[k * WT + wl] = src[q];
    }
  }
  __syncthreads();
  const bool mover = tid < WT;
  const bool live = tid < cnt;
  const int w = w0 + tid;
  double logdet = 0.0;
  if (live) {
    // FP64 refresh of both spin blocks (as k_refresh)
    bool ok = true;
    for (int s = 0; s < 2; ++s) {
      double Sm[NOCC][NOCC], Ainv[NOCC][NOCC];
      for (int i = 0; i < NOCC; ++i) {
        const int e = 2 * i + s;
        double mv[NOCC];
        oq_mo_val<NOCC>(S, d.C64, pos[(3 * e) * WT + tid], pos[(3 * e + 1) * WT + tid],
                        pos[(3 * e + 2) * WT + tid], mv);
#pragma unroll
        for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
      }
      double ld;
      const bool oks = oq_invert<NOCC>(Sm, Ainv, ld);
      ok = ok && oks;
      logdet += ld;
      for (int m = 0; m < NOCC; ++m)
        for (int j = 0; j < NOCC; ++j)
          Ai[((s * NOCC + m) * NOCC + j) * WT + tid] = oks ? (Real)Ainv[m][j] : (Real)0;
    }
    if (!ok) {
      logdet = -INFINITY;
      atomicOr(a.flags, OQ_FLAG_SINGULAR);
    }
  }
  __syncthreads();
  int nacc = 0, meas = 0;
  for (int t = 0; t < a.n_sweeps; ++t) {
    if (live) {
      const uint32_t gstep = (uint32_t)(step0 + t);
      for (int e = 0; e < NE; ++e) {
        double n3[3], u;
        oq_move_randoms(a.seed, (uint32_t)w, gstep, (uint32_t)e, n3, u);
        const double ox = pos[(3 * e) * WT + tid], oy = pos[(3 * e + 1) * WT + tid],
                     oz = pos[(3 * e + 2) * WT + tid];
        if (d.proposal == 0) {
          nacc += oq_try_move<NOCC, T, Real, B>(J, S, SP, C, pos, Ai, WT, tid, e,
                                                ox + d.step * n3[0], oy + d.step * n3[1],
                                                oz + d.step * n3[2], 0.0, 1.0, u, logdet);
        } else {
          double nx, ny, nz, mul, lx;
          oq_scaled_propose(J, ox, oy, oz, n3, d.step, d.scale_r0, d.scale_fmin, nx, ny, nz, mul,
                            lx);
          nacc += oq_try_move<NOCC, T, Real, B>(J, S, SP, C, pos, Ai, WT, tid, e, nx, ny, nz, lx,
                                                mul, u, logdet);
        }
      }
    }
    if ((t + 1) % a.measure_every != 0) continue;
    __syncthreads();
    double see = 0.0, sen = 0.0, slp = 0.0, sg2 = 0.0;
    {
      double ee = 0.0, en = 0.0, lp = 0.0, g2 = 0.0;
      if (wl < cnt)
        for (int e = part; e < NE; e += parts)
          oq_eloc_electron<NOCC, T, Real, B>(J, S, SP, C, pos + wl, (size_t)WT, Ai + wl,
                                             (size_t)WT, e, ee, en, lp, g2);
      if (parts > 1) {
        red[(part * 4 + 0) * WT + wl] = ee;
        red[(part * 4 + 1) * WT + wl] = en;
        red[(part * 4 + 2) * WT + wl] = lp;
        red[(part * 4 + 3) * WT + wl] = g2;
      } else {
        see = ee; sen = en; slp = lp; sg2 = g2;
      }
    }
    if (parts > 1) __syncthreads();
    if (mover) {
      if (parts > 1)
        for (int k = 0; k < parts; ++k) {
          see += red[(k * 4 + 0) * WT + tid];
          sen += red[(k * 4 + 1) * WT + tid];
          slp += red[(k * 4 + 2) * WT + tid];
          sg2 += red[(k * 4 + 3) * WT + tid];
        }
      const double ke = -0.5 * (slp + sg2);
      const double el = see + sen + ke + J.e_nn;
      const bool ok = live && isfinite(el);
      if (live && !ok) atomicOr(a.flags, OQ_FLAG_NAN);
      double vals[7] = {ok ? see : 0.0, ok ? sen : 0.0, ok ? ke : 0.0, ok ? el : 0.0,
                        ok ? el * el : 0.0, (double)nacc, ok ? 1.0 : 0.0};
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        double v = vals[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        vals[k] = v;
      }
      const uint64_t slot = slot0 + (uint64_t)meas;
      if ((tid & 31) == 0 && a.write_sums && slot < (uint64_t)d.cap) {
        double* sm = d.sums + slot * OQ_NSUM;
#pragma unroll
        for (int k = 0; k < 7; ++k) atomicAdd(sm + k, vals[k]);
      }
    }
    nacc = 0;
    ++meas;
  }
  __syncthreads();
  {
    double* dst = d.walkers + (size_t)w0 * 3 * NE;
    for (int q = tid; q < cnt * 3 * NE; q += NT) {
      const int wl2 = q / (3 * NE), k = q - wl2 * 3 * NE;
      dst[q] = pos[k * WT + wl2];
    }
  }
  if (tid == 0) atomicAdd(d.busy_ns, oq_globaltimer() - t_start);
  __syncthreads();
}

// Claim the next tile for the whole CTA; -1 when none is left.  The claimed
// index passes through the first word of shared memory, which belongs to the
// tile state only between this call's second barrier and the end of the
// tile (oq_batch_tile ends with a barrier).
__device__ __forceinline__ int oq_batch_next(const OqBatchArgs& a, unsigned char* smem) {
  int* slot = reinterpret_cast<int*>(smem);
  if (threadIdx.x == 0) {
    const unsigned k = atomicAdd(&a.ctl->next, 1u);
    *slot = k < (unsigned)a.n_tiles ? (int)k : -1;
  }
  __syncthreads();
  const int k = *slot;
  __syncthreads();
  return k;
}

// The last CTA to finish resets the tile counter and advances the sweep and
// measurement counters for the next launch.
__device__ __forceinline__ void oq_batch_finish(const OqBatchArgs& a) {
  if (threadIdx.x != 0) return;
  __threadfence();
  const unsigned d = atomicAdd(&a.ctl->done, 1u);
  if (d == gridDim.x - 1) {
    a.ctl->next = 0u;
    a.ctl->done = 0u;
    a.ctl->step += (unsigned long long)a.n_sweeps;
    a.ctl->slot += (unsigned long long)(a.n_sweeps / a.measure_every);
    __threadfence();
  }
}

// Counters of this launch (written only by the previous launch's last CTA).
__device__ __forceinline__ void oq_batch_counters(const OqBatchArgs& a, uint64_t& step0,
                                                  uint64_t& slot0) {
  step0 = *reinterpret_cast<volatile unsigned long long*>(&a.ctl->step);
  slot0 = *reinterpret_cast<volatile unsigned long long*>(&a.ctl->slot);
}
