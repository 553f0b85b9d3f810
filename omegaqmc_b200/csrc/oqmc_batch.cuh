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

// ---------------------------------------------------------------------------
// Several threads per walker ("lanes").  A tile of WT walkers on NT threads
// gives each walker P = NT / WT consecutive lanes of one warp (P = 1, 2, 4
// or 8), lane = tid % P.  The move of one electron is sequential in the
// state (ratio against the current inverse, Jastrow change against the
// other electrons' current positions, Sherman-Morrison update), but its
// expensive part, the molecular-orbital row at the proposed position, is
// not: the proposal of electron e depends only on e's own position and its
// random numbers.  So a sweep runs in blocks of P electrons: each lane
// proposes one electron of the block and evaluates its orbital row (the
// same straight-line code on different data, no divergence), then the P
// moves are decided in order, every lane taking part: the owner lane's
// proposal and row are broadcast with shuffles, the Jastrow pairs and
// nuclei and the columns of the Sherman-Morrison update are split over the
// lanes, and sums are combined with xor-shuffles (the same result on every
// lane, so every lane takes the same decision).

// Sum / AND over the P lanes of a walker (identical result on every lane:
// each butterfly stage adds the same two values in either order).
template <typename V>
__device__ __forceinline__ V oq_lanes_sum(V v, int P) {
  for (int o = P >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ bool oq_lanes_and(bool b, int P) {
  int v = b ? 1 : 0;
  for (int o = P >> 1; o > 0; o >>= 1) v &= __shfl_xor_sync(0xffffffffu, v, o);
  return v != 0;
}

// This lane's share of the Jastrow change of electron e moving from o to n
// (pairs j = lane, lane + P, ...; nuclei I = lane, lane + P, ...; the
// three-body term on lane 0) and of the MIN_DIST_THRESHOLD test; the same
// terms as oq_jastrow_delta.
template <int NE, typename T, class SJ>
__device__ __forceinline__ T oq_jastrow_delta_lane(const SJ& J, const OqSystem& S,
                                                   const double* pos, int ps, int e, int lane,
                                                   int P, double ox, double oy, double oz,
                                                   double nx, double ny, double nz,
                                                   bool& valid) {
  const double thr2 = 1e-4 * 1e-4;
  T dJ = (T)0;
  valid = true;
  for (int j = lane; j < NE; j += P) {
    if (j == e) continue;
    const double xj = pos[(3 * j) * ps], yj = pos[(3 * j + 1) * ps], zj = pos[(3 * j + 2) * ps];
    const double ax = nx - xj, ay = ny - yj, az = nz - zj;
    const double rn2 = ax * ax + ay * ay + az * az;
    valid = valid && (rn2 >= thr2);
    const double bx = ox - xj, by = oy - yj, bz = oz - zj;
    const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
    const bool like = (e & 1) == (j & 1);
    if (J.has_j2) {
      const int o = like ? 0 : 2;
      dJ += oq_pade_diff((T)J.j2[o], (T)J.j2[o + 1], rn2t * oq_rsqrt(rn2t),
                         ro2t * oq_rsqrt(ro2t));
    }
    if (S.has_bs2) {
      const double* c = like ? S.bs2_like : S.bs2_unlike;
      const int n = like ? S.bs2_n_like : S.bs2_n_unlike;
      const T dinv = (T)(like ? S.bs2_dinv_like : S.bs2_dinv_unlike), rc = (T)S.bs2_rcut;
      dJ += oq_bs_val<T>(c, n, dinv, rc, rn2t * oq_rsqrt(rn2t)) -
            oq_bs_val<T>(c, n, dinv, rc, ro2t * oq_rsqrt(ro2t));
    }
  }
  for (int I = lane; I < J.natm; I += P) {
    const double ax = nx - J.nuc[I][0], ay = ny - J.nuc[I][1], az = nz - J.nuc[I][2];
    const double rn2 = ax * ax + ay * ay + az * az;
    valid = valid && (rn2 >= thr2);
    const double bx = ox - J.nuc[I][0], by = oy - J.nuc[I][1], bz = oz - J.nuc[I][2];
    const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
    if (J.has_j1)
      dJ += oq_pade_diff((T)J.j1a[I], (T)J.j1b[I], rn2t * oq_rsqrt(rn2t), ro2t * oq_rsqrt(ro2t));
    if (S.has_bs1 && S.bs1_type[I] >= 0) {
      const int ty = S.bs1_type[I];
      const T dinv = (T)S.bs1_dinv[ty], rc = (T)S.bs1_rcut[ty];
      dJ += oq_bs_val<T>(S.bs1_c[ty], S.bs1_n[ty], dinv, rc, rn2t * oq_rsqrt(rn2t)) -
            oq_bs_val<T>(S.bs1_c[ty], S.bs1_n[ty], dinv, rc, ro2t * oq_rsqrt(ro2t));
    }
  }
  if (S.has_j3 && lane == 0)
    dJ -= oq_j3_electron<T>(S, pos, (size_t)ps, NE, e, 0, nx, ny, nz) -
          oq_j3_electron<T>(S, pos, (size_t)ps, NE, e, 0, ox, oy, oz);
  return dJ;
}

// One sweep of walker wl on its P lanes (P >= 2); returns the accepted
// moves on lane 0 (0 on the other lanes).  Every lane of the warp runs the
// same loop trip counts; walkers beyond the tile (live = false) never
// accept.
template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ int oq_batch_sweep_lanes(const OqBatchArgs& a, const OqBatchSys& d,
                                                    const SJ& J, const OqSystem& S,
                                                    const OqSplit& SP, const Real* C,
                                                    double* pos, Real* Ai, int WT, int wl,
                                                    int lane, int P, bool live, uint32_t w,
                                                    uint32_t gstep, const OqScaledF& pf,
                                                    double& logdet) {
  constexpr int NE = 2 * NOCC;
  constexpr int NN = NOCC * NOCC;
  int nacc = 0;
  for (int e0 = 0; e0 < NE; e0 += P) {
    // this lane's electron of the block: proposal and orbital row
    const int e = e0 + lane;
    double nx = 0.0, ny = 0.0, nz = 0.0;
    T u = (T)2, mul = (T)1, lx = (T)0;
    T v[NOCC];
#pragma unroll
    for (int m = 0; m < NOCC; ++m) v[m] = (T)0;
    if (live && e < NE) {
      float nf[3];
      uint32_t ub;
      oq_move_normals(a.seed, w, gstep, (uint32_t)e, nf, ub);
      u = oq_uniform<T>(ub);
      const double ox = pos[(3 * e) * WT + wl], oy = pos[(3 * e + 1) * WT + wl],
                   oz = pos[(3 * e + 2) * WT + wl];
      if (d.proposal == 0) {
        nx = ox + d.step * (double)nf[0];
        ny = oy + d.step * (double)nf[1];
        nz = oz + d.step * (double)nf[2];
      } else {
        oq_scaled_propose_t<T>(J, ox, oy, oz, nf, pf, nx, ny, nz, mul, lx);
      }
      B::template mo_val<T, Real>(S, SP, C, nx, ny, nz, v);
    }
    // the block's moves in order
    const int nb = min(P, NE - e0);
    for (int q = 0; q < nb; ++q) {
      const int ee = e0 + q, s = ee & 1, i = ee >> 1;
      const double bx = __shfl_sync(0xffffffffu, nx, q, P);
      const double by = __shfl_sync(0xffffffffu, ny, q, P);
      const double bz = __shfl_sync(0xffffffffu, nz, q, P);
      const T bu = __shfl_sync(0xffffffffu, u, q, P);
      const T bmul = __shfl_sync(0xffffffffu, mul, q, P);
      const T blx = __shfl_sync(0xffffffffu, lx, q, P);
      T bv[NOCC];
#pragma unroll
      for (int m = 0; m < NOCC; ++m) bv[m] = __shfl_sync(0xffffffffu, v[m], q, P);
      const double ox = pos[(3 * ee) * WT + wl], oy = pos[(3 * ee + 1) * WT + wl],
                   oz = pos[(3 * ee + 2) * WT + wl];
      bool valid;
      T dJ = oq_jastrow_delta_lane<NE, T>(J, S, pos + wl, WT, ee, lane, P, ox, oy, oz, bx, by,
                                          bz, valid);
      dJ = oq_lanes_sum(dJ, P);
      valid = oq_lanes_and(valid, P);
      Real* As = Ai + (size_t)s * NN * WT;
      T R = (T)0;
      T coli[NOCC];
#pragma unroll
      for (int k = 0; k < NOCC; ++k) {
        coli[k] = (T)As[(k * NOCC + i) * WT + wl];
        R += bv[k] * coli[k];
      }
      const bool acc = live && oq_accept<T>(R, dJ, blx, bmul, bu, valid);
      // every lane has read column i before any lane updates it
      __syncwarp();
      if (acc) {
        const T rinv = oq_rcp(R);
        for (int j = lane; j < NOCC; j += P) {
          T wj = (T)0;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) wj += bv[m] * (T)As[(m * NOCC + j) * WT + wl];
          const T f = (wj - (j == i ? (T)1 : (T)0)) * rinv;
#pragma unroll
          for (int k = 0; k < NOCC; ++k) {
            Real& ref = As[(k * NOCC + j) * WT + wl];
            ref = (Real)((T)ref - coli[k] * f);
          }
        }
        if (lane == 0) {
          pos[(3 * ee) * WT + wl] = bx;
          pos[(3 * ee + 1) * WT + wl] = by;
          pos[(3 * ee + 2) * WT + wl] = bz;
          ++nacc;
        }
        logdet += log(fabs((double)R));
      }
      // the move is visible to every lane before the next one
      __syncwarp();
    }
  }
  return nacc;
}

// Shared memory of one tile: [positions [3 NE][WT] doubles][inverses
// [2 NOCC^2][WT] Real].  The nuclei and Jastrow constants (J) are the
// system's OqJas in constant memory, written into the generated module, so
// every lane of a warp reads the same word (a broadcast) and the tile's
// shared memory holds walker state only.  With P = NT / WT lanes per walker
// (see above) the refresh splits the two spin blocks over lanes 0 and 1,
// the sweeps run in blocks of P electrons and the local energy splits the
// electrons over the lanes; lane sums are combined with shuffles.
// MODE selects the move code compiled in: 0 both (lanes chosen at run time),
// 1 one lane per walker only, 2 several lanes only (the module generated
// after tuning, when every molecule's lane count is fixed).
template <int NOCC, typename T, typename Real, class B, int MODE = 0, class SJ>
__device__ __forceinline__ void oq_batch_tile(const OqBatchArgs& a, const OqBatchSys& d,
                                              const SJ& J, int w0, uint64_t step0,
                                              uint64_t slot0, unsigned char* smem) {
  constexpr int NE = 2 * NOCC;
  const int NT = blockDim.x, tid = threadIdx.x, WT = d.wt;
  const int P = NT / WT, lane = tid & (P - 1), wl = tid / P;
  double* pos = reinterpret_cast<double*>(smem);                    // [3 NE][WT]
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
      const int wq = q / (3 * NE), k = q - wq * 3 * NE;
      pos[k * WT + wq] = src[q];
    }
  }
  __syncthreads();
  const bool live = wl < cnt;
  const int w = w0 + wl;
  double logdet = 0.0;
  {
    // FP64 refresh of the spin blocks (as k_refresh): both on the walker's
    // thread when P = 1, spin s on lane s otherwise
    bool ok = true;
    if (live && lane < 2) {
      for (int s = (P == 1 ? 0 : lane); s < (P == 1 ? 2 : lane + 1); ++s) {
        double Sm[NOCC][NOCC], Ainv[NOCC][NOCC];
        for (int i = 0; i < NOCC; ++i) {
          const int e = 2 * i + s;
          double mv[NOCC];
          oq_mo_val<NOCC>(S, d.C64, pos[(3 * e) * WT + wl], pos[(3 * e + 1) * WT + wl],
                          pos[(3 * e + 2) * WT + wl], mv);
#pragma unroll
          for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
        }
        double ld;
        const bool oks = oq_invert<NOCC>(Sm, Ainv, ld);
        ok = ok && oks;
        logdet += ld;
        for (int m = 0; m < NOCC; ++m)
          for (int j = 0; j < NOCC; ++j)
            Ai[((s * NOCC + m) * NOCC + j) * WT + wl] = oks ? (Real)Ainv[m][j] : (Real)0;
      }
    }
    if (P > 1) {
      logdet = oq_lanes_sum(logdet, P);
      ok = oq_lanes_and(ok, P);
    }
    if (live && !ok) {
      logdet = -INFINITY;
      if (lane == 0) atomicOr(a.flags, OQ_FLAG_SINGULAR);
    }
  }
  __syncthreads();
  int nacc = 0, meas = 0;
  const OqScaledF pf = oq_scaled_f(d.step, d.scale_r0, d.scale_fmin);
  for (int t = 0; t < a.n_sweeps; ++t) {
    const uint32_t gstep = (uint32_t)(step0 + t);
    if (MODE != 1 && P > 1) {
      nacc += oq_batch_sweep_lanes<NOCC, T, Real, B>(a, d, J, S, SP, C, pos, Ai, WT, wl, lane,
                                                     P, live, (uint32_t)w, gstep, pf, logdet);
    } else if (MODE != 2 && live) {
      for (int e = 0; e < NE; ++e) {
        float nf[3];
        uint32_t ub;
        oq_move_normals(a.seed, (uint32_t)w, gstep, (uint32_t)e, nf, ub);
        const T u = oq_uniform<T>(ub);
        const double ox = pos[(3 * e) * WT + wl], oy = pos[(3 * e + 1) * WT + wl],
                     oz = pos[(3 * e + 2) * WT + wl];
        if (d.proposal == 0) {
          nacc += oq_try_move<NOCC, T, Real, B>(J, S, SP, C, pos, Ai, WT, wl, e,
                                                ox + d.step * (double)nf[0],
                                                oy + d.step * (double)nf[1],
                                                oz + d.step * (double)nf[2], (T)0, (T)1, u,
                                                logdet);
        } else {
          double nx, ny, nz;
          T mul, lx;
          oq_scaled_propose_t<T>(J, ox, oy, oz, nf, pf, nx, ny, nz, mul, lx);
          nacc += oq_try_move<NOCC, T, Real, B>(J, S, SP, C, pos, Ai, WT, wl, e, nx, ny, nz, lx,
                                                mul, u, logdet);
        }
      }
    }
    if ((t + 1) % a.measure_every != 0) continue;
    // a walker's state is read and written only by its own lanes, which
    // share one warp: the moves are complete for them after a warp barrier
    __syncwarp();
    // local energy: electrons e = lane, lane + P, ... of walker wl
    double see = 0.0, sen = 0.0, slp = 0.0, sg2 = 0.0;
    if (live)
      for (int e = lane; e < NE; e += P)
        oq_eloc_electron<NOCC, T, Real, B>(J, S, SP, C, pos + wl, (size_t)WT, Ai + wl,
                                           (size_t)WT, e, see, sen, slp, sg2);
    if (P > 1) {
      see = oq_lanes_sum(see, P);
      sen = oq_lanes_sum(sen, P);
      slp = oq_lanes_sum(slp, P);
      sg2 = oq_lanes_sum(sg2, P);
    }
    {
      const double ke = -0.5 * (slp + sg2);
      const double el = see + sen + ke + J.e_nn;
      const bool mine = live && lane == 0;
      const bool ok = mine && isfinite(el);
      if (mine && !ok) atomicOr(a.flags, OQ_FLAG_NAN);
      double vals[7] = {ok ? see : 0.0, ok ? sen : 0.0, ok ? ke : 0.0, ok ? el : 0.0,
                        ok ? el * el : 0.0, lane == 0 ? (double)nacc : 0.0, ok ? 1.0 : 0.0};
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
    // the next sweep's moves change state this measurement read (the lanes
    // of a walker share one warp)
    __syncwarp();
    nacc = 0;
    ++meas;
  }
  __syncthreads();
  {
    double* dst = d.walkers + (size_t)w0 * 3 * NE;
    for (int q = tid; q < cnt * 3 * NE; q += NT) {
      const int wq = q / (3 * NE), k = q - wq * 3 * NE;
      dst[q] = pos[k * WT + wq];
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
