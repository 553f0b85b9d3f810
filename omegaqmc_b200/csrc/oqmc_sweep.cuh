// Single-electron Metropolis sweeps with Sherman-Morrison inverse updates.
//
// One thread per walker.  A CTA copies the system tables and its walkers'
// state (positions, the two inverse Slater matrices) into shared memory
// once, runs n_sweeps sweeps without touching HBM except to reduce the
// local energy of each measured sweep, and writes the state back at the end.
// Shared-memory walker arrays are walker-minor so that a warp's 32 walkers
// read 32 consecutive words.
//
// A sweep moves every electron once (Gaussian proposal of width `step`,
// exact Metropolis acceptance |R|^2 exp(2 dJ) with R the determinant ratio
// from the stored inverse) and then evaluates the local energy with the
// analytic Slater/Jastrow VGL, as the reference does after its move
// (OmegaQMC/vmc_gto.py:985-1034, psi/gto.py:2506-2579).  Proposals that
// land within MIN_DIST_THRESHOLD = 1e-4 bohr of a nucleus or another
// electron are rejected (vmc_gto.py:815-839, constants.py:23).
//
// Precision (template T/Real): T is the type of the AO/MO arithmetic and
// Real the storage type of the inverse.  FP64 build: T = Real = double.
// Mixed build: T = Real = float for moves and the MO VGL, with FP64 kept for
// positions, the periodic LU refresh (k_refresh), the Coulomb terms and all
// energy accumulation.  Exponent groups whose tightest exponent exceeds
// `tight` are evaluated in FP64 for electrons within the group's split
// radius of their nucleus (the large-exponent Laplacian term
// (4a^2 r^2 - 6a) e^{-a r^2} loses FP32 precision there).
#pragma once
#include "oqmc_eval.cuh"

template <typename T> __device__ __forceinline__ T oq_exp(T v);
template <> __device__ __forceinline__ double oq_exp<double>(double v) { return exp(v); }
template <> __device__ __forceinline__ float oq_exp<float>(float v) { return __expf(v); }

// per-group "tight" split radius squared (FP64 evaluation inside it);
// 0 disables.  Stored after the system struct in global memory.
struct OqSplit {
  double r2[OQ_MAX_GROUP];
};

// MO values at x in compute type T (accumulated in T).
template <int NOCC, typename T, typename TC>
__device__ __forceinline__ void oq_mo_val_t(const OqSystem& S, const OqSplit& SP,
                                            const TC* __restrict__ C, double x,
                                            double y, double z, T mv[NOCC]) {
#pragma unroll
  for (int m = 0; m < NOCC; ++m) mv[m] = (T)0;
  for (int g = 0; g < S.ngroup; ++g) {
    const int ia = S.g_iat[g];
    const double dxd = x - S.nuc[ia][0], dyd = y - S.nuc[ia][1], dzd = z - S.nuc[ia][2];
    const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
    const T dx = (T)dxd, dy = (T)dyd, dz = (T)dzd, r2 = (T)r2d;
    const int ncol = S.g_ncol[g], np = S.g_n[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    T R[OQ_MAX_COL] = {0, 0, 0, 0};
    for (int p = 0; p < np; ++p) {
      const T e = oq_exp<T>(-(T)S.alpha[off + p] * r2);
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol) R[k] += (T)S.norm[S.s_norm[sh0 + k] + p] * e;
    }
    const int am = S.g_am[g];
#pragma unroll
    for (int k = 0; k < OQ_MAX_COL; ++k) {
      if (k >= ncol) break;
      const int sh = sh0 + k;
      const int ao = S.s_ao[sh];
      if (am == 0) {
        T v = R[k];
        if (S.s_cusp[sh]) v = (T)oq_cusp_val(S, ia, sqrt(r2d), (double)v);
#pragma unroll
        for (int m = 0; m < NOCC; ++m) mv[m] += (T)C[ao * NOCC + m] * v;
      } else if (am == 1) {
        const T v0 = R[k] * dx, v1 = R[k] * dy, v2 = R[k] * dz;
#pragma unroll
        for (int m = 0; m < NOCC; ++m)
          mv[m] += (T)C[ao * NOCC + m] * v0 + (T)C[(ao + 1) * NOCC + m] * v1 +
                   (T)C[(ao + 2) * NOCC + m] * v2;
      } else if (am == 2) {
        T Y[5], dY[5][3];
        oq_harm_d<T>(dx, dy, dz, Y, dY);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
          const T v = R[k] * Y[c];
#pragma unroll
          for (int m = 0; m < NOCC; ++m) mv[m] += (T)C[(ao + c) * NOCC + m] * v;
        }
      } else {
        const int nc = 2 * am + 1;
        for (int c = 0; c < nc; ++c) {
          T Yc, dY[3];
          oq_harm_table<T>(S.harm, am, c, dx, dy, dz, Yc, dY);
          const T v = R[k] * Yc;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) mv[m] += (T)C[(ao + c) * NOCC + m] * v;
        }
      }
    }
  }
}

// MO value/gradient/Laplacian at x in compute type T.  Groups flagged tight
// (SP.r2[g] > r^2) run their radial part in FP64.
template <int NOCC, typename T, typename TC>
__device__ __forceinline__ void oq_mo_vgl_t(const OqSystem& S, const OqSplit& SP,
                                            const TC* __restrict__ C, double x,
                                            double y, double z, T mv[NOCC],
                                            T mg[NOCC][3], T ml[NOCC]) {
#pragma unroll
  for (int m = 0; m < NOCC; ++m) {
    mv[m] = (T)0; mg[m][0] = mg[m][1] = mg[m][2] = (T)0; ml[m] = (T)0;
  }
  for (int g = 0; g < S.ngroup; ++g) {
    const int ia = S.g_iat[g];
    const double dxd = x - S.nuc[ia][0], dyd = y - S.nuc[ia][1], dzd = z - S.nuc[ia][2];
    const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
    const T dx = (T)dxd, dy = (T)dyd, dz = (T)dzd;
    const int ncol = S.g_ncol[g], np = S.g_n[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    T R[OQ_MAX_COL], Rp[OQ_MAX_COL], Rl[OQ_MAX_COL];
    const bool fp64_radial = (sizeof(T) == 8) || (r2d < SP.r2[g]) || S.s_cusp[sh0];
    if (fp64_radial) {
      double Rd[OQ_MAX_COL] = {0, 0, 0, 0}, Rpd[OQ_MAX_COL] = {0, 0, 0, 0},
             Rld[OQ_MAX_COL] = {0, 0, 0, 0};
      for (int p = 0; p < np; ++p) {
        const double a = S.alpha[off + p];
        const double e = exp(-a * r2d);
        const double fp = -2.0 * a * e;
        const double fl = (4.0 * a * a * r2d - 6.0 * a) * e;
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
      for (int k = 0; k < OQ_MAX_COL; ++k) { R[k] = (T)Rd[k]; Rp[k] = (T)Rpd[k]; Rl[k] = (T)Rld[k]; }
    } else {
      const T r2 = (T)r2d;
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k) { R[k] = Rp[k] = Rl[k] = (T)0; }
      for (int p = 0; p < np; ++p) {
        const T a = (T)S.alpha[off + p];
        const T e = oq_exp<T>(-a * r2);
        const T fp = (T)-2 * a * e;
        const T fl = ((T)4 * a * a * r2 - (T)6 * a) * e;
#pragma unroll
        for (int k = 0; k < OQ_MAX_COL; ++k)
          if (k < ncol) {
            const T n = (T)S.norm[S.s_norm[sh0 + k] + p];
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
        const T v = R[k], l = Rl[k];
        const T gx = Rp[k] * dx, gy = Rp[k] * dy, gz = Rp[k] * dz;
#pragma unroll
        for (int m = 0; m < NOCC; ++m) {
          const T c = (T)C[ao * NOCC + m];
          mv[m] += c * v; mg[m][0] += c * gx; mg[m][1] += c * gy; mg[m][2] += c * gz;
          ml[m] += c * l;
        }
      } else {
        const int nc = 2 * am + 1;
        T Yd[5], dYd[5][3];
        if (am == 2) oq_harm_d<T>(dx, dy, dz, Yd, dYd);
        const T lfac = Rl[k] + (T)(2 * am) * Rp[k];
        for (int c = 0; c < nc; ++c) {
          T Y, dY[3];
          if (am == 1) {
            Y = (c == 0) ? dx : (c == 1) ? dy : dz;
            dY[0] = (T)(c == 0); dY[1] = (T)(c == 1); dY[2] = (T)(c == 2);
          } else if (am == 2) {
            Y = Yd[c]; dY[0] = dYd[c][0]; dY[1] = dYd[c][1]; dY[2] = dYd[c][2];
          } else {
            oq_harm_table<T>(S.harm, am, c, dx, dy, dz, Y, dY);
          }
          const T v = R[k] * Y;
          const T gx = Rp[k] * dx * Y + R[k] * dY[0];
          const T gy = Rp[k] * dy * Y + R[k] * dY[1];
          const T gz = Rp[k] * dz * Y + R[k] * dY[2];
          const T l = lfac * Y;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) {
            const T cc = (T)C[(ao + c) * NOCC + m];
            mv[m] += cc * v; mg[m][0] += cc * gx; mg[m][1] += cc * gy;
            mg[m][2] += cc * gz; ml[m] += cc * l;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Refresh: FP64 Slater matrices from positions, Gauss-Jordan inverse,
// stored as Real in the walker-minor state layout ainv[(s*N+m)*N+j][W].
// ---------------------------------------------------------------------------
template <int NOCC, typename Real>
__global__ void __launch_bounds__(128)
k_refresh(const OqSystem* __restrict__ gsys, const double* __restrict__ gC,
          const double* __restrict__ X, int W, Real* __restrict__ ainv,
          double* __restrict__ logdet, unsigned* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  double* C = reinterpret_cast<double*>(smem + sizeof(OqSystem));
  oq_load_system(&S, gsys);
  for (int i = threadIdx.x; i < S.nbf * NOCC; i += blockDim.x) C[i] = gC[i];
  __syncthreads();
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  constexpr int NE = 2 * NOCC;
  double ld_tot = 0.0;
  bool ok = true;
  for (int s = 0; s < 2; ++s) {
    double Sm[NOCC][NOCC], Ai[NOCC][NOCC];
    for (int i = 0; i < NOCC; ++i) {
      const int e = 2 * i + s;
      const double* xp = X + (size_t)w * 3 * NE + 3 * e;
      double mv[NOCC];
      oq_mo_val<NOCC>(S, C, xp[0], xp[1], xp[2], mv);
#pragma unroll
      for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
    }
    double ld;
    const bool oks = oq_invert<NOCC>(Sm, Ai, ld);
    ok = ok && oks;
    ld_tot += ld;
    for (int m = 0; m < NOCC; ++m)
      for (int j = 0; j < NOCC; ++j)
        ainv[(size_t)((s * NOCC + m) * NOCC + j) * W + w] = oks ? (Real)Ai[m][j] : (Real)0;
  }
  logdet[w] = ok ? ld_tot : -INFINITY;
  if (!ok) atomicOr(flags, OQ_FLAG_SINGULAR);
}

// number of doubles reduced per measured sweep
#define OQ_NSUM 8   // ee, en, ke, eloc, eloc^2, accepted moves, valid walkers, pad

struct OqSweepArgs {
  double* X;              // (W, n_e, 3) positions, in/out
  void* ainv;             // Real, walker-minor inverse state
  double* logdet;         // (W,) log|det up| + log|det down|
  int W;
  int n_sweeps;
  int measure_every;      // local energy after every k-th sweep (k >= 1)
  int pad;
  double step;
  uint64_t seed;
  uint64_t step_base;     // global sweep counter of the first sweep (RNG)
  double* sums;           // (n_meas, OQ_NSUM), accumulated with atomics
  double* el_trace;       // (n_meas, W) local energies or null
  double* eparts_last;    // (W, 4) ee, en, ke, eloc of the last measurement or null
  unsigned* flags;
};

template <int NOCC, typename T, typename Real>
__global__ void __launch_bounds__(128)
k_sweeps(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
         const void* __restrict__ gC, OqSweepArgs a) {
  constexpr int NE = 2 * NOCC;
  constexpr int NN = NOCC * NOCC;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  OqSplit& SP = *reinterpret_cast<OqSplit*>(smem + sizeof(OqSystem));
  unsigned char* p = smem + sizeof(OqSystem) + sizeof(OqSplit);
  Real* C = reinterpret_cast<Real*>(p);
  const int nbf = gsys->nbf;
  p += ((size_t)nbf * NOCC * sizeof(Real) + 15) & ~(size_t)15;
  const int WPB = blockDim.x;
  double* pos = reinterpret_cast<double*>(p);          // [3*NE][WPB]
  p += (size_t)3 * NE * WPB * sizeof(double);
  Real* Ai = reinterpret_cast<Real*>(p);                // [2*NN][WPB]

  oq_load_system(&S, gsys);
  {
    const double* src = reinterpret_cast<const double*>(gsplit);
    double* dst = reinterpret_cast<double*>(&SP);
    for (int i = threadIdx.x; i < OQ_MAX_GROUP; i += blockDim.x) dst[i] = src[i];
    const Real* gc = reinterpret_cast<const Real*>(gC);
    for (int i = threadIdx.x; i < nbf * NOCC; i += blockDim.x) C[i] = gc[i];
  }
  const int tid = threadIdx.x;
  const int w = blockIdx.x * WPB + tid;
  const bool live = w < a.W;
  const int W = a.W;
  const Real* gA = reinterpret_cast<const Real*>(a.ainv);
  if (live) {
    for (int k = 0; k < 3 * NE; ++k) pos[k * WPB + tid] = a.X[(size_t)w * 3 * NE + k];
    for (int k = 0; k < 2 * NN; ++k) Ai[k * WPB + tid] = gA[(size_t)k * W + w];
  }
  __syncthreads();
  double logdet = live ? a.logdet[w] : 0.0;
  unsigned bad = 0;
  const double thr2 = 1e-4 * 1e-4;
  int meas = 0;

  for (int sweep = 0; sweep < a.n_sweeps; ++sweep) {
    int nacc = 0;
    if (live) {
      const uint32_t gstep = (uint32_t)(a.step_base + sweep);
      for (int e = 0; e < NE; ++e) {
        const int s = e & 1, i = e >> 1;
        double n3[3], u;
        oq_move_randoms(a.seed, (uint32_t)w, gstep, (uint32_t)e, n3, u);
        const double ox = pos[(3 * e) * WPB + tid], oy = pos[(3 * e + 1) * WPB + tid],
                     oz = pos[(3 * e + 2) * WPB + tid];
        const double nx = ox + a.step * n3[0], ny = oy + a.step * n3[1],
                     nz = oz + a.step * n3[2];
        // Jastrow change and singularity check
        double dJ = 0.0;
        bool valid = true;
        for (int j = 0; j < NE; ++j) {
          if (j == e) continue;
          const double xj = pos[(3 * j) * WPB + tid], yj = pos[(3 * j + 1) * WPB + tid],
                       zj = pos[(3 * j + 2) * WPB + tid];
          const double ax = nx - xj, ay = ny - yj, az = nz - zj;
          const double bx = ox - xj, by = oy - yj, bz = oz - zj;
          const double rn2 = ax * ax + ay * ay + az * az;
          valid = valid && (rn2 >= thr2);
          if (S.has_j2) {
            const int o = ((e & 1) == (j & 1)) ? 0 : 2;
            dJ += oq_pade(S.j2[o], S.j2[o + 1], sqrt(rn2)) -
                  oq_pade(S.j2[o], S.j2[o + 1], sqrt(bx * bx + by * by + bz * bz));
          }
        }
        for (int I = 0; I < S.natm; ++I) {
          const double ax = nx - S.nuc[I][0], ay = ny - S.nuc[I][1], az = nz - S.nuc[I][2];
          const double rn2 = ax * ax + ay * ay + az * az;
          valid = valid && (rn2 >= thr2);
          if (S.has_j1) {
            const double bx = ox - S.nuc[I][0], by = oy - S.nuc[I][1], bz = oz - S.nuc[I][2];
            dJ += oq_pade(S.j1a[I], S.j1b[I], sqrt(rn2)) -
                  oq_pade(S.j1a[I], S.j1b[I], sqrt(bx * bx + by * by + bz * bz));
          }
        }
        // new MO row and determinant ratio against column i of the inverse
        T v[NOCC];
        oq_mo_val_t<NOCC, T, Real>(S, SP, C, nx, ny, nz, v);
        const Real* As = Ai + (size_t)s * NN * WPB;
        T wv[NOCC];
#pragma unroll
        for (int j = 0; j < NOCC; ++j) {
          T acc = (T)0;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) acc += v[m] * (T)As[(m * NOCC + j) * WPB + tid];
          wv[j] = acc;
        }
        T R = (T)0;
#pragma unroll
        for (int j = 0; j < NOCC; ++j) R = (j == i) ? wv[j] : R;
        const double Rd = (double)R;
        const double prob = Rd * Rd * exp(2.0 * dJ);
        const bool acc = valid && (u < prob) && (Rd != 0.0) && isfinite(prob);
        if (acc) {
          // Sherman-Morrison: A[k][j] -= A[k][i] (w_j - delta_ij) / R
          const T rinv = (T)1 / R;
          T coli[NOCC];
          Real* Aw = Ai + (size_t)s * NN * WPB;
#pragma unroll
          for (int k = 0; k < NOCC; ++k) {
            T c = (T)0;
#pragma unroll
            for (int j = 0; j < NOCC; ++j) c = (j == i) ? (T)Aw[(k * NOCC + j) * WPB + tid] : c;
            coli[k] = c;
          }
#pragma unroll
          for (int j = 0; j < NOCC; ++j) {
            const T f = (wv[j] - (j == i ? (T)1 : (T)0)) * rinv;
#pragma unroll
            for (int k = 0; k < NOCC; ++k) {
              Real& ref = Aw[(k * NOCC + j) * WPB + tid];
              ref = (Real)((T)ref - coli[k] * f);
            }
          }
          pos[(3 * e) * WPB + tid] = nx;
          pos[(3 * e + 1) * WPB + tid] = ny;
          pos[(3 * e + 2) * WPB + tid] = nz;
          logdet += log(fabs(Rd));
          ++nacc;
        }
      }
    }
    // ---- local energy of this sweep ----
    if (((sweep + 1) % a.measure_every) == 0) {
      double ee = 0.0, en = 0.0, ke = 0.0, el = 0.0;
      bool ok = live;
      if (live) {
        double lap_tot = 0.0, g2 = 0.0;
        for (int e = 0; e < NE; ++e) {
          const int s = e & 1, i = e >> 1;
          const double xe = pos[(3 * e) * WPB + tid], ye = pos[(3 * e + 1) * WPB + tid],
                       ze = pos[(3 * e + 2) * WPB + tid];
          T mv[NOCC], mg[NOCC][3], ml[NOCC];
          oq_mo_vgl_t<NOCC, T, Real>(S, SP, C, xe, ye, ze, mv, mg, ml);
          const Real* As = Ai + (size_t)s * NN * WPB;
          T gx = 0, gy = 0, gz = 0, lp = 0;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) {
            T am = (T)0;
#pragma unroll
            for (int j = 0; j < NOCC; ++j) am = (j == i) ? (T)As[(m * NOCC + j) * WPB + tid] : am;
            gx += am * mg[m][0]; gy += am * mg[m][1]; gz += am * mg[m][2];
            lp += am * ml[m];
          }
          double Gx = gx, Gy = gy, Gz = gz;
          double L = (double)lp - (Gx * Gx + Gy * Gy + Gz * Gz);
          for (int j = 0; j < NE; ++j) {
            if (j == e) continue;
            const double dx = xe - pos[(3 * j) * WPB + tid], dy = ye - pos[(3 * j + 1) * WPB + tid],
                         dz = ze - pos[(3 * j + 2) * WPB + tid];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (j > e) ee += 1.0 / sqrt(r2 + OQ_EPS);
            if (S.has_j2) {
              const int o = ((e & 1) == (j & 1)) ? 0 : 2;
              double upr, l;
              oq_pade_vgl(S.j2[o], S.j2[o + 1], sqrt(r2), upr, l);
              Gx += upr * dx; Gy += upr * dy; Gz += upr * dz; L += l;
            }
          }
          for (int I = 0; I < S.natm; ++I) {
            const double dx = xe - S.nuc[I][0], dy = ye - S.nuc[I][1], dz = ze - S.nuc[I][2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            en -= S.Z[I] / sqrt(r2 + OQ_EPS);
            if (S.has_j1) {
              double upr, l;
              oq_pade_vgl(S.j1a[I], S.j1b[I], sqrt(r2), upr, l);
              Gx += upr * dx; Gy += upr * dy; Gz += upr * dz; L += l;
            }
          }
          lap_tot += L;
          g2 += Gx * Gx + Gy * Gy + Gz * Gz;
        }
        ke = -0.5 * (lap_tot + g2);
        el = ee + en + ke + S.e_nn;
        ok = isfinite(el);
        if (!ok) bad |= OQ_FLAG_NAN;
        if (a.el_trace) a.el_trace[(size_t)meas * W + w] = el;
        if (a.eparts_last && meas * a.measure_every + a.measure_every >= a.n_sweeps) {
          double* ep = a.eparts_last + (size_t)w * 4;
          ep[0] = ee; ep[1] = en; ep[2] = ke; ep[3] = el;
        }
      }
      // fused walker reduction: warp shuffles, one atomic per warp and value
      double vals[7] = {ok ? ee : 0.0, ok ? en : 0.0, ok ? ke : 0.0, ok ? el : 0.0,
                        ok ? el * el : 0.0, (double)nacc, ok ? 1.0 : 0.0};
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        double v = vals[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        vals[k] = v;
      }
      if ((tid & 31) == 0) {
        double* dst = a.sums + (size_t)meas * OQ_NSUM;
#pragma unroll
        for (int k = 0; k < 7; ++k) atomicAdd(dst + k, vals[k]);
      }
      ++meas;
    }
  }
  if (live) {
    for (int k = 0; k < 3 * NE; ++k) a.X[(size_t)w * 3 * NE + k] = pos[k * WPB + tid];
    Real* gAw = reinterpret_cast<Real*>(a.ainv);
    for (int k = 0; k < 2 * NN; ++k) gAw[(size_t)k * W + w] = Ai[k * WPB + tid];
    a.logdet[w] = logdet;
  }
  if (bad) atomicOr(a.flags, bad);
}
