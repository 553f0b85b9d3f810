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

// exp(-a r2) of a basis primitive in the generated code, given a and
// al2 = a log2(e) as literals: FP64 exp in the FP64 build; in FP32 the
// power of two 2^(-al2 r2) straight from the hardware approximation
// (ex2.approx, relative error ~2^-22), one multiply per primitive.
template <typename T> __device__ __forceinline__ T oq_exp_neg(T a, T al2, T r2);
template <> __device__ __forceinline__ double oq_exp_neg<double>(double a, double, double r2) {
  return exp(-a * r2);
}
template <> __device__ __forceinline__ float oq_exp_neg<float>(float, float al2, float r2) {
  float p;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p) : "f"(-al2 * r2));
  return p;
}

// exp(-a r2d) for a tight exponent a, the argument formed in FP64 (in FP32
// the rounding of a large argument would dominate the error), given a and
// al2 = a log2(e) as literals.  FP32 form: t = al2 r2d = k + f with k the
// nearest integer, taken by adding 1.5 * 2^52 (t < 2^51, so the sum is an
// integer whose low word is k: no conversion instruction) and f = t - k in
// [-1/2, 1/2] exactly; only 2^-f is evaluated in FP32 (ex2.approx), then
// scaled by 2^-k through the exponent field.  FP32 relative accuracy for
// every argument, without an FP64 exponential or a branch.
template <typename T> __device__ __forceinline__ T oq_exp_tight(double a, double al2, double r2d);
template <> __device__ __forceinline__ double oq_exp_tight<double>(double a, double, double r2d) {
  return exp(-(a * r2d));
}
template <> __device__ __forceinline__ float oq_exp_tight<float>(double, double al2, double r2d) {
  const double shift = 6755399441055744.0;                    // 1.5 * 2^52
  const double t = fmin(al2 * r2d, 125.0);                    // >= 0; 2^-125 is a normal float
  const double y = t + shift;
  const int k = __double2loint(y);                            // round(t), in [0, 125]
  const float f = (float)(t - (y - shift));                  // exact, in [-1/2, 1/2]
  float p;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(p) : "f"(-f));
  return p * __int_as_float((127 - k) << 23);                // 2^-k
}

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
    if (S.has_spl) {
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol && S.s_spl[sh0 + k] >= 0) {
          double gv, gp, gpp;
          oq_spline_gdd(S, S.s_spl[sh0 + k], r2d, gv, gp, gpp);
          R[k] = (T)gv;
        }
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
    if (S.has_spl) {
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol && S.s_spl[sh0 + k] >= 0) {
          double gv, gp, gpp;
          oq_spline_gdd(S, S.s_spl[sh0 + k], r2d, gv, gp, gpp);
          R[k] = (T)gv;
          Rp[k] = (T)(2.0 * gp);
          Rl[k] = (T)(6.0 * gp + 4.0 * r2d * gpp);
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

// Basis policy: how a kernel evaluates the occupied MOs at one position.
// OqBasisTable reads the system tables (any molecule); a per-system policy
// generated at run time (oqmc_specialize) has the same two members with the
// exponents and coefficients compiled in.
template <int NOCC>
struct OqBasisTable {
  template <typename T, typename TC>
  __device__ static __forceinline__ void mo_val(const OqSystem& S, const OqSplit& SP,
                                                const TC* __restrict__ C, double x, double y,
                                                double z, T* mv) {
    oq_mo_val_t<NOCC, T, TC>(S, SP, C, x, y, z, mv);
  }
  template <typename T, typename TC>
  __device__ static __forceinline__ void mo_vgl(const OqSystem& S, const OqSplit& SP,
                                                const TC* __restrict__ C, double x, double y,
                                                double z, T* mv, T (*mg)[3], T* ml) {
    oq_mo_vgl_t<NOCC, T, TC>(S, SP, C, x, y, z, mv, mg, ml);
  }
  // gradient and Laplacian of sum_m ac[m] phi_m
  template <typename T, typename TC>
  __device__ static __forceinline__ void mo_vgl_contract(const OqSystem& S, const OqSplit& SP,
                                                         const TC* __restrict__ C, double x,
                                                         double y, double z, const T* ac, T& gx,
                                                         T& gy, T& gz, T& lp) {
    T mv[NOCC], mg[NOCC][3], ml[NOCC];
    oq_mo_vgl_t<NOCC, T, TC>(S, SP, C, x, y, z, mv, mg, ml);
    gx = gy = gz = lp = (T)0;
#pragma unroll
    for (int m = 0; m < NOCC; ++m) {
      gx += ac[m] * mg[m][0]; gy += ac[m] * mg[m][1]; gz += ac[m] * mg[m][2];
      lp += ac[m] * ml[m];
    }
  }
};

// ---------------------------------------------------------------------------
// Sampler state in global memory, walker-minor so consecutive threads
// (walkers) touch consecutive words:
//   pos    [3*NE][W] double        positions, pos[(3e+c)*W + w]
//   ainv   [2*N*N][W] Real         ainv[((s*N + m)*N + j)*W + w] = (S_s^-1)[m][j]
//   logdet [W] double              log|det up| + log|det down|
// ---------------------------------------------------------------------------

// Refresh: FP64 Slater matrices from positions, Gauss-Jordan inverse,
// stored as Real.  One thread per walker.
template <int NOCC, typename Real>
__global__ void __launch_bounds__(128)
k_refresh(const OqSystem* __restrict__ gsys, const double* __restrict__ gC,
          const double* __restrict__ pos, int W, Real* __restrict__ ainv,
          double* __restrict__ logdet, unsigned* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  double* C = reinterpret_cast<double*>(smem + sizeof(OqSystem));
  oq_load_system(&S, gsys);
  // the count comes from global memory: the shared copy S is complete only
  // after the barrier below
  const int nbf_g = gsys->nbf;
  for (int i = threadIdx.x; i < nbf_g * NOCC; i += blockDim.x) C[i] = gC[i];
  __syncthreads();
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  double ld_tot = 0.0;
  bool ok = true;
  for (int s = 0; s < 2; ++s) {
    double Sm[NOCC][NOCC], Ai[NOCC][NOCC];
    for (int i = 0; i < NOCC; ++i) {
      const int e = 2 * i + s;
      double mv[NOCC];
      oq_mo_val<NOCC>(S, C, pos[(size_t)(3 * e) * W + w], pos[(size_t)(3 * e + 1) * W + w],
                      pos[(size_t)(3 * e + 2) * W + w], mv);
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

// All-electron Metropolis steps, the reference's move (metropolis_move_alle
// and metropolis_move_1w, OmegaQMC/vmc_gto.py:815-905): every electron is
// displaced by step * N(0, 1); a proposal with an electron-electron or
// electron-nucleus distance below 1e-4 bohr is rejected (ratio 0,
// constants.py:23); otherwise it is accepted when u < exp(2 (ln|psi'| -
// ln|psi|)), ln|psi| = log|det up| + log|det down| + J evaluated afresh in
// FP64 (Gauss-Jordan inverses of the proposed Slater matrices, which become
// the state's inverses on acceptance).  Random numbers: electron e's
// normals from the Philox block (walker, step, e, 0), u from electron 0's
// block.  One thread per walker, state in global memory (layout above).
template <int NOCC, typename Real>
__global__ void __launch_bounds__(128)
k_moves_alle(const OqSystem* __restrict__ gsys, const double* __restrict__ gC, double* pos,
             Real* __restrict__ ainv, double* __restrict__ logdet, int W, int n_steps,
             double step, uint64_t seed, uint64_t step_base, double* acc_sum,
             unsigned* __restrict__ flags) {
  constexpr int NE = 2 * NOCC;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  double* C = reinterpret_cast<double*>(smem + sizeof(OqSystem));
  oq_load_system(&S, gsys);
  // the count comes from global memory: the shared copy S is complete only
  // after the barrier below
  const int nbf_g = gsys->nbf;
  for (int i = threadIdx.x; i < nbf_g * NOCC; i += blockDim.x) C[i] = gC[i];
  __syncthreads();
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = w < W;
  int nacc = 0;
  if (live) {
    double x[3 * NE];
    for (int k = 0; k < 3 * NE; ++k) x[k] = pos[(size_t)k * W + w];
    double lpsi = logdet[w] + oq_jastrow_value(S, x, NE);
    for (int t = 0; t < n_steps; ++t) {
      const uint32_t gstep = (uint32_t)(step_base + t);
      double xn[3 * NE], u = 0.0;
      for (int e = 0; e < NE; ++e) {
        double n3[3], ue;
        oq_move_randoms(seed, (uint32_t)w, gstep, (uint32_t)e, n3, ue);
        if (e == 0) u = ue;
        for (int c = 0; c < 3; ++c) xn[3 * e + c] = x[3 * e + c] + step * n3[c];
      }
      bool valid = true;
      for (int i = 0; i < NE; ++i) {
        for (int j = i + 1; j < NE; ++j) {
          const double dx = xn[3 * i] - xn[3 * j], dy = xn[3 * i + 1] - xn[3 * j + 1],
                       dz = xn[3 * i + 2] - xn[3 * j + 2];
          valid = valid && (dx * dx + dy * dy + dz * dz >= 1e-8);
        }
        for (int I = 0; I < S.natm; ++I) {
          const double dx = xn[3 * i] - S.nuc[I][0], dy = xn[3 * i + 1] - S.nuc[I][1],
                       dz = xn[3 * i + 2] - S.nuc[I][2];
          valid = valid && (dx * dx + dy * dy + dz * dz >= 1e-8);
        }
      }
      if (!valid) continue;
      double An[2][NOCC][NOCC], ld = 0.0;
      bool ok = true;
      for (int s = 0; s < 2; ++s) {
        double Sm[NOCC][NOCC];
        for (int i = 0; i < NOCC; ++i) {
          const int e = 2 * i + s;
          double mv[NOCC];
          oq_mo_val<NOCC>(S, C, xn[3 * e], xn[3 * e + 1], xn[3 * e + 2], mv);
#pragma unroll
          for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
        }
        double lds;
        ok = ok && oq_invert<NOCC>(Sm, An[s], lds);
        ld += lds;
      }
      if (!ok) continue;
      const double lpn = ld + oq_jastrow_value(S, xn, NE);
      if (!isfinite(lpn)) { atomicOr(flags, OQ_FLAG_NAN); continue; }
      // an old state with psi = 0 (log -inf) accepts any finite proposal
      if (isfinite(lpsi) && !(log(u) < 2.0 * (lpn - lpsi))) continue;
      ++nacc;
      lpsi = lpn;
      for (int k = 0; k < 3 * NE; ++k) x[k] = xn[k];
      for (int s = 0; s < 2; ++s)
        for (int m = 0; m < NOCC; ++m)
          for (int j = 0; j < NOCC; ++j)
            ainv[(size_t)((s * NOCC + m) * NOCC + j) * W + w] = (Real)An[s][m][j];
      logdet[w] = ld;
    }
    for (int k = 0; k < 3 * NE; ++k) pos[(size_t)k * W + w] = x[k];
  }
  if (acc_sum) {
    double v = (double)nacc * NE;   // accepted electron moves, as the sweeps count them
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc_sum, v);
  }
}

// number of doubles reduced per measured sweep
#define OQ_NSUM 8   // ee, en, ke, eloc, eloc^2, accepted moves, finite walkers, pad

struct OqMoveArgs {
  double* pos;            // state positions (SoA)
  void* ainv;             // state inverses (Real, SoA)
  double* logdet;
  int W;
  int n_steps;            // sweeps (mode 0) or basin relocations (mode 1)
  int mode;               // 0: Gaussian single-electron sweeps; 1: basin relocation
  int proposal;           // mode 0: 0 = fixed width, 1 = nucleus-scaled width
  double step;            // Gaussian width (mode 0) or blob width sigma (mode 1)
  double scale_r0;        // nucleus-scaled width: sigma = step * clamp(r_near/r0, fmin, 1)
  double scale_fmin;
  uint64_t seed;
  uint64_t step_base;     // RNG counter of the first step
  double* acc_sum;        // += accepted moves (may be null)
  unsigned* flags;
  const double* step_dev; // when set, the Gaussian width is read here (device-side step
                          // adaptation, oqmc_equilibrate); else `step`
};

// The nucleus-scaled proposal's constants in FP32 (set once per launch or tile).
struct OqScaledF {
  float step, inv_r0, fmin;
};
__device__ __forceinline__ OqScaledF oq_scaled_f(double step, double r0, double fmn) {
  return {(float)step, 1.0f / (float)r0, (float)fmn};
}

// Proposal width at x for the nucleus-scaled Gaussian move,
// sigma(x) = step * clamp(r_near(x) / r0, fmin, 1): the nearest nucleus's
// squared distance in FP64, then sqrt.approx, the clamp and the product in
// FP32.  The width only has to be the same function of position on both
// sides of the ratio; the FP64 and the mixed samplers use this same
// function, so for the same random numbers they propose the same positions.
template <class SJ>
__device__ __forceinline__ float oq_scaled_width_f(const SJ& S, double x, double y, double z,
                                                   const OqScaledF& p) {
  double r2 = 1e300;
  for (int I = 0; I < S.natm; ++I) {
    const double dx = x - S.nuc[I][0], dy = y - S.nuc[I][1], dz = z - S.nuc[I][2];
    r2 = fmin(r2, dx * dx + dy * dy + dz * dz);
  }
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"((float)r2));
  return p.step * fminf(1.0f, fmaxf(p.fmin, r * p.inv_r0));
}

template <class SJ>
__device__ __forceinline__ double oq_scaled_width(const SJ& S, double x, double y,
                                                  double z, double step, double r0,
                                                  double fmn) {
  return (double)oq_scaled_width_f(S, x, y, z, oq_scaled_f(step, r0, fmn));
}

// Nucleus-scaled Gaussian proposal from (ox, oy, oz) with the FP32 standard
// normals nf: the new position (FP64) and the proposal-density ratio
// q(old | new) / q(new | old) = (so / sn)^3 exp(d^2 (1 / so^2 - 1 / sn^2) / 2),
// with d = so n: (so / sn)^3 exp(|n|^2 (1 - (so / sn)^2) / 2), returned as a
// factor mul and an exponent lx (no logarithm on the move path), in the
// working precision T (FP32 in the mixed build: its rounding, ~1e-7
// relative, is far below any statistical resolution).
template <typename T, class SJ>
__device__ __forceinline__ void oq_scaled_propose_t(const SJ& S, double ox, double oy, double oz,
                                                    const float nf[3], const OqScaledF& pf,
                                                    double& nx, double& ny, double& nz, T& mul,
                                                    T& lx) {
  const float so = oq_scaled_width_f(S, ox, oy, oz, pf);
  const double sod = (double)so;
  nx = ox + sod * (double)nf[0];
  ny = oy + sod * (double)nf[1];
  nz = oz + sod * (double)nf[2];
  const float sn = oq_scaled_width_f(S, nx, ny, nz, pf);
  if (sizeof(T) == 8) {
    const double q = sod / (double)sn;
    const double n2 = (double)nf[0] * (double)nf[0] + (double)nf[1] * (double)nf[1] +
                      (double)nf[2] * (double)nf[2];
    mul = (T)(q * q * q);
    lx = (T)(0.5 * n2 * (1.0 - q * q));
  } else {
    const float q = so * oq_rcp(sn);
    mul = (T)(q * q * q);
    lx = (T)(0.5f * (nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2]) * (1.0f - q * q));
  }
}

// The Metropolis-Hastings test u < |R|^2 exp(2 dJ + log_extra) mul_extra in
// the working precision T (FP32 in the mixed build: the accurate expf, whose
// ~1e-7 relative error moves acceptance probabilities far below any
// statistical resolution), without logarithms.
template <typename T>
__device__ __forceinline__ bool oq_accept(T R, T dJ, T log_extra, T mul_extra, T u, bool valid) {
  const T ex = (sizeof(T) == 8) ? (T)exp((double)((T)2 * dJ + log_extra))
                                : (T)expf((float)((T)2 * dJ + log_extra));
  const T ratio = R * R * mul_extra * ex;
  return valid && (R != (T)0) && isfinite(R) && isfinite(dJ) && isfinite(log_extra) &&
         (u < ratio);
}

// Change of the Jastrow factor (arithmetic in T) when electron e moves from
// (ox, oy, oz) to (nx, ny, nz), and the MIN_DIST_THRESHOLD test of the new
// position (FP64; OmegaQMC/constants.py:23): valid is cleared when an
// electron-electron or electron-nucleus distance falls below 1e-4.  The
// other electrons' coordinate c is pos[(3 j + c) * ps].
template <int NE, typename T, class SJ>
__device__ __forceinline__ T oq_jastrow_delta(const SJ& J, const OqSystem& S, const double* pos,
                                              int ps, int e, double ox, double oy, double oz,
                                              double nx, double ny, double nz, bool& valid) {
  const double thr2 = 1e-4 * 1e-4;
  T dJ = (T)0;
  valid = true;
  for (int j = 0; j < NE; ++j) {
    if (j == e) continue;
    const double xj = pos[(3 * j) * ps], yj = pos[(3 * j + 1) * ps], zj = pos[(3 * j + 2) * ps];
    const double ax = nx - xj, ay = ny - yj, az = nz - zj;
    const double rn2 = ax * ax + ay * ay + az * az;
    valid = valid && (rn2 >= thr2);
    if (J.has_j2) {
      const double bx = ox - xj, by = oy - yj, bz = oz - zj;
      const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
      const int o = ((e & 1) == (j & 1)) ? 0 : 2;
      const T pa = (T)J.j2[o], pb = (T)J.j2[o + 1];
      dJ += oq_pade_diff(pa, pb, rn2t * oq_rsqrt(rn2t), ro2t * oq_rsqrt(ro2t));
    }
    if (S.has_bs2) {
      const double bx = ox - xj, by = oy - yj, bz = oz - zj;
      const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
      const bool like = (e & 1) == (j & 1);
      const double* c = like ? S.bs2_like : S.bs2_unlike;
      const int n = like ? S.bs2_n_like : S.bs2_n_unlike;
      const T dinv = (T)(like ? S.bs2_dinv_like : S.bs2_dinv_unlike), rc = (T)S.bs2_rcut;
      dJ += oq_bs_val<T>(c, n, dinv, rc, rn2t * oq_rsqrt(rn2t)) -
            oq_bs_val<T>(c, n, dinv, rc, ro2t * oq_rsqrt(ro2t));
    }
  }
  for (int I = 0; I < J.natm; ++I) {
    const double ax = nx - J.nuc[I][0], ay = ny - J.nuc[I][1], az = nz - J.nuc[I][2];
    const double rn2 = ax * ax + ay * ay + az * az;
    valid = valid && (rn2 >= thr2);
    if (J.has_j1) {
      const double bx = ox - J.nuc[I][0], by = oy - J.nuc[I][1], bz = oz - J.nuc[I][2];
      const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
      const T pa = (T)J.j1a[I], pb = (T)J.j1b[I];
      dJ += oq_pade_diff(pa, pb, rn2t * oq_rsqrt(rn2t), ro2t * oq_rsqrt(ro2t));
    }
    if (S.has_bs1 && S.bs1_type[I] >= 0) {
      const int ty = S.bs1_type[I];
      const double bx = ox - J.nuc[I][0], by = oy - J.nuc[I][1], bz = oz - J.nuc[I][2];
      const T rn2t = (T)rn2, ro2t = (T)(bx * bx + by * by + bz * bz);
      const T dinv = (T)S.bs1_dinv[ty], rc = (T)S.bs1_rcut[ty];
      dJ += oq_bs_val<T>(S.bs1_c[ty], S.bs1_n[ty], dinv, rc, rn2t * oq_rsqrt(rn2t)) -
            oq_bs_val<T>(S.bs1_c[ty], S.bs1_n[ty], dinv, rc, ro2t * oq_rsqrt(ro2t));
    }
  }
  if (S.has_j3)
    dJ -= oq_j3_electron<T>(S, pos, (size_t)ps, NE, e, 0, nx, ny, nz) -
          oq_j3_electron<T>(S, pos, (size_t)ps, NE, e, 0, ox, oy, oz);
  return dJ;
}

// One single-electron Metropolis move of electron e to (nx, ny, nz) against
// one walker's state: its positions pos[(3 j + c) ps] and its inverse
// matrices A[k as] (either in shared or in global memory); the
// proposal-density ratio q(old)/q(new) is
// mul_extra * exp(log_extra) (1 for symmetric proposals).  The move is
// accepted when u < |R|^2 exp(2 dJ) q(old)/q(new), the Metropolis-Hastings
// test of metropolis_move_1w (OmegaQMC/vmc_gto.py:841-905) without
// logarithms.  Returns acceptance.
// J supplies the nuclei and Jastrow constants (natm, nuc, has_j1, j1a, j1b,
// has_j2, j2): the system struct itself or a compact copy of those fields;
// S is handed to the basis policy.
template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ bool oq_try_move_s(const SJ& J, const OqSystem& S, const OqSplit& SP,
                                              const Real* __restrict__ C, double* pos, int ps,
                                              Real* A, int as, int e, double nx, double ny,
                                              double nz, T log_extra, T mul_extra, T u,
                                              double& logdet) {
  constexpr int NE = 2 * NOCC;
  constexpr int NN = NOCC * NOCC;
  const int s = e & 1, i = e >> 1;
  const double ox = pos[(3 * e) * ps], oy = pos[(3 * e + 1) * ps], oz = pos[(3 * e + 2) * ps];
  // Jastrow change (arithmetic in T) and the MIN_DIST_THRESHOLD test (FP64)
  bool valid;
  const T dJ = oq_jastrow_delta<NE, T>(J, S, pos, ps, e, ox, oy, oz, nx, ny, nz, valid);
  // new MO row and the ratio R = sum_m v_m A[m][i] (column i of the inverse)
  T v[NOCC];
  B::template mo_val<T, Real>(S, SP, C, nx, ny, nz, v);
  Real* As = A + (size_t)s * NN * as;
  T R = (T)0;
#pragma unroll
  for (int m = 0; m < NOCC; ++m) R += v[m] * (T)As[(m * NOCC + i) * as];
  const bool acc = oq_accept<T>(R, dJ, log_extra, mul_extra, u, valid);
  if (acc) {
    // Sherman-Morrison with the ratio vector w_j = sum_m v_m A[m][j]:
    // A[k][j] -= A[k][i] (w_j - delta_ij) / R, column i taken before the update
    const T rinv = oq_rcp(R);
    T coli[NOCC];
#pragma unroll
    for (int k = 0; k < NOCC; ++k) coli[k] = (T)As[(k * NOCC + i) * as];
#pragma unroll
    for (int j = 0; j < NOCC; ++j) {
      T w = (T)0;
#pragma unroll
      for (int m = 0; m < NOCC; ++m) w += v[m] * (T)As[(m * NOCC + j) * as];
      const T f = (w - (j == i ? (T)1 : (T)0)) * rinv;
#pragma unroll
      for (int k = 0; k < NOCC; ++k) {
        Real& ref = As[(k * NOCC + j) * as];
        ref = (Real)((T)ref - coli[k] * f);
      }
    }
    pos[(3 * e) * ps] = nx;
    pos[(3 * e + 1) * ps] = ny;
    pos[(3 * e + 2) * ps] = nz;
    logdet += log(fabs((double)R));
  }
  return acc;
}

// The same move with positions and inverses in one walker-minor layout of
// stride WPB (this walker at index tid).
template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ bool oq_try_move(const SJ& J, const OqSystem& S, const OqSplit& SP,
                                            const Real* __restrict__ C, double* pos,
                                            Real* Ai, int WPB, int tid, int e,
                                            double nx, double ny, double nz,
                                            T log_extra, T mul_extra, T u,
                                            double& logdet) {
  return oq_try_move_s<NOCC, T, Real, B>(J, S, SP, C, pos + tid, WPB, Ai + tid, WPB, e, nx, ny,
                                         nz, log_extra, mul_extra, u, logdet);
}

// Basin relocation proposal (basin_move_1w, OmegaQMC/vmc_gto.py:925-957):
// one random electron to N(R_J, sigma^2) around a random nucleus J.  Returns
// the electron; sets its proposed position, the log proposal ratio
// log q(old) - log q(new) with q(x) = sum_J exp(-|x - R_J|^2 / 2 sigma^2)
// (computed as a log-sum-exp) and the acceptance uniform u.
template <int NE>
__device__ __forceinline__ int oq_basin_propose(const OqSystem& S, const double* pos, int ps,
                                                uint64_t seed, uint32_t w, uint32_t gstep,
                                                double sg, double& nx, double& ny, double& nz,
                                                double& log_qratio, double& u) {
  double n3[3];
  oq_move_randoms(seed, w, gstep, 0xB0000000u, n3, u);
  const OqU4 c = {w, gstep, 0xB0000001u, 2u};
  const OqU4 r = oq_philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const int e = (int)(((uint64_t)r.x * NE) >> 32);
  const int J = (int)(((uint64_t)r.y * S.natm) >> 32);
  const double inv2s2 = 1.0 / (2.0 * sg * sg);
  nx = S.nuc[J][0] + sg * n3[0];
  ny = S.nuc[J][1] + sg * n3[1];
  nz = S.nuc[J][2] + sg * n3[2];
  const double ox = pos[(3 * e) * ps], oy = pos[(3 * e + 1) * ps], oz = pos[(3 * e + 2) * ps];
  double mo = -INFINITY, mn = -INFINITY;
  for (int I = 0; I < S.natm; ++I) {
    const double dox = ox - S.nuc[I][0], doy = oy - S.nuc[I][1], doz = oz - S.nuc[I][2];
    const double dnx = nx - S.nuc[I][0], dny = ny - S.nuc[I][1], dnz = nz - S.nuc[I][2];
    mo = fmax(mo, -(dox * dox + doy * doy + doz * doz) * inv2s2);
    mn = fmax(mn, -(dnx * dnx + dny * dny + dnz * dnz) * inv2s2);
  }
  double so = 0.0, sn = 0.0;
  for (int I = 0; I < S.natm; ++I) {
    const double dox = ox - S.nuc[I][0], doy = oy - S.nuc[I][1], doz = oz - S.nuc[I][2];
    const double dnx = nx - S.nuc[I][0], dny = ny - S.nuc[I][1], dnz = nz - S.nuc[I][2];
    so += exp(-(dox * dox + doy * doy + doz * doz) * inv2s2 - mo);
    sn += exp(-(dnx * dnx + dny * dny + dnz * dnz) * inv2s2 - mn);
  }
  log_qratio = (mo + log(so)) - (mn + log(sn));
  return e;
}

// Metropolis moves, one thread per walker, state resident in shared memory
// for the whole launch.  PROP (compile time) selects the proposal: 0 fixed-
// width Gaussian, 1 nucleus-scaled Gaussian, 2 basin relocation.  mode 0: n_steps sweeps over all electrons with
// Gaussian proposals (metropolis_move_1w, OmegaQMC/vmc_gto.py:841-905, as
// single-electron moves).  mode 1: n_steps basin relocations: one random
// electron proposed at N(R_J, sigma^2) around a random nucleus J, accepted
// with the exact proposal ratio q(old)/q(new), q(x) = sum_J
// exp(-|x-R_J|^2 / 2 sigma^2) (basin_move_1w, vmc_gto.py:925-957).
template <int NOCC, typename T, typename Real, int PROP, class B = OqBasisTable<NOCC>>
__global__ void __launch_bounds__(128, 4)
k_moves(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
        const void* __restrict__ gC, OqMoveArgs a) {
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
  Real* gA = reinterpret_cast<Real*>(a.ainv);
  if (live) {
    for (int k = 0; k < 3 * NE; ++k) pos[k * WPB + tid] = a.pos[(size_t)k * W + w];
    for (int k = 0; k < 2 * NN; ++k) Ai[k * WPB + tid] = gA[(size_t)k * W + w];
  }
  __syncthreads();
  const double step = a.step_dev ? *a.step_dev : a.step;
  const OqScaledF pf = oq_scaled_f(step, a.scale_r0, a.scale_fmin);
  double logdet = live ? a.logdet[w] : 0.0;
  int nacc = 0;
  for (int t = 0; t < (live ? a.n_steps : 0); ++t) {
    const uint32_t gstep = (uint32_t)(a.step_base + t);
    if (PROP == 0) {
      for (int e = 0; e < NE; ++e) {
        float nf[3];
        uint32_t ub;
        oq_move_normals(a.seed, (uint32_t)w, gstep, (uint32_t)e, nf, ub);
        const double nx = pos[(3 * e) * WPB + tid] + step * (double)nf[0];
        const double ny = pos[(3 * e + 1) * WPB + tid] + step * (double)nf[1];
        const double nz = pos[(3 * e + 2) * WPB + tid] + step * (double)nf[2];
        nacc += oq_try_move<NOCC, T, Real, B>(S, S, SP, C, pos, Ai, WPB, tid, e, nx, ny, nz,
                                           (T)0, (T)1, oq_uniform<T>(ub), logdet);
      }
    } else if (PROP == 1) {
      // nucleus-scaled Gaussian: sigma(x) = step * clamp(r_near(x)/r0, fmin, 1);
      // exact MH with log q(x|x') - log q(x'|x) for the asymmetric proposal
      for (int e = 0; e < NE; ++e) {
        float nf[3];
        uint32_t ub;
        oq_move_normals(a.seed, (uint32_t)w, gstep, (uint32_t)e, nf, ub);
        const double ox = pos[(3 * e) * WPB + tid], oy = pos[(3 * e + 1) * WPB + tid],
                     oz = pos[(3 * e + 2) * WPB + tid];
        double nx, ny, nz;
        T mul, lx;
        oq_scaled_propose_t<T>(S, ox, oy, oz, nf, pf, nx, ny, nz, mul, lx);
        nacc += oq_try_move<NOCC, T, Real, B>(S, S, SP, C, pos, Ai, WPB, tid, e, nx, ny, nz, lx,
                                           mul, oq_uniform<T>(ub), logdet);
      }
    } else {
      double u, nx, ny, nz, log_qratio;
      const int e = oq_basin_propose<NE>(S, pos + tid, WPB, a.seed, (uint32_t)w, gstep, step,
                                         nx, ny, nz, log_qratio, u);
      nacc += oq_try_move<NOCC, T, Real, B>(S, S, SP, C, pos, Ai, WPB, tid, e, nx, ny, nz,
                                         (T)log_qratio, (T)1, (T)u, logdet);
    }
  }
  if (live) {
    for (int k = 0; k < 3 * NE; ++k) a.pos[(size_t)k * W + w] = pos[k * WPB + tid];
    for (int k = 0; k < 2 * NN; ++k) gA[(size_t)k * W + w] = Ai[k * WPB + tid];
    a.logdet[w] = logdet;
  }
  if (a.acc_sum) {
    double v = (double)nacc;   // every lane of the warp reaches here
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((tid & 31) == 0) atomicAdd(a.acc_sum, v);
  }
}

// Jastrow gradient and Laplacian of electron e at (xe, ye, ze) (Padé,
// B-spline and three-body terms; gto.py:1575-1649, 1657-1931, 2042-2196),
// accumulated into (jx, jy, jz, jl), and its Coulomb terms (e-e counted once,
// for partners j > e; e-n; gto.py:2406-2451) into ee, en.  The other
// electrons' coordinate c is pos[(3 j + c) * ps].
template <int NE, typename T, class SJ>
__device__ __forceinline__ void oq_jastrow_vgl_coulomb(const SJ& J, const OqSystem& S,
                                                       const double* pos, size_t ps, int e,
                                                       double xe, double ye, double ze, T& jx,
                                                       T& jy, T& jz, T& jl, double& ee,
                                                       double& en) {
  // The gradient sums run in FP64 on the FP64 displacements: in the mixed
  // build that converts one value per pair (u'(r)/r) to FP64 instead of
  // three displacement components to FP32.  The working-precision Coulomb
  // terms of one electron are summed in T and converted once.  In the FP64
  // build both forms are the same arithmetic in the same order.
  double gx = 0.0, gy = 0.0, gz = 0.0;
  T eet = (T)0, ent = (T)0;
  for (int j = 0; j < NE; ++j) {
    if (j == e) continue;
    const double dx = xe - pos[(size_t)(3 * j) * ps], dy = ye - pos[(size_t)(3 * j + 1) * ps],
                 dz = ze - pos[(size_t)(3 * j + 2) * ps];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const T r2t = (T)r2, rinv = oq_rsqrt(r2t);
    // Coulomb: FP64 with the reference's eps in FP64 kernels; the working-
    // precision 1/r otherwise (eps is below FP32 resolution beyond the
    // 1e-4 bohr minimum distance)
    if (j > e) {
      if (sizeof(T) == 8)
        ee += rsqrt(r2 + OQ_EPS);
      else
        eet += rinv;
    }
    if (J.has_j2) {
      const int o = ((e & 1) == (j & 1)) ? 0 : 2;
      T upr, l;
      oq_pade_vgl_q((T)J.j2[o], (T)J.j2[o + 1], r2t * rinv, rinv, upr, l);
      const double u = (double)upr;
      gx += u * dx; gy += u * dy; gz += u * dz; jl += l;
    }
    if (S.has_bs2) {
      const bool like = (e & 1) == (j & 1);
      T upr, l;
      oq_bs_vgl<T>(like ? S.bs2_like : S.bs2_unlike, like ? S.bs2_n_like : S.bs2_n_unlike,
                   (T)(like ? S.bs2_dinv_like : S.bs2_dinv_unlike), (T)S.bs2_rcut, r2t * rinv,
                   rinv, upr, l);
      const double u = (double)upr;
      gx += u * dx; gy += u * dy; gz += u * dz; jl += l;
    }
  }
  for (int I = 0; I < J.natm; ++I) {
    const double dx = xe - J.nuc[I][0], dy = ye - J.nuc[I][1], dz = ze - J.nuc[I][2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const T r2t = (T)r2, rinv = oq_rsqrt(r2t);
    if (sizeof(T) == 8)
      en -= J.Z[I] * rsqrt(r2 + OQ_EPS);
    else
      ent -= (T)J.Z[I] * rinv;
    if (J.has_j1) {
      T upr, l;
      oq_pade_vgl_q((T)J.j1a[I], (T)J.j1b[I], r2t * rinv, rinv, upr, l);
      const double u = (double)upr;
      gx += u * dx; gy += u * dy; gz += u * dz; jl += l;
    }
    if (S.has_bs1 && S.bs1_type[I] >= 0) {
      const int ty = S.bs1_type[I];
      T upr, l;
      oq_bs_vgl<T>(S.bs1_c[ty], S.bs1_n[ty], (T)S.bs1_dinv[ty], (T)S.bs1_rcut[ty], r2t * rinv,
                   rinv, upr, l);
      const double u = (double)upr;
      gx += u * dx; gy += u * dy; gz += u * dz; jl += l;
    }
  }
  if (sizeof(T) != 8) {
    ee += (double)eet;
    en += (double)ent;
  }
  jx += (T)gx; jy += (T)gy; jz += (T)gz;
  if (S.has_j3) oq_j3_vgl_electron<T>(S, pos, ps, NE, e, xe, ye, ze, jx, jy, jz, jl);
}

// Local-energy contributions of electron e of one walker: its Coulomb terms
// (e-e counted once, for partners j > e; gto.py:2406-2451), the Laplacian
// term lap_e = sum_m A[m][i] L[i][m] - |Gamma_e|^2 + lap J_e and the squared
// total gradient |Gamma_e + grad J_e|^2 (_slater_det_assemble, gto.py:728-778;
// Padé VGL, gto.py:1575-1649).  pos points at the walker's x of electron 0
// with stride ps between coordinates; A at its inverse entry (0,0,0) with
// stride as between entries.  The four outputs are accumulated (+=).
// The _out form also returns electron e's gradient of log|psi| (Gx, Gy, Gz)
// and its Laplacian of log|psi| (lap_e).
template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ void oq_eloc_electron_out(const SJ& J, const OqSystem& S,
                                                     const OqSplit& SP,
                                                     const Real* __restrict__ C,
                                                     const double* pos, size_t ps,
                                                     const Real* A, size_t as, int e,
                                                     double& ee, double& en, double& lp_tot,
                                                     double& g2, double& gxo, double& gyo,
                                                     double& gzo, double& lape) {
  constexpr int NE = 2 * NOCC;
  const int s = e & 1, i = e >> 1;
  const double xe = pos[(size_t)(3 * e) * ps], ye = pos[(size_t)(3 * e + 1) * ps],
               ze = pos[(size_t)(3 * e + 2) * ps];
  // Gamma = sum_m A[m][i] grad phi_m, sum_m A[m][i] lap phi_m: the MO
  // coefficients contracted with column i of the inverse first
  T ac[NOCC];
#pragma unroll
  for (int m = 0; m < NOCC; ++m) ac[m] = (T)A[(size_t)((s * NOCC + m) * NOCC + i) * as];
  T gx, gy, gz, lp;
  B::template mo_vgl_contract<T, Real>(S, SP, C, xe, ye, ze, ac, gx, gy, gz, lp);
  T jx = (T)0, jy = (T)0, jz = (T)0, jl = (T)0;
  oq_jastrow_vgl_coulomb<NE, T>(J, S, pos, ps, e, xe, ye, ze, jx, jy, jz, jl, ee, en);
  const double sgx = (double)gx, sgy = (double)gy, sgz = (double)gz;
  const double Gx = sgx + (double)jx, Gy = sgy + (double)jy, Gz = sgz + (double)jz;
  lape = (double)lp - (sgx * sgx + sgy * sgy + sgz * sgz) + (double)jl;
  lp_tot += lape;
  g2 += Gx * Gx + Gy * Gy + Gz * Gz;
  gxo = Gx; gyo = Gy; gzo = Gz;
}

template <int NOCC, typename T, typename Real, class B, class SJ>
__device__ __forceinline__ void oq_eloc_electron(const SJ& J, const OqSystem& S,
                                                 const OqSplit& SP, const Real* __restrict__ C,
                                                 const double* pos, size_t ps, const Real* A,
                                                 size_t as, int e, double& ee, double& en,
                                                 double& lp_tot, double& g2) {
  double gx, gy, gz, le;
  oq_eloc_electron_out<NOCC, T, Real, B>(J, S, SP, C, pos, ps, A, as, e, ee, en, lp_tot, g2,
                                         gx, gy, gz, le);
}

// Electron e's share of the Jastrow value J (log_trial_wavefunction,
// gto.py:2220-2254): its pairs with the electrons j > e and its
// electron-nucleus terms, each term in working precision T, summed in FP64.
// Summed over all electrons this is J1 + J2 (+ B-spline, J3).
template <int NE, typename T>
__device__ __forceinline__ double oq_jastrow_value_electron(const OqSystem& S, const double* pos,
                                                           size_t ps, int e, double xe,
                                                           double ye, double ze) {
  double J = 0.0;
  for (int j = e + 1; j < NE; ++j) {
    const double dx = xe - pos[(size_t)(3 * j) * ps], dy = ye - pos[(size_t)(3 * j + 1) * ps],
                 dz = ze - pos[(size_t)(3 * j + 2) * ps];
    const T r = sqrt((T)(dx * dx + dy * dy + dz * dz));
    const bool like = (e & 1) == (j & 1);
    if (S.has_j2) {
      const int o = like ? 0 : 2;
      J += (double)oq_pade<T>((T)S.j2[o], (T)S.j2[o + 1], r);
    }
    if (S.has_bs2)
      J += (double)oq_bs_val<T>(like ? S.bs2_like : S.bs2_unlike,
                                like ? S.bs2_n_like : S.bs2_n_unlike,
                                (T)(like ? S.bs2_dinv_like : S.bs2_dinv_unlike),
                                (T)S.bs2_rcut, r);
  }
  for (int I = 0; I < S.natm; ++I) {
    const double dx = xe - S.nuc[I][0], dy = ye - S.nuc[I][1], dz = ze - S.nuc[I][2];
    const T r = sqrt((T)(dx * dx + dy * dy + dz * dz));
    if (S.has_j1) J += (double)oq_pade<T>((T)S.j1a[I], (T)S.j1b[I], r);
    if (S.has_bs1 && S.bs1_type[I] >= 0) {
      const int ty = S.bs1_type[I];
      J += (double)oq_bs_val<T>(S.bs1_c[ty], S.bs1_n[ty], (T)S.bs1_dinv[ty],
                                (T)S.bs1_rcut[ty], r);
    }
  }
  if (S.has_j3) J -= (double)oq_j3_electron<T>(S, pos, ps, NE, e, e + 1, xe, ye, ze);
  return J;
}

struct OqElocArgs {
  const double* pos;
  const void* ainv;
  int W;
  int pad;
  double* sums;           // OQ_NSUM slot of this measurement (accumulated)
  double* el_trace;       // (W) local energies of this measurement, or null
  double* eparts;         // (W, 4) ee, en, ke, E_L, or null
  unsigned* flags;
  // per-walker outputs of oqmc_state_eval (null in the sampling kernels)
  double* logpsi;         // (W): holds log|det| on entry; each electron adds its J share
  double* grad;           // (W, NE, 3) gradient of log|psi|
  double* lap;            // (W, NE) Laplacian of log|psi|
};

// Local energy, one thread per (walker, electron): blockDim = (32, NE), lane
// x = walker, y = electron.  Each thread forms its electron's MO VGL, the
// Slater gradient/Laplacian against column i of the inverse
// (_slater_det_assemble, gto.py:728-778), the Padé Jastrow VGL
// (gto.py:1575-1649) and its Coulomb terms (gto.py:2406-2451); the CTA then
// reduces over electrons (local_energy_ke, gto.py:2506-2579) and over
// walkers (fused reduction of E, E^2 and the parts).
template <int NOCC, typename T, typename Real, class B = OqBasisTable<NOCC>>
__global__ void __launch_bounds__(64 * NOCC, (NOCC <= 6) ? 2 : 1)
k_eloc(const OqSystem* __restrict__ gsys, const OqSplit* __restrict__ gsplit,
       const void* __restrict__ gC, OqElocArgs a) {
  constexpr int NE = 2 * NOCC;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  OqSplit& SP = *reinterpret_cast<OqSplit*>(smem + sizeof(OqSystem));
  unsigned char* p = smem + sizeof(OqSystem) + sizeof(OqSplit);
  Real* C = reinterpret_cast<Real*>(p);
  const int nbf = gsys->nbf;
  p += ((size_t)nbf * NOCC * sizeof(Real) + 15) & ~(size_t)15;
  double* red = reinterpret_cast<double*>(p);          // [NE][4][32]
  const int lane = threadIdx.x, e = threadIdx.y;
  const int flat = e * 32 + lane, nthr = 32 * NE;
  {
    const int4* s4 = reinterpret_cast<const int4*>(gsys);
    int4* d4 = reinterpret_cast<int4*>(&S);
    for (int i = flat; i < (int)(sizeof(OqSystem) / 16); i += nthr) d4[i] = s4[i];
    const double* src = reinterpret_cast<const double*>(gsplit);
    double* dst = reinterpret_cast<double*>(&SP);
    for (int i = flat; i < OQ_MAX_GROUP; i += nthr) dst[i] = src[i];
    const Real* gc = reinterpret_cast<const Real*>(gC);
    for (int i = flat; i < nbf * NOCC; i += nthr) C[i] = gc[i];
  }
  __syncthreads();
  const int W = a.W;
  const int w = blockIdx.x * 32 + lane;
  const bool live = w < W;
  double ee = 0.0, en = 0.0, lp_tot = 0.0, g2 = 0.0;
  if (live) {
    double gx, gy, gz, le;
    oq_eloc_electron_out<NOCC, T, Real, B>(S, S, SP, C, a.pos + w, (size_t)W,
                                           reinterpret_cast<const Real*>(a.ainv) + w,
                                           (size_t)W, e, ee, en, lp_tot, g2, gx, gy, gz, le);
    if (a.grad) {
      double* g = a.grad + ((size_t)w * NE + e) * 3;
      g[0] = gx; g[1] = gy; g[2] = gz;
    }
    if (a.lap) a.lap[(size_t)w * NE + e] = le;
    if (a.logpsi) {
      const double* pw = a.pos + w;
      atomicAdd(a.logpsi + w,
                oq_jastrow_value_electron<NE, T>(S, pw, (size_t)W, e, pw[(size_t)(3 * e) * W],
                                                 pw[(size_t)(3 * e + 1) * W],
                                                 pw[(size_t)(3 * e + 2) * W]));
    }
  }
  red[(e * 4 + 0) * 32 + lane] = ee;
  red[(e * 4 + 1) * 32 + lane] = en;
  red[(e * 4 + 2) * 32 + lane] = lp_tot;
  red[(e * 4 + 3) * 32 + lane] = g2;
  __syncthreads();
  if (e != 0) return;
  double see = 0.0, sen = 0.0, slp = 0.0, sg2 = 0.0;
  for (int k = 0; k < NE; ++k) {
    see += red[(k * 4 + 0) * 32 + lane];
    sen += red[(k * 4 + 1) * 32 + lane];
    slp += red[(k * 4 + 2) * 32 + lane];
    sg2 += red[(k * 4 + 3) * 32 + lane];
  }
  const double ke = -0.5 * (slp + sg2);
  const double el = see + sen + ke + S.e_nn;
  const bool ok = live && isfinite(el);
  if (live) {
    if (a.el_trace) a.el_trace[w] = el;
    if (a.eparts) {
      double* ep = a.eparts + (size_t)w * 4;
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
  if (lane == 0 && a.sums) {
#pragma unroll
    for (int k = 0; k < 5; ++k) atomicAdd(a.sums + k, vals[k]);
    atomicAdd(a.sums + 6, vals[5]);
  }
}
