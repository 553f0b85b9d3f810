// Full FP64 per-walker evaluation (the parity surface): log|psi|,
// grad log|psi|, per-electron Laplacian of log|psi| and the local-energy
// parts, with a fresh inverse of each spin block.  One thread per walker.
//
// Follows log_trial_wavefunction (OmegaQMC/psi/gto.py:2220-2254),
// _slater_det_assemble (gto.py:728-778), the Padé VGL helpers
// (gto.py:1575-1649), classical_coulomb_energy (gto.py:2406-2451) and
// local_energy_ke (gto.py:2506-2579).
#pragma once
#include "oqmc_ao.cuh"

#define OQ_EPS 2.220446049250313e-16

// Gauss-Jordan inverse with partial pivoting of the N x N matrix a
// (destroyed); returns false if a pivot is exactly zero or not finite.
// logdet = log|det a|; *sign (when given) = the sign of det a.
template <int N>
__device__ bool oq_invert(double (&a)[N][N], double (&inv)[N][N], double& logdet,
                          double* sign = nullptr) {
  double sg = 1.0;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) inv[i][j] = (i == j) ? 1.0 : 0.0;
  logdet = 0.0;
  for (int k = 0; k < N; ++k) {
    int piv = k;
    double best = fabs(a[k][k]);
    for (int i = k + 1; i < N; ++i) {
      const double v = fabs(a[i][k]);
      if (v > best) { best = v; piv = i; }
    }
    if (!(best > 0.0) || !isfinite(best)) return false;
    if (piv != k) {
      sg = -sg;
      for (int j = 0; j < N; ++j) {
        double t = a[k][j]; a[k][j] = a[piv][j]; a[piv][j] = t;
        t = inv[k][j]; inv[k][j] = inv[piv][j]; inv[piv][j] = t;
      }
    }
    const double d = a[k][k];
    logdet += log(fabs(d));
    if (d < 0.0) sg = -sg;
    const double rd = 1.0 / d;
    for (int j = 0; j < N; ++j) { a[k][j] *= rd; inv[k][j] *= rd; }
    for (int i = 0; i < N; ++i) {
      if (i == k) continue;
      const double f = a[i][k];
      if (f != 0.0) {
        for (int j = 0; j < N; ++j) { a[i][j] -= f * a[k][j]; inv[i][j] -= f * inv[k][j]; }
      }
    }
  }
  if (sign) *sign = sg;
  return true;
}

// Jastrow value J1 + J2 (+ J3) for walker positions x[n_e][3] (in
// registers/local).
__device__ __forceinline__ double oq_jastrow_value(const OqSystem& S, const double* x,
                                                   int n_e) {
  double J = 0.0;
  if (S.has_j2) {
    for (int i = 0; i < n_e; ++i)
      for (int j = i + 1; j < n_e; ++j) {
        const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1],
                     dz = x[3 * i + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const int o = ((i & 1) == (j & 1)) ? 0 : 2;
        J += oq_pade(S.j2[o], S.j2[o + 1], r);
      }
  }
  if (S.has_j1) {
    for (int i = 0; i < n_e; ++i)
      for (int I = 0; I < S.natm; ++I) {
        const double dx = x[3 * i] - S.nuc[I][0], dy = x[3 * i + 1] - S.nuc[I][1],
                     dz = x[3 * i + 2] - S.nuc[I][2];
        J += oq_pade(S.j1a[I], S.j1b[I], sqrt(dx * dx + dy * dy + dz * dz));
      }
  }
  if (S.has_bs2) {
    for (int i = 0; i < n_e; ++i)
      for (int j = i + 1; j < n_e; ++j) {
        const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1],
                     dz = x[3 * i + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const bool like = (i & 1) == (j & 1);
        J += oq_bs_val<double>(like ? S.bs2_like : S.bs2_unlike,
                               like ? S.bs2_n_like : S.bs2_n_unlike,
                               like ? S.bs2_dinv_like : S.bs2_dinv_unlike, S.bs2_rcut, r);
      }
  }
  if (S.has_bs1) {
    for (int i = 0; i < n_e; ++i)
      for (int I = 0; I < S.natm; ++I) {
        const int ty = S.bs1_type[I];
        if (ty < 0) continue;
        const double dx = x[3 * i] - S.nuc[I][0], dy = x[3 * i + 1] - S.nuc[I][1],
                     dz = x[3 * i + 2] - S.nuc[I][2];
        J += oq_bs_val<double>(S.bs1_c[ty], S.bs1_n[ty], S.bs1_dinv[ty], S.bs1_rcut[ty],
                               sqrt(dx * dx + dy * dy + dz * dz));
      }
  }
  if (S.has_j3) {
    for (int i = 0; i < n_e; ++i)
      J -= oq_j3_electron<double>(S, x, 1, n_e, i, i + 1, x[3 * i], x[3 * i + 1], x[3 * i + 2]);
  }
  return J;
}

template <int NOCC>
__global__ void __launch_bounds__(128)
k_eval(const OqSystem* __restrict__ gsys, const double* __restrict__ gC,
       const double* __restrict__ X, int W, double* __restrict__ logpsi,
       double* __restrict__ grad, double* __restrict__ lap,
       double* __restrict__ eparts, unsigned* __restrict__ flags) {
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
  constexpr int NE = 2 * NOCC;
  double x[3 * NE];
  for (int k = 0; k < 3 * NE; ++k) x[k] = X[(size_t)w * 3 * NE + k];

  // pass 1: MO values -> Slater matrices and their inverses
  double A[2][NOCC][NOCC];
  double logdet_tot = 0.0;
  bool ok = true;
  for (int s = 0; s < 2; ++s) {
    double Sm[NOCC][NOCC];
    for (int i = 0; i < NOCC; ++i) {
      const int e = 2 * i + s;
      double mv[NOCC];
      oq_mo_val<NOCC>(S, C, x[3 * e], x[3 * e + 1], x[3 * e + 2], mv);
#pragma unroll
      for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
    }
    double ld;
    ok = ok && oq_invert<NOCC>(Sm, A[s], ld);
    logdet_tot += ld;
  }

  // pass 2: per-electron MO VGL against the inverse; Jastrow VGL
  double ke_lap = 0.0, ke_g2 = 0.0;
  for (int e = 0; e < NE; ++e) {
    const int s = e & 1, i = e >> 1;
    double mv[NOCC], mg[NOCC][3], ml[NOCC];
    oq_mo_vgl<NOCC>(S, C, x[3 * e], x[3 * e + 1], x[3 * e + 2], mv, mg, ml);
    double gx = 0.0, gy = 0.0, gz = 0.0, lp = 0.0;
#pragma unroll
    for (int m = 0; m < NOCC; ++m) {
      const double am = A[s][m][i];
      gx += am * mg[m][0]; gy += am * mg[m][1]; gz += am * mg[m][2];
      lp += am * ml[m];
    }
    lp -= gx * gx + gy * gy + gz * gz;
    // Jastrow contributions to electron e
    if (S.has_j2) {
      for (int j = 0; j < NE; ++j) {
        if (j == e) continue;
        const double dx = x[3 * e] - x[3 * j], dy = x[3 * e + 1] - x[3 * j + 1],
                     dz = x[3 * e + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const int o = ((e & 1) == (j & 1)) ? 0 : 2;
        double upr, l;
        oq_pade_vgl(S.j2[o], S.j2[o + 1], r, upr, l);
        gx += upr * dx; gy += upr * dy; gz += upr * dz; lp += l;
      }
    }
    if (S.has_bs2) {
      for (int j = 0; j < NE; ++j) {
        if (j == e) continue;
        const double dx = x[3 * e] - x[3 * j], dy = x[3 * e + 1] - x[3 * j + 1],
                     dz = x[3 * e + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const bool like = (e & 1) == (j & 1);
        double upr, l;
        oq_bs_vgl<double>(like ? S.bs2_like : S.bs2_unlike, like ? S.bs2_n_like : S.bs2_n_unlike,
                          like ? S.bs2_dinv_like : S.bs2_dinv_unlike, S.bs2_rcut, r, 1.0 / r,
                          upr, l);
        gx += upr * dx; gy += upr * dy; gz += upr * dz; lp += l;
      }
    }
    if (S.has_j1) {
      for (int I = 0; I < S.natm; ++I) {
        const double dx = x[3 * e] - S.nuc[I][0], dy = x[3 * e + 1] - S.nuc[I][1],
                     dz = x[3 * e + 2] - S.nuc[I][2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        double upr, l;
        oq_pade_vgl(S.j1a[I], S.j1b[I], r, upr, l);
        gx += upr * dx; gy += upr * dy; gz += upr * dz; lp += l;
      }
    }
    if (S.has_bs1) {
      for (int I = 0; I < S.natm; ++I) {
        const int ty = S.bs1_type[I];
        if (ty < 0) continue;
        const double dx = x[3 * e] - S.nuc[I][0], dy = x[3 * e + 1] - S.nuc[I][1],
                     dz = x[3 * e + 2] - S.nuc[I][2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        double upr, l;
        oq_bs_vgl<double>(S.bs1_c[ty], S.bs1_n[ty], S.bs1_dinv[ty], S.bs1_rcut[ty], r, 1.0 / r,
                          upr, l);
        gx += upr * dx; gy += upr * dy; gz += upr * dz; lp += l;
      }
    }
    if (S.has_j3)
      oq_j3_vgl_electron<double>(S, x, 1, NE, e, x[3 * e], x[3 * e + 1], x[3 * e + 2], gx, gy, gz,
                                 lp);
    if (grad) {
      double* gp = grad + (size_t)w * 3 * NE + 3 * e;
      gp[0] = gx; gp[1] = gy; gp[2] = gz;
    }
    if (lap) lap[(size_t)w * NE + e] = lp;
    ke_lap += lp;
    ke_g2 += gx * gx + gy * gy + gz * gz;
  }
  const double lpsi = logdet_tot + oq_jastrow_value(S, x, NE);
  double ee = 0.0, en = 0.0;
  for (int i = 0; i < NE; ++i) {
    for (int j = i + 1; j < NE; ++j) {
      const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1],
                   dz = x[3 * i + 2] - x[3 * j + 2];
      ee += 1.0 / sqrt(dx * dx + dy * dy + dz * dz + OQ_EPS);
    }
    for (int I = 0; I < S.natm; ++I) {
      const double dx = x[3 * i] - S.nuc[I][0], dy = x[3 * i + 1] - S.nuc[I][1],
                   dz = x[3 * i + 2] - S.nuc[I][2];
      en -= S.Z[I] / sqrt(dx * dx + dy * dy + dz * dz + OQ_EPS);
    }
  }
  const double ke = -0.5 * (ke_lap + ke_g2);
  logpsi[w] = ok ? lpsi : -INFINITY;
  if (eparts) {
    double* ep = eparts + (size_t)w * 4;
    ep[0] = ee; ep[1] = en; ep[2] = ke; ep[3] = ee + en + ke + S.e_nn;
  }
  if (!ok) atomicOr(flags, OQ_FLAG_SINGULAR);
  else if (!isfinite(ke) || !isfinite(lpsi)) atomicOr(flags, OQ_FLAG_NAN);
}

// log|psi| only (value path: cgs_sph_get + slogdet + J), one thread per walker.
template <int NOCC>
__global__ void __launch_bounds__(128)
k_logpsi(const OqSystem* __restrict__ gsys, const double* __restrict__ gC,
         const double* __restrict__ X, int W, double* __restrict__ logpsi,
         unsigned* __restrict__ flags) {
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
  constexpr int NE = 2 * NOCC;
  double x[3 * NE];
  for (int k = 0; k < 3 * NE; ++k) x[k] = X[(size_t)w * 3 * NE + k];
  double ld_tot = 0.0;
  bool ok = true;
  for (int s = 0; s < 2; ++s) {
    double Sm[NOCC][NOCC], Ai[NOCC][NOCC];
    for (int i = 0; i < NOCC; ++i) {
      const int e = 2 * i + s;
      double mv[NOCC];
      oq_mo_val<NOCC>(S, C, x[3 * e], x[3 * e + 1], x[3 * e + 2], mv);
#pragma unroll
      for (int m = 0; m < NOCC; ++m) Sm[i][m] = mv[m];
    }
    double ld;
    ok = ok && oq_invert<NOCC>(Sm, Ai, ld);
    ld_tot += ld;
  }
  const double l = ld_tot + oq_jastrow_value(S, x, NE);
  logpsi[w] = ok ? l : -INFINITY;
  if (!ok) atomicOr(flags, OQ_FLAG_SINGULAR);
}

// Occupied MO values per (walker, electron): out[(w*n_e + e)*NOCC + m]
// (get_psi_mo, OmegaQMC/psi/gto.py:1058-1070).  One thread per electron.
template <int NOCC>
__global__ void __launch_bounds__(128)
k_mo_values(const OqSystem* __restrict__ gsys, const double* __restrict__ gC,
            const double* __restrict__ X, int W, double* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  double* C = reinterpret_cast<double*>(smem + sizeof(OqSystem));
  oq_load_system(&S, gsys);
  // the count comes from global memory: the shared copy S is complete only
  // after the barrier below
  const int nbf_g = gsys->nbf;
  for (int i = threadIdx.x; i < nbf_g * NOCC; i += blockDim.x) C[i] = gC[i];
  __syncthreads();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)W * 2 * NOCC) return;
  const double* xp = X + 3 * t;
  double mv[NOCC];
  oq_mo_val<NOCC>(S, C, xp[0], xp[1], xp[2], mv);
#pragma unroll
  for (int m = 0; m < NOCC; ++m) out[t * NOCC + m] = mv[m];
}
