// Multi-determinant Slater part (trial expansions; OmegaQMC/psi/gto.py:
// 846-863 _parse_mol, 1312-1488 log_slater_multidet and
// log_slater_multidet_analytic), FP64.
//
//   psi_S = sum_d c_d det(Phi_up[:, occ_up[d]]) det(Phi_dn[:, occ_dn[d]])
//
// Different terms share spin determinants, so each distinct up and down
// occupation list is a "unique determinant" u with its own inverse, log|det|
// and sign; term d combines unique up determinant det[d][0] and unique down
// determinant det[d][1] (nu0 up ones first, then nu1 down ones).  A move of
// an electron of spin s changes only the unique determinants of that spin.
// MO columns: the M (8 or 16, zero-padded) orbitals the expansion uses.
//
// Per-walker state, walker-minor (stride W): inverses [(nu0+nu1) N N],
// entry (slot m, electron j) of unique determinant u at (u N + m) N + j;
// log|det| [(nu0+nu1)]; sign [(nu0+nu1)] (0: singular until the next
// refresh).  One thread per walker in every kernel.
#pragma once
#include "oqmc_sweep.cuh"

#define OQ_MD_MAXU 64           // unique determinants per spin

struct OqMdTables {
  const double* C;      // nbf x M coefficients of the used orbitals (row-major)
  const double* coef;   // ndet CI coefficients
  const int* det;       // ndet x 2: unique up / unique down determinant of each term
  const int* occ;       // (nu0 + nu1) x N orbital column of each slot
  int ndet, nu0, nu1, pad;
};

struct OqMdState {
  double* pos;          // [3 n_e][W]
  double* ainv;
  double* ldet;
  double* sgn;
  int W, pad;
};

// lmax = the largest log|c_d D_up D_dn| and sum = sum_d c_d s_up s_dn
// exp(log|D_up D_dn| - lmax), the signed log-sum-exp of log_slater_multidet
// (gto.py:1341-1352).  State pointers are offset to the walker (stride W).
__device__ __forceinline__ double oq_md_sum(const OqMdTables& T, const double* ld,
                                            const double* sg, int W, double& sum) {
  double lmax = -INFINITY;
  for (int d = 0; d < T.ndet; ++d) {
    const int a = T.det[2 * d], b = T.det[2 * d + 1];
    if (sg[a * W] == 0.0 || sg[b * W] == 0.0) continue;
    lmax = fmax(lmax, log(fabs(T.coef[d])) + ld[a * W] + ld[b * W]);
  }
  sum = 0.0;
  if (!(lmax > -INFINITY)) return lmax;
  for (int d = 0; d < T.ndet; ++d) {
    const int a = T.det[2 * d], b = T.det[2 * d + 1];
    const double s = sg[a * W] * sg[b * W];
    if (s == 0.0) continue;
    sum += T.coef[d] * s * exp(ld[a * W] + ld[b * W] - lmax);
  }
  return lmax;
}

// FP64 inverses, log|det| and signs of every unique determinant.
template <int N, int M>
__global__ void __launch_bounds__(128)
k_md_refresh(const OqSystem* __restrict__ gsys, OqMdTables T, OqMdState st,
             unsigned* __restrict__ flags) {
  constexpr int NN = N * N;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  oq_load_system(&S, gsys);
  __syncthreads();
  const int W = st.W, w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const double* pos = st.pos + w;
  bool any = false;
  for (int s = 0; s < 2; ++s) {
    double mo[N][M];
    for (int i = 0; i < N; ++i) {
      const int e = 2 * i + s;
      double v[M];
      oq_mo_val<M>(S, T.C, pos[(3 * e) * W], pos[(3 * e + 1) * W], pos[(3 * e + 2) * W], v);
#pragma unroll
      for (int m = 0; m < M; ++m) mo[i][m] = v[m];
    }
    const int u0 = s ? T.nu0 : 0, nu = s ? T.nu1 : T.nu0;
    for (int u = u0; u < u0 + nu; ++u) {
      double a[N][N], inv[N][N], ld, sg;
      for (int i = 0; i < N; ++i)
        for (int k = 0; k < N; ++k) a[i][k] = mo[i][T.occ[u * N + k]];
      if (!oq_invert<N>(a, inv, ld, &sg)) {
        ld = -INFINITY;
        sg = 0.0;
        for (int i = 0; i < N; ++i)
          for (int k = 0; k < N; ++k) inv[i][k] = 0.0;
      }
      any = any || sg != 0.0;
      double* A = st.ainv + (size_t)u * NN * W + w;
      for (int m = 0; m < N; ++m)
        for (int j = 0; j < N; ++j) A[(size_t)(m * N + j) * W] = inv[m][j];
      st.ldet[(size_t)u * W + w] = ld;
      st.sgn[(size_t)u * W + w] = sg;
    }
  }
  if (!any) atomicOr(flags, OQ_FLAG_SINGULAR);
}

// One single-electron Metropolis move of electron e to (nx, ny, nz): the
// ratio of the expansion is sum_d c_d D_d R_d / sum_d c_d D_d with R_d the
// ratio of the moving spin's unique determinant; accepted moves update
// every unique determinant of that spin (Sherman-Morrison) and their
// log|det| and sign.
template <int N, int M>
__device__ __forceinline__ bool oq_md_try_move(const OqSystem& S, const OqMdTables& T,
                                               double* pos, double* A, double* ld, double* sg,
                                               int W, int e, double nx, double ny, double nz,
                                               double log_extra, double u) {
  constexpr int NE = 2 * N, NN = N * N;
  const int s = e & 1, i = e >> 1;
  const double ox = pos[(3 * e) * W], oy = pos[(3 * e + 1) * W], oz = pos[(3 * e + 2) * W];
  bool valid;
  const double dJ = oq_jastrow_delta<NE, double>(S, S, pos, W, e, ox, oy, oz, nx, ny, nz, valid);
  double v[M];
  oq_mo_val<M>(S, T.C, nx, ny, nz, v);
  const int u0 = s ? T.nu0 : 0, nu = s ? T.nu1 : T.nu0;
  double R[OQ_MD_MAXU];
  for (int k = 0; k < nu; ++k) {
    const int uu = u0 + k;
    const double* Au = A + (size_t)uu * NN * W;
    double r = 0.0;
    for (int m = 0; m < N; ++m) r += v[T.occ[uu * N + m]] * Au[(size_t)(m * N + i) * W];
    R[k] = r;
  }
  double den;
  const double lmax = oq_md_sum(T, ld, sg, W, den);
  double num = 0.0;
  if (lmax > -INFINITY) {
    for (int d = 0; d < T.ndet; ++d) {
      const int a = T.det[2 * d], b = T.det[2 * d + 1];
      const double sd = sg[a * W] * sg[b * W];
      if (sd == 0.0) continue;
      num += T.coef[d] * sd * exp(ld[a * W] + ld[b * W] - lmax) * R[(s ? b : a) - u0];
    }
  }
  const double ratio = num / den;
  const double logp = 2.0 * log(fabs(ratio)) + 2.0 * dJ + log_extra;
  const bool acc = valid && (lmax > -INFINITY) && ratio != 0.0 && isfinite(logp) &&
                   (log(u) < logp);
  if (!acc) return false;
  for (int k = 0; k < nu; ++k) {
    const int uu = u0 + k;
    const double r = R[k];
    if (sg[uu * W] == 0.0) continue;                     // singular until the next refresh
    if (r == 0.0 || !isfinite(r)) {
      ld[uu * W] = -INFINITY;
      sg[uu * W] = 0.0;
      continue;
    }
    double* Au = A + (size_t)uu * NN * W;
    double wv[N], coli[N];
    for (int j = 0; j < N; ++j) {
      double acc2 = 0.0;
      for (int m = 0; m < N; ++m) acc2 += v[T.occ[uu * N + m]] * Au[(size_t)(m * N + j) * W];
      wv[j] = acc2;
    }
    for (int m = 0; m < N; ++m) coli[m] = Au[(size_t)(m * N + i) * W];
    const double rinv = 1.0 / r;
    for (int j = 0; j < N; ++j) {
      const double f = (wv[j] - (j == i ? 1.0 : 0.0)) * rinv;
      for (int m = 0; m < N; ++m) Au[(size_t)(m * N + j) * W] -= coli[m] * f;
    }
    ld[uu * W] += log(fabs(r));
    if (r < 0.0) sg[uu * W] = -sg[uu * W];
  }
  pos[(3 * e) * W] = nx;
  pos[(3 * e + 1) * W] = ny;
  pos[(3 * e + 2) * W] = nz;
  return true;
}

// Metropolis moves with a multi-determinant Slater part (mode 0: sweeps of
// fixed-width or nucleus-scaled Gaussian single-electron moves; mode 1:
// basin relocations), state in global memory.
template <int N, int M>
__global__ void __launch_bounds__(128)
k_md_moves(const OqSystem* __restrict__ gsys, OqMdTables T, OqMoveArgs a, double* gsgn) {
  constexpr int NE = 2 * N;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  oq_load_system(&S, gsys);
  __syncthreads();
  const int W = a.W, w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = w < W;
  int nacc = 0;
  if (live) {
    double* pos = a.pos + w;
    double* A = reinterpret_cast<double*>(a.ainv) + w;
    double* ld = a.logdet + w;
    double* sg = gsgn + w;
    for (int t = 0; t < a.n_steps; ++t) {
      const uint32_t gstep = (uint32_t)(a.step_base + t);
      if (a.mode == 0) {
        for (int e = 0; e < NE; ++e) {
          double n3[3], u;
          oq_move_randoms(a.seed, (uint32_t)w, gstep, (uint32_t)e, n3, u);
          const double ox = pos[(3 * e) * W], oy = pos[(3 * e + 1) * W],
                       oz = pos[(3 * e + 2) * W];
          double so = a.step, sn = a.step, log_extra = 0.0;
          if (a.proposal == 1) so = oq_scaled_width(S, ox, oy, oz, a.step, a.scale_r0,
                                                    a.scale_fmin);
          const double nx = ox + so * n3[0], ny = oy + so * n3[1], nz = oz + so * n3[2];
          if (a.proposal == 1) {
            sn = oq_scaled_width(S, nx, ny, nz, a.step, a.scale_r0, a.scale_fmin);
            const double d2 =
                (nx - ox) * (nx - ox) + (ny - oy) * (ny - oy) + (nz - oz) * (nz - oz);
            log_extra = 3.0 * log(so / sn) + 0.5 * d2 * (1.0 / (so * so) - 1.0 / (sn * sn));
          }
          nacc += oq_md_try_move<N, M>(S, T, pos, A, ld, sg, W, e, nx, ny, nz, log_extra, u);
        }
      } else {
        double u, nx, ny, nz, log_q;
        const int e = oq_basin_propose<NE>(S, pos, W, a.seed, (uint32_t)w, gstep, a.step, nx,
                                           ny, nz, log_q, u);
        nacc += oq_md_try_move<N, M>(S, T, pos, A, ld, sg, W, e, nx, ny, nz, log_q, u);
      }
    }
  }
  if (a.acc_sum) {
    double v = (double)nacc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(a.acc_sum, v);
  }
}

// Local energy and its parts from the tracked inverses: the Slater
// gradient and Laplacian of the expansion (log_slater_multidet_analytic,
// gto.py:1354-1480: weights w_d = c_d D_d / psi_S; grad = sum_d w_d Gamma_d,
// lap = sum_d w_d sum_m A_d[m][i] L[i][m] - |grad|^2), the Jastrow VGL and
// the Coulomb terms.  Optional per-walker outputs: logpsi (W), grad
// (W, n_e, 3), lap (W, n_e), eparts (W, 4); el_trace (W) and the walker sums
// (OQ_NSUM slot) as k_eloc.
template <int N, int M>
__global__ void __launch_bounds__(128)
k_md_local(const OqSystem* __restrict__ gsys, OqMdTables T, OqMdState st, OqElocArgs a,
           double* __restrict__ logpsi, double* __restrict__ grad, double* __restrict__ lap) {
  constexpr int NE = 2 * N, NN = N * N;
  extern __shared__ __align__(16) unsigned char smem[];
  OqSystem& S = *reinterpret_cast<OqSystem*>(smem);
  oq_load_system(&S, gsys);
  __syncthreads();
  const int W = st.W, w = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = w < W;
  double ee = 0.0, en = 0.0, lp_tot = 0.0, g2 = 0.0, lps = 0.0;
  if (live) {
    const double* pos = st.pos + w;
    const double* A = st.ainv + w;
    const double* ld = st.ldet + w;
    const double* sg = st.sgn + w;
    double sum;
    const double lmax = oq_md_sum(T, ld, sg, W, sum);
    lps = log(fabs(sum)) + lmax;
    // weight of each unique determinant: sum of w_d over the terms using it
    double wu[2][OQ_MD_MAXU];
    for (int k = 0; k < T.nu0; ++k) wu[0][k] = 0.0;
    for (int k = 0; k < T.nu1; ++k) wu[1][k] = 0.0;
    for (int d = 0; d < T.ndet; ++d) {
      const int p = T.det[2 * d], q = T.det[2 * d + 1];
      const double sd = sg[p * W] * sg[q * W];
      if (sd == 0.0) continue;
      const double wd = T.coef[d] * sd * exp(ld[p * W] + ld[q * W] - lmax) / sum;
      wu[0][p] += wd;
      wu[1][q - T.nu0] += wd;
    }
    for (int e = 0; e < NE; ++e) {
      const int s = e & 1, i = e >> 1;
      const double xe = pos[(3 * e) * W], ye = pos[(3 * e + 1) * W], ze = pos[(3 * e + 2) * W];
      double mv[M], mg[M][3], ml[M];
      oq_mo_vgl<M>(S, T.C, xe, ye, ze, mv, mg, ml);
      double gx = 0.0, gy = 0.0, gz = 0.0, second = 0.0;
      const int u0 = s ? T.nu0 : 0, nu = s ? T.nu1 : T.nu0;
      for (int k = 0; k < nu; ++k) {
        const int uu = u0 + k;
        const double* Au = A + (size_t)uu * NN * W;
        double Gx = 0.0, Gy = 0.0, Gz = 0.0, Lm = 0.0;
        for (int m = 0; m < N; ++m) {
          const int c = T.occ[uu * N + m];
          const double am = Au[(size_t)(m * N + i) * W];
          Gx += am * mg[c][0]; Gy += am * mg[c][1]; Gz += am * mg[c][2];
          Lm += am * ml[c];
        }
        const double wk = wu[s][k];
        gx += wk * Gx; gy += wk * Gy; gz += wk * Gz;
        second += wk * Lm;
      }
      const double lap_s = second - (gx * gx + gy * gy + gz * gz);
      double jx = 0.0, jy = 0.0, jz = 0.0, jl = 0.0;
      oq_jastrow_vgl_coulomb<NE, double>(S, S, pos, (size_t)W, e, xe, ye, ze, jx, jy, jz, jl,
                                         ee, en);
      const double Gx = gx + jx, Gy = gy + jy, Gz = gz + jz, le = lap_s + jl;
      if (grad) {
        double* gp = grad + ((size_t)w * NE + e) * 3;
        gp[0] = Gx; gp[1] = Gy; gp[2] = Gz;
      }
      if (lap) lap[(size_t)w * NE + e] = le;
      lp_tot += le;
      g2 += Gx * Gx + Gy * Gy + Gz * Gz;
    }
    if (logpsi) {
      double x[3 * NE];
      for (int k = 0; k < NE; ++k)
        for (int c = 0; c < 3; ++c) x[3 * k + c] = pos[(3 * k + c) * W];
      logpsi[w] = lps + oq_jastrow_value(S, x, NE);
    }
  }
  const double ke = -0.5 * (lp_tot + g2);
  const double el = ee + en + ke + S.e_nn;
  const bool ok = live && isfinite(el);
  if (live) {
    if (a.el_trace) a.el_trace[w] = el;
    if (a.eparts) {
      double* ep = a.eparts + (size_t)w * 4;
      ep[0] = ee; ep[1] = en; ep[2] = ke; ep[3] = el;
    }
    if (!ok) atomicOr(a.flags, OQ_FLAG_NAN);
  }
  if (!a.sums) return;
  double vals[6] = {ok ? ee : 0.0, ok ? en : 0.0, ok ? ke : 0.0, ok ? el : 0.0,
                    ok ? el * el : 0.0, ok ? 1.0 : 0.0};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    double v = vals[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    vals[k] = v;
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 5; ++k) atomicAdd(a.sums + k, vals[k]);
    atomicAdd(a.sums + 6, vals[5]);
  }
}
