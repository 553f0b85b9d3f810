// AO -> MO evaluation at one electron position, fused: the contracted radial
// part of every exponent group is formed once, the angular factors applied
// per shell component, and each AO is folded into the occupied-MO
// accumulators straight away (no AO row is ever stored).
//
// Follows cgs_sph_get / cgs_sph_vgl (OmegaQMC/psi/gto.py:1012-1186),
// _radial_vgl (gto.py:781-811) and evaluate_cusp_s[_vgl]
// (OmegaQMC/psi/shell.py:54-148).
#pragma once
#include "oqmc_common.cuh"

// C is (nbf x NOCC) row-major in shared memory, element type TC.
// Value only: mv[m] = sum_a C[a][m] chi_a(x).
template <int NOCC, typename TC>
__device__ __forceinline__ void oq_mo_val(const OqSystem& S, const TC* __restrict__ C,
                                          double x, double y, double z,
                                          double mv[NOCC]) {
#pragma unroll
  for (int m = 0; m < NOCC; ++m) mv[m] = 0.0;
  for (int g = 0; g < S.ngroup; ++g) {
    const int ia = S.g_iat[g];
    const double dx = x - S.nuc[ia][0], dy = y - S.nuc[ia][1], dz = z - S.nuc[ia][2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const int ncol = S.g_ncol[g], np = S.g_n[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    double R[OQ_MAX_COL] = {0.0, 0.0, 0.0, 0.0};
    for (int p = 0; p < np; ++p) {
      const double e = exp(-S.alpha[off + p] * r2);
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol) R[k] += S.norm[S.s_norm[sh0 + k] + p] * e;
    }
    if (S.has_spl) {
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol && S.s_spl[sh0 + k] >= 0) {
          double gp, gpp;
          oq_spline_gdd(S, S.s_spl[sh0 + k], r2, R[k], gp, gpp);
        }
    }
    const int am = S.g_am[g];
#pragma unroll
    for (int k = 0; k < OQ_MAX_COL; ++k) {
      if (k >= ncol) break;
      const int sh = sh0 + k;
      const int ao = S.s_ao[sh];
      if (am == 0) {
        double v = R[k];
        if (S.s_cusp[sh]) v = oq_cusp_val(S, ia, sqrt(r2), v);
#pragma unroll
        for (int m = 0; m < NOCC; ++m) mv[m] += (double)C[ao * NOCC + m] * v;
      } else if (am == 1) {
        const double v0 = R[k] * dx, v1 = R[k] * dy, v2 = R[k] * dz;
#pragma unroll
        for (int m = 0; m < NOCC; ++m)
          mv[m] += (double)C[ao * NOCC + m] * v0 + (double)C[(ao + 1) * NOCC + m] * v1 +
                   (double)C[(ao + 2) * NOCC + m] * v2;
      } else if (am == 2) {
        double Y[5], dY[5][3];
        oq_harm_d<double>(dx, dy, dz, Y, dY);
        for (int c = 0; c < 5; ++c) {
          const double v = R[k] * Y[c];
#pragma unroll
          for (int m = 0; m < NOCC; ++m) mv[m] += (double)C[(ao + c) * NOCC + m] * v;
        }
      } else {
        const int nc = 2 * am + 1;
        for (int c = 0; c < nc; ++c) {
          double Yc, dY[3];
          oq_harm_table<double>(S.harm, am, c, dx, dy, dz, Yc, dY);
          const double v = R[k] * Yc;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) mv[m] += (double)C[(ao + c) * NOCC + m] * v;
        }
      }
    }
  }
}

// Value, gradient and Laplacian of the occupied MOs at x (FP64).
template <int NOCC, typename TC>
__device__ __forceinline__ void oq_mo_vgl(const OqSystem& S, const TC* __restrict__ C,
                                          double x, double y, double z,
                                          double mv[NOCC], double mg[NOCC][3],
                                          double ml[NOCC]) {
#pragma unroll
  for (int m = 0; m < NOCC; ++m) {
    mv[m] = 0.0; mg[m][0] = mg[m][1] = mg[m][2] = 0.0; ml[m] = 0.0;
  }
  for (int g = 0; g < S.ngroup; ++g) {
    const int ia = S.g_iat[g];
    const double dx = x - S.nuc[ia][0], dy = y - S.nuc[ia][1], dz = z - S.nuc[ia][2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const int ncol = S.g_ncol[g], np = S.g_n[g], off = S.g_off[g], sh0 = S.g_shell0[g];
    double R[OQ_MAX_COL] = {0, 0, 0, 0}, Rp[OQ_MAX_COL] = {0, 0, 0, 0},
           Rl[OQ_MAX_COL] = {0, 0, 0, 0};
    for (int p = 0; p < np; ++p) {
      const double a = S.alpha[off + p];
      const double e = exp(-a * r2);
      const double fp = -2.0 * a * e;
      const double fl = (4.0 * a * a * r2 - 6.0 * a) * e;
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol) {
          const double n = S.norm[S.s_norm[sh0 + k] + p];
          R[k] += n * e;
          Rp[k] += n * fp;
          Rl[k] += n * fl;
        }
    }
    if (S.has_spl) {
      // spline triple (g, 2 g', 6 g' + 4 s g''), _radial_vgl_spline (gto.py:226-240)
#pragma unroll
      for (int k = 0; k < OQ_MAX_COL; ++k)
        if (k < ncol && S.s_spl[sh0 + k] >= 0) {
          double gv, gp, gpp;
          oq_spline_gdd(S, S.s_spl[sh0 + k], r2, gv, gp, gpp);
          R[k] = gv;
          Rp[k] = 2.0 * gp;
          Rl[k] = 6.0 * gp + 4.0 * r2 * gpp;
        }
    }
    const int am = S.g_am[g];
#pragma unroll
    for (int k = 0; k < OQ_MAX_COL; ++k) {
      if (k >= ncol) break;
      const int sh = sh0 + k;
      const int ao = S.s_ao[sh];
      if (am == 0) {
        double v = R[k], gp = Rp[k], l = Rl[k];
        if (S.s_cusp[sh]) oq_cusp_vgl(S, ia, sqrt(r2), v, gp, l);
        const double gx = gp * dx, gy = gp * dy, gz = gp * dz;
#pragma unroll
        for (int m = 0; m < NOCC; ++m) {
          const double c = (double)C[ao * NOCC + m];
          mv[m] += c * v; mg[m][0] += c * gx; mg[m][1] += c * gy; mg[m][2] += c * gz;
          ml[m] += c * l;
        }
      } else {
        const int nc = 2 * am + 1;
        double Yd[5], dYd[5][3];
        if (am == 2) oq_harm_d<double>(dx, dy, dz, Yd, dYd);
        const double lfac = Rl[k] + 2.0 * am * Rp[k];
        for (int c = 0; c < nc; ++c) {
          double Y, dY[3];
          if (am == 1) {
            Y = (c == 0) ? dx : (c == 1) ? dy : dz;
            dY[0] = (c == 0); dY[1] = (c == 1); dY[2] = (c == 2);
          } else if (am == 2) {
            Y = Yd[c]; dY[0] = dYd[c][0]; dY[1] = dYd[c][1]; dY[2] = dYd[c][2];
          } else {
            oq_harm_table<double>(S.harm, am, c, dx, dy, dz, Y, dY);
          }
          const double v = R[k] * Y;
          const double gx = Rp[k] * dx * Y + R[k] * dY[0];
          const double gy = Rp[k] * dy * Y + R[k] * dY[1];
          const double gz = Rp[k] * dz * Y + R[k] * dY[2];
          const double l = lfac * Y;
#pragma unroll
          for (int m = 0; m < NOCC; ++m) {
            const double cc = (double)C[(ao + c) * NOCC + m];
            mv[m] += cc * v; mg[m][0] += cc * gx; mg[m][1] += cc * gy;
            mg[m][2] += cc * gz; ml[m] += cc * l;
          }
        }
      }
    }
  }
}
