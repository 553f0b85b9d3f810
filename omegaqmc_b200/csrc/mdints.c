/*
 * mdints.c -- one- and two-electron integrals over Cartesian Gaussian
 * primitives by the McMurchie-Davidson scheme (Hermite expansion
 * coefficients E, Hermite Coulomb integrals R with the Boys function).
 * Host code for the RHF front end that supplies molecular orbitals when no
 * quantum-chemistry package is available.
 *
 * A primitive function f = x_A^i y_A^j z_A^k exp(-a |r - A|^2) (unnormalised).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LMAX 4
#define LSUM (4 * LMAX)     /* largest t+u+v in (ab|cd) */
#define NH (2 * LMAX + 1)   /* Hermite range of one pair, per dimension */

/* Boys function F_n(T), n = 0..nmax, by series (small T) or the
 * asymptotic form (large T) at nmax followed by downward recursion. */
static void boys(int nmax, double T, double* F) {
  if (T < 1e-12) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1);
    return;
  }
  const double eT = exp(-T);
  if (T < 35.0) {
    /* F_nmax = e^{-T} sum_k (2T)^k / ((2n+1)(2n+3)...(2n+2k+1)) */
    double term = 1.0 / (2 * nmax + 1), sum = term;
    for (int k = 1; k < 400; ++k) {
      term *= 2.0 * T / (2 * nmax + 2 * k + 1);
      sum += term;
      if (term < 1e-17 * sum) break;
    }
    F[nmax] = eT * sum;
  } else {
    /* F_n(T) ~ (2n-1)!! / 2^{n+1} sqrt(pi / T^{2n+1}) */
    double df = 1.0;
    for (int k = 1; k <= 2 * nmax - 1; k += 2) df *= k;
    F[nmax] = df / pow(2.0, nmax + 1) * sqrt(M_PI / pow(T, 2 * nmax + 1));
  }
  for (int n = nmax; n > 0; --n) F[n - 1] = (2.0 * T * F[n] + eT) / (2 * n - 1);
}

/* 1-D Hermite coefficients E[i][j][t] for exponents a, b and A-B = Qx */
static void hermite_e(int imax, int jmax, double a, double b, double Qx,
                      double E[LMAX + 3][LMAX + 3][2 * LMAX + 6]) {
  const double p = a + b, mu = a * b / p;
  const double XPA = -b / p * Qx, XPB = a / p * Qx;
  memset(E, 0, sizeof(double) * (LMAX + 3) * (LMAX + 3) * (2 * LMAX + 6));
  E[0][0][0] = exp(-mu * Qx * Qx);
  for (int i = 0; i <= imax; ++i)
    for (int j = 0; j <= jmax; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        double v;
        if (j == 0) {
          v = XPA * E[i - 1][j][t] + (t + 1) * E[i - 1][j][t + 1];
          if (t > 0) v += E[i - 1][j][t - 1] / (2 * p);
        } else {
          v = XPB * E[i][j - 1][t] + (t + 1) * E[i][j - 1][t + 1];
          if (t > 0) v += E[i][j - 1][t - 1] / (2 * p);
        }
        E[i][j][t] = v;
      }
    }
}

/* Hermite Coulomb integrals R[t][u][v] (n = 0) for exponent p, vector PC */
static void hermite_r(int L, double p, double X, double Y, double Z,
                      double R[LSUM + 1][LSUM + 1][LSUM + 1]) {
  static __thread double Rn[LSUM + 1][LSUM + 1][LSUM + 1][LSUM + 1];
  double F[LSUM + 1];
  boys(L, p * (X * X + Y * Y + Z * Z), F);
  double pw = 1.0;
  for (int n = 0; n <= L; ++n) {
    Rn[n][0][0][0] = pw * F[n];
    pw *= -2.0 * p;
  }
  /* R^n_{t,u,v} from R^{n+1} with t+u+v <= L-n */
  for (int n = L - 1; n >= 0; --n) {
    for (int t = 0; t <= L - n; ++t)
      for (int u = 0; u <= L - n - t; ++u)
        for (int v = 0; v <= L - n - t - u; ++v) {
          if (t + u + v == 0) continue;
          double val;
          if (t > 0) {
            val = X * Rn[n + 1][t - 1][u][v];
            if (t > 1) val += (t - 1) * Rn[n + 1][t - 2][u][v];
          } else if (u > 0) {
            val = Y * Rn[n + 1][t][u - 1][v];
            if (u > 1) val += (u - 1) * Rn[n + 1][t][u - 2][v];
          } else {
            val = Z * Rn[n + 1][t][u][v - 1];
            if (v > 1) val += (v - 1) * Rn[n + 1][t][u][v - 2];
          }
          Rn[n][t][u][v] = val;
        }
  }
  for (int t = 0; t <= L; ++t)
    for (int u = 0; u <= L - t; ++u)
      for (int v = 0; v <= L - t - u; ++v) R[t][u][v] = Rn[0][t][u][v];
}

typedef struct {
  double E[3][LMAX + 3][LMAX + 3][2 * LMAX + 6];
} pairE_t;

/* Overlap, kinetic and nuclear-attraction matrices over n primitives.
 * ctr (n,3), alpha (n), pw (n,3) Cartesian powers; nuclei (natm,3), Z. */
int md_one_electron(int n, const double* ctr, const double* alpha, const int* pw,
                    int natm, const double* nuc, const double* Z, double* S, double* T,
                    double* V) {
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      const double ea = alpha[a], eb = alpha[b], p = ea + eb;
      const int* ia = pw + 3 * a;
      const int* ib = pw + 3 * b;
      double E[3][LMAX + 3][LMAX + 3][2 * LMAX + 6];
      for (int d = 0; d < 3; ++d)
        hermite_e(ia[d] + 1, ib[d] + 2, ea, eb, ctr[3 * a + d] - ctr[3 * b + d], E[d]);
      const double pref = pow(M_PI / p, 1.5);
      double s1[3], d1[3];
      for (int d = 0; d < 3; ++d) {
        const int i = ia[d], j = ib[d];
        s1[d] = E[d][i][j][0];
        double dd = -2.0 * eb * (2 * j + 1) * E[d][i][j][0] + 4.0 * eb * eb * E[d][i][j + 2][0];
        if (j >= 2) dd += j * (j - 1) * E[d][i][j - 2][0];
        d1[d] = dd;
      }
      S[a * n + b] = pref * s1[0] * s1[1] * s1[2];
      T[a * n + b] = -0.5 * pref * (d1[0] * s1[1] * s1[2] + s1[0] * d1[1] * s1[2] +
                                    s1[0] * s1[1] * d1[2]);
      /* nuclear attraction */
      const double P[3] = {(ea * ctr[3 * a] + eb * ctr[3 * b]) / p,
                           (ea * ctr[3 * a + 1] + eb * ctr[3 * b + 1]) / p,
                           (ea * ctr[3 * a + 2] + eb * ctr[3 * b + 2]) / p};
      const int L = ia[0] + ib[0] + ia[1] + ib[1] + ia[2] + ib[2];
      double v = 0.0;
      for (int c = 0; c < natm; ++c) {
        double R[LSUM + 1][LSUM + 1][LSUM + 1];
        hermite_r(L, p, P[0] - nuc[3 * c], P[1] - nuc[3 * c + 1], P[2] - nuc[3 * c + 2], R);
        double acc = 0.0;
        for (int t = 0; t <= ia[0] + ib[0]; ++t)
          for (int u = 0; u <= ia[1] + ib[1]; ++u)
            for (int w = 0; w <= ia[2] + ib[2]; ++w)
              acc += E[0][ia[0]][ib[0]][t] * E[1][ia[1]][ib[1]][u] * E[2][ia[2]][ib[2]][w] *
                     R[t][u][w];
        v -= Z[c] * acc;
      }
      V[a * n + b] = 2.0 * M_PI / p * v;
    }
  return 0;
}

/* Two-electron integrals (ab|cd) over n primitives, full n^4 output
 * (chemists' notation), using the 8-fold permutational symmetry. */
int md_eri(int n, const double* ctr, const double* alpha, const int* pw, double* out) {
  const int np = n * (n + 1) / 2;
  /* Hermite expansion of every pair: coefficient lists over (t,u,v) */
  int* pa = (int*)malloc(sizeof(int) * np);
  int* pb = (int*)malloc(sizeof(int) * np);
  double* pp = (double*)malloc(sizeof(double) * np);
  double* PP = (double*)malloc(sizeof(double) * 3 * np);
  const int NHC = (2 * LMAX + 1) * (2 * LMAX + 1) * (2 * LMAX + 1);
  double* Ehc = (double*)calloc((size_t)np * NHC, sizeof(double));
  int* Lp = (int*)malloc(sizeof(int) * 3 * np);
  int k = 0;
  for (int a = 0; a < n; ++a)
    for (int b = 0; b <= a; ++b, ++k) {
      pa[k] = a; pb[k] = b;
      const double ea = alpha[a], eb = alpha[b], p = ea + eb;
      pp[k] = p;
      double E[3][LMAX + 3][LMAX + 3][2 * LMAX + 6];
      for (int d = 0; d < 3; ++d) {
        hermite_e(pw[3 * a + d], pw[3 * b + d], ea, eb, ctr[3 * a + d] - ctr[3 * b + d], E[d]);
        PP[3 * k + d] = (ea * ctr[3 * a + d] + eb * ctr[3 * b + d]) / p;
        Lp[3 * k + d] = pw[3 * a + d] + pw[3 * b + d];
      }
      for (int t = 0; t <= Lp[3 * k]; ++t)
        for (int u = 0; u <= Lp[3 * k + 1]; ++u)
          for (int v = 0; v <= Lp[3 * k + 2]; ++v)
            Ehc[(size_t)k * NHC + (t * (2 * LMAX + 1) + u) * (2 * LMAX + 1) + v] =
                E[0][pw[3 * a]][pw[3 * b]][t] * E[1][pw[3 * a + 1]][pw[3 * b + 1]][u] *
                E[2][pw[3 * a + 2]][pw[3 * b + 2]][v];
    }
#pragma omp parallel for schedule(dynamic, 4)
  for (int k1 = 0; k1 < np; ++k1) {
    double R[LSUM + 1][LSUM + 1][LSUM + 1];
    for (int k2 = 0; k2 <= k1; ++k2) {
      const double p = pp[k1], q = pp[k2], al = p * q / (p + q);
      const int L = Lp[3 * k1] + Lp[3 * k1 + 1] + Lp[3 * k1 + 2] + Lp[3 * k2] + Lp[3 * k2 + 1] +
                    Lp[3 * k2 + 2];
      hermite_r(L, al, PP[3 * k1] - PP[3 * k2], PP[3 * k1 + 1] - PP[3 * k2 + 1],
                PP[3 * k1 + 2] - PP[3 * k2 + 2], R);
      double acc = 0.0;
      const double* E1 = Ehc + (size_t)k1 * NHC;
      const double* E2 = Ehc + (size_t)k2 * NHC;
      for (int t = 0; t <= Lp[3 * k1]; ++t)
        for (int u = 0; u <= Lp[3 * k1 + 1]; ++u)
          for (int v = 0; v <= Lp[3 * k1 + 2]; ++v) {
            const double e1 = E1[(t * (2 * LMAX + 1) + u) * (2 * LMAX + 1) + v];
            if (e1 == 0.0) continue;
            double inner = 0.0;
            for (int tt = 0; tt <= Lp[3 * k2]; ++tt)
              for (int uu = 0; uu <= Lp[3 * k2 + 1]; ++uu)
                for (int vv = 0; vv <= Lp[3 * k2 + 2]; ++vv) {
                  const double e2 = E2[(tt * (2 * LMAX + 1) + uu) * (2 * LMAX + 1) + vv];
                  const double sg = ((tt + uu + vv) & 1) ? -1.0 : 1.0;
                  inner += sg * e2 * R[t + tt][u + uu][v + vv];
                }
            acc += e1 * inner;
          }
      const double val = 2.0 * pow(M_PI, 2.5) / (p * q * sqrt(p + q)) * acc;
      const int a = pa[k1], b = pb[k1], c = pa[k2], d = pb[k2];
      const size_t n1 = n, n2 = (size_t)n * n, n3 = n2 * n;
      out[a * n3 + b * n2 + c * n1 + d] = val;
      out[b * n3 + a * n2 + c * n1 + d] = val;
      out[a * n3 + b * n2 + d * n1 + c] = val;
      out[b * n3 + a * n2 + d * n1 + c] = val;
      out[c * n3 + d * n2 + a * n1 + b] = val;
      out[d * n3 + c * n2 + a * n1 + b] = val;
      out[c * n3 + d * n2 + b * n1 + a] = val;
      out[d * n3 + c * n2 + b * n1 + a] = val;
    }
  }
  free(pa); free(pb); free(pp); free(PP); free(Ehc); free(Lp);
  return 0;
}
