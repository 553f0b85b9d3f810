/*
 * vmc_ref.c -- CPU FP64 restatement of the reference's GTO-VMC algorithm
 * (TEST INFRASTRUCTURE: the oracle's compiled leg and the timed CPU
 * baseline; never part of the product path).
 *
 * Follows the reference step by step:
 *  - all-electron Gaussian proposal, rejected (ratio 0) when any e-e or e-n
 *    distance is below MIN_DIST_THRESHOLD = 1e-4 (OmegaQMC/vmc_gto.py:815-839);
 *  - log|psi| recomputed for the old AND the new configuration every step
 *    (vmc_gto.py:893-897), acceptance u < exp(2 dlogpsi) * ratio (899-902);
 *  - the local energy of every walker after each step
 *    (vmc_gto.py:1019-1026): Coulomb with eps inside the sqrt
 *    (psi/gto.py:2406-2451) and the analytic kinetic energy with a fresh
 *    inverse of each spin block (gto.py:728-778, 2506-2579);
 *  - AO values and VGL as cgs_sph_get / cgs_sph_vgl (gto.py:1012-1186),
 *    cusp-corrected s shells as evaluate_cusp_s[_vgl] (psi/shell.py:54-148).
 * Random numbers: one xoshiro256** stream per walker (numpy/JAX streams
 * cannot be reproduced here), so comparisons with the GPU are statistical.
 * OpenMP over walkers.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

#include "../include/oqmc_b200.h"

#define MAXE 32
#define MAXO 16
#define MAXBF 160
#define EPSD 2.220446049250313e-16

typedef struct {
  const oqmc_system_desc* d;
  int ao_of_shell[512];
  int norm_of_shell[512];
  int prim_of_group[256];
} sys_t;

static void sys_init(sys_t* s, const oqmc_system_desc* d) {
  s->d = d;
  int ao = 0, sh = 0, no = 0, pr = 0;
  for (int g = 0; g < d->ngroup; ++g) {
    s->prim_of_group[g] = pr;
    for (int k = 0; k < d->group_ncol[g]; ++k) {
      s->ao_of_shell[sh] = ao;
      s->norm_of_shell[sh] = no;
      ao += 2 * d->group_am[g] + 1;
      no += d->group_nprim[g];
      ++sh;
    }
    pr += d->group_nprim[g];
  }
}

/* real solid harmonics, order of _angular_cartesian (gto.py:607-671) */
static void harm(int am, double x, double y, double z, double* Y, double (*G)[3]) {
  const double cd1 = 1.7320508075688772, cd2 = 0.8660254037844386;
  if (am == 1) {
    Y[0] = x; Y[1] = y; Y[2] = z;
    for (int c = 0; c < 3; ++c) for (int k = 0; k < 3; ++k) G[c][k] = (c == k);
    return;
  }
  if (am == 2) {
    Y[0] = cd1 * x * y; Y[1] = cd1 * y * z; Y[2] = 0.5 * (2 * z * z - x * x - y * y);
    Y[3] = cd1 * x * z; Y[4] = cd2 * (x * x - y * y);
    double g[5][3] = {{cd1 * y, cd1 * x, 0}, {0, cd1 * z, cd1 * y}, {-x, -y, 2 * z},
                      {cd1 * z, 0, cd1 * x}, {cd1 * x, -cd1 * y, 0}};
    memcpy(G, g, sizeof(g));
    return;
  }
  if (am == 3) {
    const double f1 = sqrt(2.5) * 0.5, f2 = 3 * f1, f3 = sqrt(15.0), f4 = sqrt(1.5) * 0.5,
                 f5 = sqrt(6.0), f6 = 1.5, f7 = f3 * 0.5;
    const double xx = x * x, yy = y * y, zz = z * z;
    Y[0] = y * (f2 * xx - f1 * yy);
    Y[1] = f3 * x * y * z;
    Y[2] = y * (f5 * zz - f4 * (xx + yy));
    Y[3] = z * (zz - f6 * (xx + yy));
    Y[4] = x * (f5 * zz - f4 * (xx + yy));
    Y[5] = z * f7 * (xx - yy);
    Y[6] = -x * (f2 * yy - f1 * xx);
    double g[7][3] = {
        {2 * f2 * x * y, f2 * xx - 3 * f1 * yy, 0},
        {f3 * y * z, f3 * x * z, f3 * x * y},
        {-2 * f4 * x * y, f5 * zz - f4 * xx - 3 * f4 * yy, 2 * f5 * y * z},
        {-2 * f6 * x * z, -2 * f6 * y * z, 3 * zz - f6 * (xx + yy)},
        {f5 * zz - 3 * f4 * xx - f4 * yy, -2 * f4 * x * y, 2 * f5 * x * z},
        {2 * f7 * x * z, -2 * f7 * y * z, f7 * (xx - yy)},
        {-f2 * yy + 3 * f1 * xx, -2 * f2 * x * y, 0}};
    memcpy(G, g, sizeof(g));
    return;
  }
  if (am == 4) {
    const double c1 = 2.9580398915498085, c2 = 6.2749501990055672, c3 = 2.0916500663351894,
                 c4 = 1.1180339887498949, c5 = 6.7082039324993694, c6 = 2.3717082451262845,
                 c7 = 3.1622776601683795, c8 = 0.55901699437494745, c9 = 3.3541019662496847,
                 c10 = 0.73950997288745213, c11 = 4.4370598373247132;
    const double xx = x * x, yy = y * y, zz = z * z;
    Y[0] = c1 * (xx * x * y - x * yy * y);
    Y[1] = y * z * (c2 * xx - c3 * yy);
    Y[2] = x * y * c4 * (-xx - yy) + c5 * x * y * zz;
    Y[3] = -c6 * xx * y * z - c6 * yy * y * z + c7 * y * zz * z;
    Y[4] = 0.375 * (xx * xx + yy * yy + 2 * xx * yy) + zz * zz - 3 * zz * (xx + yy);
    Y[5] = -(c6 * xx * x * z + c6 * x * yy * z - c7 * x * zz * z);
    Y[6] = c8 * (yy * yy - xx * xx) + c9 * zz * (xx - yy);
    Y[7] = -x * z * (c2 * yy - c3 * xx);
    Y[8] = c10 * (xx * xx + yy * yy) - c11 * xx * yy;
    double g[9][3] = {
        {c1 * (3 * xx * y - yy * y), c1 * (xx * x - 3 * x * yy), 0},
        {2 * c2 * x * y * z, c2 * xx * z - 3 * c3 * yy * z, c2 * xx * y - c3 * yy * y},
        {-3 * c4 * xx * y - c4 * yy * y + c5 * y * zz, -c4 * xx * x - 3 * c4 * x * yy + c5 * x * zz,
         2 * c5 * x * y * z},
        {-2 * c6 * x * y * z, -c6 * xx * z - 3 * c6 * yy * z + c7 * zz * z,
         -c6 * xx * y - c6 * yy * y + 3 * c7 * y * zz},
        {1.5 * xx * x + 1.5 * x * yy - 6 * x * zz, 1.5 * yy * y + 1.5 * xx * y - 6 * y * zz,
         4 * zz * z - 6 * z * (xx + yy)},
        {-3 * c6 * xx * z - c6 * yy * z + c7 * zz * z, -2 * c6 * x * y * z,
         -c6 * xx * x - c6 * x * yy + 3 * c7 * x * zz},
        {-4 * c8 * xx * x + 2 * c9 * x * zz, 4 * c8 * yy * y - 2 * c9 * y * zz,
         2 * c9 * z * (xx - yy)},
        {-c2 * yy * z + 3 * c3 * xx * z, -2 * c2 * x * y * z, -c2 * x * yy + c3 * xx * x},
        {4 * c10 * xx * x - 2 * c11 * x * yy, 4 * c10 * yy * y - 2 * c11 * xx * y, 0}};
    memcpy(G, g, sizeof(g));
    return;
  }
  Y[0] = 1.0;
  G[0][0] = G[0][1] = G[0][2] = 0.0;
}

static double cusp_val(const oqmc_system_desc* d, int ia, double r, double R) {
  const double rc = d->cusp_rc[ia];
  const double* c = d->cusp_coeff + 8 * ia;
  double b = 0.0;
  if (r < rc) {
    const double s = r / rc;
    b = 1.0 - 10.0 * s * s * s + 15.0 * s * s * s * s - 6.0 * s * s * s * s * s;
  }
  const double sl = d->cusp_q0[ia] * exp(-d->Z[ia] * r);
  double poly = c[1];
  const double s = r / rc;
  double sk = s * s;
  for (int k = 2; k < 8; ++k) { poly += c[k] * sk; sk *= s; }
  return c[0] * (1.0 - b) * R + b * sl * poly;
}

static void cusp_vgl(const oqmc_system_desc* d, int ia, double r, double* R, double* Rp,
                     double* Rl) {
  const double rc = d->cusp_rc[ia], Z = d->Z[ia];
  const double* c = d->cusp_coeff + 8 * ia;
  const double c0 = c[0];
  if (!(r < rc)) { *R *= c0; *Rp *= c0; *Rl *= c0; return; }
  const double s = r / rc, oms = 1.0 - s;
  const double b = 1.0 - 10.0 * s * s * s + 15.0 * s * s * s * s - 6.0 * s * s * s * s * s;
  const double bp = -(30.0 / rc) * s * s * oms * oms;
  const double bp_r = -(30.0 / (rc * rc * rc)) * r * oms * oms;
  const double bpp = -(60.0 / (rc * rc)) * s * oms * (1.0 - 2.0 * s);
  const double BL = bpp + 2.0 * bp_r;
  const double Av = c0 * (1.0 - b) * *R;
  const double Ag = c0 * (-bp_r * *R + (1.0 - b) * *Rp);
  const double Al = c0 * (-BL * *R + (1.0 - b) * *Rl - 2.0 * r * bp * *Rp);
  const double Sl = d->cusp_q0[ia] * exp(-Z * r);
  double P = c[1], P1 = 0.0, P2 = 0.0;
  for (int k = 2; k < 8; ++k) {
    P += c[k] * pow(s, k);
    P1 += k * c[k] * pow(s, k - 1) / rc;
    P2 += k * (k - 1) * c[k] * pow(s, k - 2) / (rc * rc);
  }
  const double Q = b * Sl * P;
  const double Qp = bp * Sl * P - Z * b * Sl * P + b * Sl * P1;
  const double Qpp = bpp * Sl * P + Z * Z * b * Sl * P + b * Sl * P2 +
                     2.0 * (-Z * bp * Sl * P + bp * Sl * P1 - Z * b * Sl * P1);
  *R = Av + Q;
  *Rp = Ag + Qp / r;
  *Rl = Al + Qpp + 2.0 * Qp / r;
}

/* MO values (and optionally gradients/Laplacians) at one position */
static void mo_eval(const sys_t* S, const double* x, double* mv, double (*mg)[3], double* ml) {
  const oqmc_system_desc* d = S->d;
  const int no = d->nocc;
  for (int m = 0; m < no; ++m) {
    mv[m] = 0.0;
    if (mg) { mg[m][0] = mg[m][1] = mg[m][2] = 0.0; ml[m] = 0.0; }
  }
  int sh = 0;
  for (int g = 0; g < d->ngroup; ++g) {
    const int ia = d->group_atom[g], am = d->group_am[g], np = d->group_nprim[g];
    const double dx = x[0] - d->nuc[3 * ia], dy = x[1] - d->nuc[3 * ia + 1],
                 dz = x[2] - d->nuc[3 * ia + 2];
    const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
    const double* al = d->alpha + S->prim_of_group[g];
    double Y[9], G[9][3];
    harm(am, dx, dy, dz, Y, G);
    for (int k = 0; k < d->group_ncol[g]; ++k, ++sh) {
      const double* nm = d->norm + S->norm_of_shell[sh];
      double R = 0.0, Rp = 0.0, Rl = 0.0;
      for (int p = 0; p < np; ++p) {
        const double e = exp(-al[p] * r2) * nm[p];
        R += e;
        if (mg) { Rp += -2.0 * al[p] * e; Rl += (4.0 * al[p] * al[p] * r2 - 6.0 * al[p]) * e; }
      }
      const int cusp = d->cusp && am == 0 && d->shell_cusp[sh];
      const int ao = S->ao_of_shell[sh];
      if (!mg) {
        if (cusp) R = cusp_val(d, ia, r, R);
        for (int c = 0; c < 2 * am + 1; ++c) {
          const double v = R * Y[c];
          for (int m = 0; m < no; ++m) mv[m] += d->C[(ao + c) * no + m] * v;
        }
      } else {
        if (cusp) cusp_vgl(d, ia, r, &R, &Rp, &Rl);
        const double lf = Rl + 2.0 * am * Rp;
        for (int c = 0; c < 2 * am + 1; ++c) {
          const double v = R * Y[c];
          const double gx = Rp * dx * Y[c] + R * G[c][0];
          const double gy = Rp * dy * Y[c] + R * G[c][1];
          const double gz = Rp * dz * Y[c] + R * G[c][2];
          const double l = lf * Y[c];
          for (int m = 0; m < no; ++m) {
            const double cc = d->C[(ao + c) * no + m];
            mv[m] += cc * v; mg[m][0] += cc * gx; mg[m][1] += cc * gy; mg[m][2] += cc * gz;
            ml[m] += cc * l;
          }
        }
      }
    }
  }
}

/* LU with partial pivoting: log|det| and (optionally) the inverse */
static int lu_inv(int n, double* a, double* inv, double* logdet) {
  int piv[MAXO];
  *logdet = 0.0;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = fabs(a[k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (fabs(a[i * n + k]) > best) { best = fabs(a[i * n + k]); p = i; }
    piv[k] = p;
    if (!(best > 0.0)) return 0;
    if (p != k)
      for (int j = 0; j < n; ++j) { double t = a[k * n + j]; a[k * n + j] = a[p * n + j]; a[p * n + j] = t; }
    *logdet += log(fabs(a[k * n + k]));
    for (int i = k + 1; i < n; ++i) {
      const double f = a[i * n + k] / a[k * n + k];
      a[i * n + k] = f;
      for (int j = k + 1; j < n; ++j) a[i * n + j] -= f * a[k * n + j];
    }
  }
  if (!inv) return 1;
  for (int col = 0; col < n; ++col) {
    double b[MAXO];
    for (int i = 0; i < n; ++i) b[i] = (i == col);
    for (int k = 0; k < n; ++k) { const double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
    for (int i = 0; i < n; ++i) for (int j = 0; j < i; ++j) b[i] -= a[i * n + j] * b[j];
    for (int i = n - 1; i >= 0; --i) {
      for (int j = i + 1; j < n; ++j) b[i] -= a[i * n + j] * b[j];
      b[i] /= a[i * n + i];
    }
    for (int i = 0; i < n; ++i) inv[i * n + col] = b[i];
  }
  return 1;
}

static double pade(double a, double b, double r) { return a * r / (1.0 + b * r); }

static double jastrow(const oqmc_system_desc* d, const double* X) {
  const int ne = d->n_e;
  double J = 0.0;
  if (d->has_j2)
    for (int i = 0; i < ne; ++i)
      for (int j = i + 1; j < ne; ++j) {
        const double dx = X[3 * i] - X[3 * j], dy = X[3 * i + 1] - X[3 * j + 1],
                     dz = X[3 * i + 2] - X[3 * j + 2];
        const int o = ((i & 1) == (j & 1)) ? 0 : 2;
        J += pade(d->j2[o], d->j2[o + 1], sqrt(dx * dx + dy * dy + dz * dz));
      }
  if (d->has_j1)
    for (int i = 0; i < ne; ++i)
      for (int I = 0; I < d->natm; ++I) {
        const double dx = X[3 * i] - d->nuc[3 * I], dy = X[3 * i + 1] - d->nuc[3 * I + 1],
                     dz = X[3 * i + 2] - d->nuc[3 * I + 2];
        J += pade(d->j1[2 * I], d->j1[2 * I + 1], sqrt(dx * dx + dy * dy + dz * dz));
      }
  return J;
}

static double log_psi(const sys_t* S, const double* X) {
  const oqmc_system_desc* d = S->d;
  const int no = d->nocc;
  double tot = 0.0;
  for (int s = 0; s < 2; ++s) {
    double a[MAXO * MAXO];
    for (int i = 0; i < no; ++i) mo_eval(S, X + 3 * (2 * i + s), a + i * no, NULL, NULL);
    double ld;
    if (!lu_inv(no, a, NULL, &ld)) return -INFINITY;
    tot += ld;
  }
  return tot + jastrow(d, X);
}

/* ee, en, ke, total */
static void local_energy(const sys_t* S, const double* X, double* out) {
  const oqmc_system_desc* d = S->d;
  const int no = d->nocc, ne = d->n_e;
  double A[2][MAXO * MAXO];
  for (int s = 0; s < 2; ++s) {
    double a[MAXO * MAXO], ld;
    for (int i = 0; i < no; ++i) mo_eval(S, X + 3 * (2 * i + s), a + i * no, NULL, NULL);
    if (!lu_inv(no, a, A[s], &ld)) { out[0] = out[1] = out[2] = out[3] = NAN; return; }
  }
  double lap_tot = 0.0, g2 = 0.0, ee = 0.0, en = 0.0;
  for (int e = 0; e < ne; ++e) {
    const int s = e & 1, i = e >> 1;
    double mv[MAXO], mg[MAXO][3], ml[MAXO];
    mo_eval(S, X + 3 * e, mv, mg, ml);
    double gx = 0, gy = 0, gz = 0, lp = 0;
    for (int m = 0; m < no; ++m) {
      const double am = A[s][m * no + i];
      gx += am * mg[m][0]; gy += am * mg[m][1]; gz += am * mg[m][2]; lp += am * ml[m];
    }
    lp -= gx * gx + gy * gy + gz * gz;
    for (int j = 0; j < ne; ++j) {
      if (j == e) continue;
      const double dx = X[3 * e] - X[3 * j], dy = X[3 * e + 1] - X[3 * j + 1],
                   dz = X[3 * e + 2] - X[3 * j + 2];
      const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
      if (j > e) ee += 1.0 / sqrt(r2 + EPSD);
      if (d->has_j2) {
        const int o = ((e & 1) == (j & 1)) ? 0 : 2;
        const double a = d->j2[o], b = d->j2[o + 1], den = 1.0 + b * r;
        const double up = a / (den * den), upp = -2.0 * a * b / (den * den * den);
        gx += up / r * dx; gy += up / r * dy; gz += up / r * dz; lp += upp + 2.0 * up / r;
      }
    }
    for (int I = 0; I < d->natm; ++I) {
      const double dx = X[3 * e] - d->nuc[3 * I], dy = X[3 * e + 1] - d->nuc[3 * I + 1],
                   dz = X[3 * e + 2] - d->nuc[3 * I + 2];
      const double r2 = dx * dx + dy * dy + dz * dz, r = sqrt(r2);
      en -= d->Z[I] / sqrt(r2 + EPSD);
      if (d->has_j1) {
        const double a = d->j1[2 * I], b = d->j1[2 * I + 1], den = 1.0 + b * r;
        const double up = a / (den * den), upp = -2.0 * a * b / (den * den * den);
        gx += up / r * dx; gy += up / r * dy; gz += up / r * dz; lp += upp + 2.0 * up / r;
      }
    }
    lap_tot += lp;
    g2 += gx * gx + gy * gy + gz * gz;
  }
  out[0] = ee; out[1] = en; out[2] = -0.5 * (lap_tot + g2);
  out[3] = ee + en + out[2] + d->e_nn;
}

/* xoshiro256** (Blackman & Vigna) seeded by splitmix64 */
typedef struct { uint64_t s[4]; int has; double spare; } rng_t;
static uint64_t splitmix(uint64_t* x) {
  uint64_t z = (*x += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t next64(rng_t* r) {
  const uint64_t res = rotl(r->s[1] * 5, 7) * 9, t = r->s[1] << 17;
  r->s[2] ^= r->s[0]; r->s[3] ^= r->s[1]; r->s[1] ^= r->s[2]; r->s[0] ^= r->s[3];
  r->s[2] ^= t; r->s[3] = rotl(r->s[3], 45);
  return res;
}
static double u01(rng_t* r) { return ((next64(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double normal(rng_t* r) {
  if (r->has) { r->has = 0; return r->spare; }
  const double a = sqrt(-2.0 * log(u01(r))), t = 6.283185307179586 * u01(r);
  r->spare = a * sin(t); r->has = 1;
  return a * cos(t);
}

static int valid_move(const oqmc_system_desc* d, const double* X) {
  const double thr = 1e-4;
  for (int i = 0; i < d->n_e; ++i) {
    for (int j = i + 1; j < d->n_e; ++j) {
      const double dx = X[3 * i] - X[3 * j], dy = X[3 * i + 1] - X[3 * j + 1],
                   dz = X[3 * i + 2] - X[3 * j + 2];
      if (sqrt(dx * dx + dy * dy + dz * dz) < thr) return 0;
    }
    for (int I = 0; I < d->natm; ++I) {
      const double dx = X[3 * i] - d->nuc[3 * I], dy = X[3 * i + 1] - d->nuc[3 * I + 1],
                   dz = X[3 * i + 2] - d->nuc[3 * I + 2];
      if (sqrt(dx * dx + dy * dy + dz * dz) < thr) return 0;
    }
  }
  return 1;
}

/* The restatement covers Pade J1/J2, cusp-corrected s shells and a single
 * determinant; descriptors with B-spline, J3 or spline-AO terms are refused
 * rather than evaluated without them. */
static int supported(const oqmc_system_desc* d) {
  return !d->has_bs1 && !d->has_bs2 && !d->has_j3 && !d->has_spl && d->n_e <= MAXE &&
         d->nocc <= MAXO && d->nbf <= MAXBF;
}

/* Full evaluation of W walkers: logpsi (W) and eparts (W x 4).  Returns 0,
 * or -1 for a descriptor outside the restatement. */
int vmc_ref_eval(const oqmc_system_desc* d, const double* X, int W, double* logpsi,
                 double* eparts, int nthreads) {
  if (!supported(d)) return -1;
  sys_t S;
  sys_init(&S, d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int w = 0; w < W; ++w) {
    const double* x = X + (size_t)w * 3 * d->n_e;
    logpsi[w] = log_psi(&S, x);
    local_energy(&S, x, eparts + 4 * (size_t)w);
  }
  return 0;
}

/* n_steps reference steps (all-electron move + E_L) on W walkers in place.
 * series: (n_steps, 4) walker means of ee, en, ke, E_L; acc: mean acceptance.
 * Returns 0, or -1 for a descriptor outside the restatement. */
int vmc_ref_run(const oqmc_system_desc* d, double* X, int W, int n_steps, double step,
                uint64_t seed, double* series, double* acc, int nthreads) {
  if (!supported(d)) return -1;
  sys_t S;
  sys_init(&S, d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int ne = d->n_e;
  double* ep = (double*)malloc(sizeof(double) * 4 * (size_t)W);
  int* accw = (int*)calloc((size_t)W, sizeof(int));
  memset(series, 0, sizeof(double) * 4 * (size_t)n_steps);
  for (int t = 0; t < n_steps; ++t) {
#pragma omp parallel for schedule(static)
    for (int w = 0; w < W; ++w) {
      rng_t r;
      uint64_t sm = seed ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(w + 1)) ^ ((uint64_t)t << 32);
      for (int k = 0; k < 4; ++k) r.s[k] = splitmix(&sm);
      r.has = 0;
      double* x = X + (size_t)w * 3 * ne;
      double prop[3 * MAXE];
      for (int k = 0; k < 3 * ne; ++k) prop[k] = x[k] + step * normal(&r);
      const double ratio = valid_move(d, prop) ? 1.0 : 0.0;
      const double lo = log_psi(&S, x), ln = log_psi(&S, prop);
      if (u01(&r) < exp(2.0 * (ln - lo)) * ratio) {
        memcpy(x, prop, sizeof(double) * 3 * ne);
        accw[w] += 1;
      }
      local_energy(&S, x, ep + 4 * (size_t)w);
    }
    double s[4] = {0, 0, 0, 0};
    for (int w = 0; w < W; ++w) for (int k = 0; k < 4; ++k) s[k] += ep[4 * (size_t)w + k];
    for (int k = 0; k < 4; ++k) series[4 * t + k] = s[k] / W;
  }
  double a = 0.0;
  for (int w = 0; w < W; ++w) a += accw[w];
  *acc = a / ((double)W * (n_steps > 0 ? n_steps : 1));
  free(ep);
  free(accw);
  return 0;
}
