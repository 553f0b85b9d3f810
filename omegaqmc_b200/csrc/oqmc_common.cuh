// Shared device-side pieces of the GTO Slater-Jastrow kernels (sm_100a).
//
// The system tables (nuclei, exponent groups, contracted shells, Jastrow and
// cusp constants) live in one POD struct that every CTA copies into shared
// memory once; all threads then read them as broadcasts.  Walker data is
// laid out walker-minor ("structure of arrays") wherever consecutive threads
// handle consecutive walkers, so global accesses coalesce.
#pragma once
#ifdef __CUDACC_RTC__
// run-time compilation (NVRTC): no host headers
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
#ifndef INFINITY
#define INFINITY __longlong_as_double(0x7ff0000000000000ULL)
#endif
#else
#include <cstdint>
#include <cuda_runtime.h>
#endif

#define OQ_MAX_NUC 16
#define OQ_MAX_GROUP 96
#define OQ_MAX_SHELL 128
#define OQ_MAX_PRIM 256
#define OQ_MAX_NORM 512
#define OQ_MAX_BF 160
#define OQ_MAX_OCC 16
#define OQ_MAX_E 32
#define OQ_MAX_COL 4          // contraction columns sharing one exponent list
#define OQ_MAX_TERMS 96       // monomial terms of the f and g harmonics
#define OQ_MAX_BSC 32         // B-spline Jastrow coefficients (parameters + 4)
#define OQ_MAX_BST 4          // element types with a one-body B-spline

// Harmonic monomial tables for am = 3, 4 (am <= 2 are hand-written).
// term t of component c of am: coef * x^i y^j z^k, packed i | j<<4 | k<<8.
struct OqHarmTable {
  double coef[OQ_MAX_TERMS];
  int pow[OQ_MAX_TERMS];
  int first[2][10];        // [am-3][c] first term, [c+1] end
};

// Exponent group = one basis entry of one atom: nprim exponents shared by
// ncol contracted shells (the columns of a general contraction).
struct OqSystem {
  int natm, nbf, nocc, n_e;
  int ngroup, nshell, has_j1, has_j2;
  int cusp, nprim_total, pad0, pad1;
  double e_nn;
  double nuc[OQ_MAX_NUC][3];
  double Z[OQ_MAX_NUC];
  double j1a[OQ_MAX_NUC], j1b[OQ_MAX_NUC];
  double j2[4];                    // like a, like b, unlike a, unlike b
  double rc[OQ_MAX_NUC], q0[OQ_MAX_NUC], cc[OQ_MAX_NUC][8];
  int g_iat[OQ_MAX_GROUP], g_off[OQ_MAX_GROUP], g_n[OQ_MAX_GROUP];
  int g_shell0[OQ_MAX_GROUP], g_ncol[OQ_MAX_GROUP], g_am[OQ_MAX_GROUP];
  int s_ao[OQ_MAX_SHELL], s_norm[OQ_MAX_SHELL], s_cusp[OQ_MAX_SHELL];
  int pad2;
  double alpha[OQ_MAX_PRIM];
  double norm[OQ_MAX_NORM];
  // cubic B-spline Jastrow terms (coefficients c[0..n+3], knots k/dinv,
  // zero beyond the cutoff): two-body like/unlike, one-body per element type
  int has_bs1, has_bs2, bs2_n_like, bs2_n_unlike;
  double bs2_rcut, bs2_dinv_like, bs2_dinv_unlike, bs_pad;
  double bs2_like[OQ_MAX_BSC], bs2_unlike[OQ_MAX_BSC];
  int bs1_type[OQ_MAX_NUC];          // element type of each atom, -1: none
  int bs1_n[OQ_MAX_BST];
  double bs1_rcut[OQ_MAX_BST], bs1_dinv[OQ_MAX_BST];
  double bs1_c[OQ_MAX_BST][OQ_MAX_BSC];
  // three-body electron-electron-nucleus polynomial Jastrow: gamma blocks
  // [type][like 0 / unlike 1][nI + 1][nI + 1][nE + 1] in device memory
  int has_j3, j3_nI, j3_nE, j3_pad;
  double j3_L;                       // half cutoff: u = 0 unless r_1I, r_2I < L
  const double* j3_gamma;
  int j3_type[OQ_MAX_NUC];           // element type of each atom, -1: none
  int j3_on[OQ_MAX_BST][2];          // block present
  // quintic radial splines in s = r^2 (tables in device memory)
  int has_spl, spl_npts, spl_pad0, spl_pad1;
  double spl_smin, spl_pad2;
  const double* spl_knots;           // [table][npts]
  const double* spl_coef;            // [table][npts - 1][6]
  int s_spl[OQ_MAX_SHELL];           // table of each shell, -1: analytic radial
  OqHarmTable harm;
};

// Status codes shared by host and device.
enum OqStatus {
  OQ_OK = 0,
  OQ_ERR_ARG = -1,
  OQ_ERR_CUDA = -2,
  OQ_ERR_NAN = -3,
  OQ_ERR_SINGULAR = -4,
  OQ_ERR_TIMEOUT = -5,
  OQ_ERR_UNSUPPORTED = -6,
  OQ_ERR_NOMEM = -7,
};

// Device flag bits written by kernels (OR-ed into a per-launch word).
#define OQ_FLAG_NAN 1u
#define OQ_FLAG_SINGULAR 2u
#define OQ_FLAG_TIMEOUT 4u


// ---------------------------------------------------------------------------
// Copy the system struct into shared memory (all threads cooperate).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void oq_load_system(OqSystem* dst, const OqSystem* src) {
  const int n = sizeof(OqSystem) / 16;
  const int4* s = reinterpret_cast<const int4*>(src);
  int4* d = reinterpret_cast<int4*>(dst);
  for (int i = threadIdx.x; i < n; i += blockDim.x) d[i] = s[i];
}

// ---------------------------------------------------------------------------
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).
// ---------------------------------------------------------------------------
struct OqU4 { uint32_t x, y, z, w; };

__device__ __forceinline__ OqU4 oq_philox(OqU4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    OqU4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform in (0, 1] from 32 random bits
__device__ __forceinline__ double oq_u01(uint32_t v) {
  return ((double)v + 1.0) * 2.3283064365386963e-10;
}

// Three standard normals and the 32 bits of the acceptance uniform for a
// single-electron proposal from one Philox4x32-10 block, counter = (walker,
// step, electron, 0), key = seed.  Box-Muller in FP32 on the top 23 bits of
// the four words (the deviates only set proposal widths, 23-bit resolution
// is ample and the FP32 transcendental units are cheap; square roots by
// sqrt.approx); the uniform's bits are the four low bytes, disjoint from
// those, so all deviates are independent.
__device__ __forceinline__ void oq_move_normals(uint64_t seed, uint32_t walker, uint32_t step,
                                                uint32_t elec, float nf[3], uint32_t& ubits) {
  const OqU4 c0 = {walker, step, elec, 0u};
  const OqU4 r0 = oq_philox(c0, (uint32_t)seed, (uint32_t)(seed >> 32));
  // uniforms from the top 23 bits of each word as the mantissa of a float
  // in [1, 2) (no conversion instruction): m - 1 in [0, 1), 2 - m in (0, 1]
  auto m = [](uint32_t v) { return __uint_as_float(0x3f800000u | (v >> 9)); };
  float a, b;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(a) : "f"(-2.0f * __logf(2.0f - m(r0.x))));
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(b) : "f"(-2.0f * __logf(2.0f - m(r0.z))));
  float s, c;
  __sincosf(6.283185307179586f * (m(r0.y) - 1.0f), &s, &c);
  const float c2 = __cosf(6.283185307179586f * (m(r0.w) - 1.0f));   // third normal only
  nf[0] = a * c;
  nf[1] = a * s;
  nf[2] = b * c2;
  ubits = ((r0.x & 255u) << 24) | ((r0.y & 255u) << 16) | ((r0.z & 255u) << 8) | (r0.w & 255u);
}

// The acceptance uniform in [0, 1) in the working precision: all 32 bits in
// FP64; in FP32 the top 23 bits as the mantissa of a float in [1, 2) minus 1
// (no conversion instruction).  Both compare u < ratio on the same bits.
template <typename T> __device__ __forceinline__ T oq_uniform(uint32_t ubits);
template <> __device__ __forceinline__ double oq_uniform<double>(uint32_t ubits) {
  return (double)ubits * 2.3283064365386963e-10;
}
template <> __device__ __forceinline__ float oq_uniform<float>(uint32_t ubits) {
  return __uint_as_float(0x3f800000u | (ubits >> 9)) - 1.0f;
}

// The normals and the uniform as doubles (the FP64 proposals).
__device__ __forceinline__ void oq_move_randoms(uint64_t seed, uint32_t walker,
                                                uint32_t step, uint32_t elec,
                                                double n3[3], double& u) {
  float nf[3];
  uint32_t ubits;
  oq_move_normals(seed, walker, step, elec, nf, ubits);
  n3[0] = (double)nf[0];
  n3[1] = (double)nf[1];
  n3[2] = (double)nf[2];
  u = oq_uniform<double>(ubits);
}

// reciprocal / reciprocal square root in the working precision; in FP32 the
// hardware approximations themselves (rcp.approx / rsqrt.approx, relative
// error ~2^-23, subnormals flushed: the arguments here are distances and
// Jastrow denominators, far from the subnormal range)
__device__ __forceinline__ double oq_rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float oq_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double oq_rsqrt(double x) { return rsqrt(x); }
__device__ __forceinline__ float oq_rsqrt(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Padé u = a r / (1 + b r) from r and 1/r with one reciprocal:
// q = 1/(1+br), u = a r q, u'/r = a q^2 / r, u'' + 2u'/r = -2ab q^3 + 2u'/r
template <typename T>
__device__ __forceinline__ T oq_pade_q(T a, T b, T r) {
  return a * r * oq_rcp((T)1 + b * r);
}
// Change of a r / (1 + b r) from r_o to r_n.  FP32: the algebraically
// equal a (r_n - r_o) / ((1 + b r_n)(1 + b r_o)), one reciprocal instead of
// two (and no cancellation between two values); FP64: the difference of the
// two values.
template <typename T>
__device__ __forceinline__ T oq_pade_diff(T a, T b, T rn, T ro) {
  if (sizeof(T) == 8) return oq_pade_q(a, b, rn) - oq_pade_q(a, b, ro);
  return a * (rn - ro) * oq_rcp(((T)1 + b * rn) * ((T)1 + b * ro));
}
template <typename T>
__device__ __forceinline__ void oq_pade_vgl_q(T a, T b, T r, T rinv, T& up_r, T& lap) {
  const T q = oq_rcp((T)1 + b * r);
  const T aq2 = a * q * q;
  up_r = aq2 * rinv;
  lap = (T)-2 * b * aq2 * q + (T)2 * up_r;
}

// Uniform-knot cubic B-spline u(r) = sum_k w_k(t) c[i+k], x = r dinv,
// i = clamp(floor(x), 0, n), t = x - i, with the cubic B-spline weights
// (1-t)^3/6, (3t^3-6t^2+4)/6, (-3t^3+3t^2+3t+1)/6, t^3/6; zero for r >= rcut
// (_bspline_eval / _bspline_eval_vgl and the callers' cutoff mask,
// OmegaQMC/psi/gto.py:36-119, 1684-1931).
template <typename T> __device__ __forceinline__ T oq_floor(T x);
template <> __device__ __forceinline__ double oq_floor<double>(double x) { return floor(x); }
template <> __device__ __forceinline__ float oq_floor<float>(float x) { return floorf(x); }

template <typename T>
__device__ __forceinline__ int oq_bs_index(T x, int n, T& t) {
  int i = (int)oq_floor<T>(x);
  i = i < 0 ? 0 : (i > n ? n : i);
  t = x - (T)i;
  return i;
}

template <typename T>
__device__ __forceinline__ T oq_bs_val(const double* c, int n, T dinv, T rcut, T r) {
  if (!(r < rcut)) return (T)0;
  T t;
  const int i = oq_bs_index<T>(r * dinv, n, t);
  const T t2 = t * t, t3 = t2 * t;
  return (T)(1.0 / 6.0) *
         ((-t3 + (T)3 * t2 - (T)3 * t + (T)1) * (T)c[i] +
          ((T)3 * t3 - (T)6 * t2 + (T)4) * (T)c[i + 1] +
          ((T)-3 * t3 + (T)3 * t2 + (T)3 * t + (T)1) * (T)c[i + 2] + t3 * (T)c[i + 3]);
}

// u'/r and u'' + 2u'/r of the B-spline (the Jastrow gradient factor and
// Laplacian of one pair), both zero beyond the cutoff.
template <typename T>
__device__ __forceinline__ void oq_bs_vgl(const double* c, int n, T dinv, T rcut, T r, T rinv,
                                          T& up_r, T& lap) {
  if (!(r < rcut)) {
    up_r = (T)0;
    lap = (T)0;
    return;
  }
  T t;
  const int i = oq_bs_index<T>(r * dinv, n, t);
  const T t2 = t * t;
  const T c0 = (T)c[i], c1 = (T)c[i + 1], c2 = (T)c[i + 2], c3 = (T)c[i + 3];
  const T d1 = (T)(1.0 / 6.0) * dinv *
               ((-(T)3 * t2 + (T)6 * t - (T)3) * c0 + ((T)9 * t2 - (T)12 * t) * c1 +
                (-(T)9 * t2 + (T)6 * t + (T)3) * c2 + (T)3 * t2 * c3);
  const T d2 = (T)(1.0 / 6.0) * dinv * dinv *
               ((-(T)6 * t + (T)6) * c0 + ((T)18 * t - (T)12) * c1 +
                (-(T)18 * t + (T)6) * c2 + (T)6 * t * c3);
  up_r = d1 * rinv;
  lap = d2 + (T)2 * up_r;
}

// ---------------------------------------------------------------------------
// Quintic radial spline of table id at s = r^2 (_locate_and_horner,
// psi/gto.py:200-217): g(s), g'(s), g''(s); zero from the last knot on.  The
// segment is the one searchsorted(knots, s, 'right') - 1 picks: a first guess
// from the log grid, then corrected against the knots.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void oq_spline_gdd(const OqSystem& S, int id, double s, double& g,
                                              double& gp, double& gpp) {
  const int n = S.spl_npts;
  const double* kn = S.spl_knots + (size_t)id * n;
  const double send = kn[n - 1];
  if (!(s < send)) {
    g = gp = gpp = 0.0;
    return;
  }
  int j = 0;
  if (s >= kn[1]) {
    const double f = log(s / S.spl_smin) / log(send / S.spl_smin);
    j = 1 + (int)floor(f * (double)(n - 2));
    j = j < 1 ? 1 : (j > n - 2 ? n - 2 : j);
    while (j < n - 2 && kn[j + 1] <= s) ++j;
    while (j > 0 && kn[j] > s) --j;
  }
  const double* c = S.spl_coef + ((size_t)id * (n - 1) + j) * 6;
  const double d = s - kn[j];
  g = ((((c[0] * d + c[1]) * d + c[2]) * d + c[3]) * d + c[4]) * d + c[5];
  gp = (((5.0 * c[0] * d + 4.0 * c[1]) * d + 3.0 * c[2]) * d + 2.0 * c[3]) * d + c[4];
  gpp = ((20.0 * c[0] * d + 12.0 * c[1]) * d + 6.0 * c[2]) * d + 2.0 * c[3];
}

// ---------------------------------------------------------------------------
// Three-body electron-electron-nucleus Jastrow (J3_eeI, psi/gto.py:474-604,
// 1933-2196; QMCPACK PolynomialFunctor3D).  For electrons 1, 2 and nucleus I
// with r_1I, r_2I < L = r_cut / 2,
//   u = (r_1I - L)^3 (r_2I - L)^3 sum_lmn g[l][m][n] r_1I^l r_2I^m r_12^n,
// and J3 = -(sum over nuclei and electron pairs of u).  g is the block of
// the nucleus's element and the pair's spins, symmetric in (l, m), so u is
// symmetric in the two electrons.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T oq_j3_u(const double* __restrict__ g, int nI, int nE, T L, T r12,
                                     T r1, T r2) {
  T P = (T)0;
  for (int l = nI; l >= 0; --l) {
    T a = (T)0;
    for (int m = nI; m >= 0; --m) {
      const double* gp = g + (l * (nI + 1) + m) * (nE + 1);
      T q = (T)0;
      for (int n = nE; n >= 0; --n) q = q * r12 + (T)gp[n];
      a = a * r2 + q;
    }
    P = P * r1 + a;
  }
  const T e = (r1 - L) * (r2 - L);
  return P * e * e * e;
}

// Partials of u with electron 1 as the moving particle (_eval_eeI_poly_vgl,
// gto.py:508-604): u1 = du/dr_1I, ue = du/dr_12, u11, uee and the mixed u1e.
// Horner in r_12, r_2I, r_1I carrying first and second derivatives.
template <typename T>
__device__ __forceinline__ void oq_j3_partials(const double* __restrict__ g, int nI, int nE, T L,
                                               T r12, T r1, T r2, T& u1, T& ue, T& u11, T& uee,
                                               T& u1e) {
  T P = (T)0, P1 = (T)0, P11 = (T)0, Q = (T)0, Q1 = (T)0, R = (T)0;
  for (int l = nI; l >= 0; --l) {
    T a = (T)0, b = (T)0, c = (T)0;
    for (int m = nI; m >= 0; --m) {
      const double* gp = g + (l * (nI + 1) + m) * (nE + 1);
      T q = (T)0, qd = (T)0, qdd = (T)0;
      for (int n = nE; n >= 0; --n) {
        qdd = qdd * r12 + (T)2 * qd;
        qd = qd * r12 + q;
        q = q * r12 + (T)gp[n];
      }
      a = a * r2 + q;
      b = b * r2 + qd;
      c = c * r2 + qdd;
    }
    P11 = P11 * r1 + (T)2 * P1;
    P1 = P1 * r1 + P;
    P = P * r1 + a;
    Q1 = Q1 * r1 + Q;
    Q = Q * r1 + b;
    R = R * r1 + c;
  }
  const T s1 = r1 - L, s2 = r2 - L, s1s = s1 * s1, s2c = s2 * s2 * s2;
  const T E = s1s * s1 * s2c, E1 = (T)3 * s1s * s2c, E11 = (T)6 * s1 * s2c;
  u1 = P1 * E + P * E1;
  ue = Q * E;
  u11 = P11 * E + (T)2 * P1 * E1 + P * E11;
  uee = R * E;
  u1e = Q1 * E + Q * E1;
}

// Sum of u over the triplets of electron e at (x, y, z) with the electrons
// j >= j0, j != e, whose coordinate c is pos[(3 j + c) * ps].
template <typename T>
__device__ __forceinline__ T oq_j3_electron(const OqSystem& S, const double* pos, size_t ps,
                                            int ne, int e, int j0, double x, double y, double z) {
  const int nI = S.j3_nI, nE = S.j3_nE, bsz = (nI + 1) * (nI + 1) * (nE + 1);
  const T L = (T)S.j3_L;
  T acc = (T)0;
  for (int I = 0; I < S.natm; ++I) {
    const int ty = S.j3_type[I];
    if (ty < 0) continue;
    const double ax = x - S.nuc[I][0], ay = y - S.nuc[I][1], az = z - S.nuc[I][2];
    const T r1 = sqrt((T)(ax * ax + ay * ay + az * az));
    if (!(r1 < L)) continue;
    for (int j = j0; j < ne; ++j) {
      if (j == e) continue;
      const int blk = (e ^ j) & 1;
      if (!S.j3_on[ty][blk]) continue;
      const double xj = pos[(size_t)(3 * j) * ps], yj = pos[(size_t)(3 * j + 1) * ps],
                   zj = pos[(size_t)(3 * j + 2) * ps];
      const double bx = xj - S.nuc[I][0], by = yj - S.nuc[I][1], bz = zj - S.nuc[I][2];
      const T r2 = sqrt((T)(bx * bx + by * by + bz * bz));
      if (!(r2 < L)) continue;
      const double dx = x - xj, dy = y - yj, dz = z - zj;
      const T r12 = sqrt((T)(dx * dx + dy * dy + dz * dz));
      acc += oq_j3_u<T>(S.j3_gamma + (size_t)(2 * ty + blk) * bsz, nI, nE, L, r12, r1, r2);
    }
  }
  return acc;
}

// Gradient and Laplacian of J3 with respect to electron e at (x, y, z),
// subtracted from (gx, gy, gz, lp) (J3 = -sum u; J3_eeI_vgl,
// gto.py:2042-2196).
template <typename T>
__device__ __forceinline__ void oq_j3_vgl_electron(const OqSystem& S, const double* pos, size_t ps,
                                                   int ne, int e, double x, double y, double z,
                                                   T& gx, T& gy, T& gz, T& lp) {
  const int nI = S.j3_nI, nE = S.j3_nE, bsz = (nI + 1) * (nI + 1) * (nE + 1);
  const T L = (T)S.j3_L;
  for (int I = 0; I < S.natm; ++I) {
    const int ty = S.j3_type[I];
    if (ty < 0) continue;
    const T ax = (T)(x - S.nuc[I][0]), ay = (T)(y - S.nuc[I][1]), az = (T)(z - S.nuc[I][2]);
    const T r1 = sqrt(ax * ax + ay * ay + az * az);
    if (!(r1 < L)) continue;
    const T i1 = (T)1 / r1;
    const T e1x = ax * i1, e1y = ay * i1, e1z = az * i1;
    for (int j = 0; j < ne; ++j) {
      if (j == e) continue;
      const int blk = (e ^ j) & 1;
      if (!S.j3_on[ty][blk]) continue;
      const double xj = pos[(size_t)(3 * j) * ps], yj = pos[(size_t)(3 * j + 1) * ps],
                   zj = pos[(size_t)(3 * j + 2) * ps];
      const T bx = (T)(xj - S.nuc[I][0]), by = (T)(yj - S.nuc[I][1]), bz = (T)(zj - S.nuc[I][2]);
      const T r2 = sqrt(bx * bx + by * by + bz * bz);
      if (!(r2 < L)) continue;
      const T dx = (T)(x - xj), dy = (T)(y - yj), dz = (T)(z - zj);
      const T r12 = sqrt(dx * dx + dy * dy + dz * dz);
      const T i12 = (T)1 / r12;
      const T ex = dx * i12, ey = dy * i12, ez = dz * i12;
      T u1, ue, u11, uee, u1e;
      oq_j3_partials<T>(S.j3_gamma + (size_t)(2 * ty + blk) * bsz, nI, nE, L, r12, r1, r2, u1, ue,
                        u11, uee, u1e);
      gx -= u1 * e1x + ue * ex;
      gy -= u1 * e1y + ue * ey;
      gz -= u1 * e1z + ue * ez;
      lp -= u11 + (T)2 * u1 * i1 + uee + (T)2 * ue * i12 +
            (T)2 * u1e * (e1x * ex + e1y * ey + e1z * ez);
    }
  }
}

// ---------------------------------------------------------------------------
// Real solid harmonics (value and gradient), order of _angular_cartesian.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void oq_harm_d(T x, T y, T z, T Y[5], T dY[5][3]) {
  const T cd1 = (T)1.7320508075688772;
  const T cd2 = (T)0.8660254037844386;
  Y[0] = cd1 * x * y;
  Y[1] = cd1 * y * z;
  Y[2] = (T)0.5 * ((T)2 * z * z - x * x - y * y);
  Y[3] = cd1 * x * z;
  Y[4] = cd2 * (x * x - y * y);
  dY[0][0] = cd1 * y; dY[0][1] = cd1 * x; dY[0][2] = (T)0;
  dY[1][0] = (T)0;    dY[1][1] = cd1 * z; dY[1][2] = cd1 * y;
  dY[2][0] = -x;      dY[2][1] = -y;      dY[2][2] = (T)2 * z;
  dY[3][0] = cd1 * z; dY[3][1] = (T)0;    dY[3][2] = cd1 * x;
  dY[4][0] = cd1 * x; dY[4][1] = -cd1 * y; dY[4][2] = (T)0;
}

template <typename T>
__device__ __forceinline__ T oq_ipow(T v, int n) {
  T r = (T)1;
  for (int i = 0; i < n; ++i) r *= v;
  return r;
}

// component c of am (3 or 4) from the monomial table
template <typename T>
__device__ __forceinline__ void oq_harm_table(const OqHarmTable& H, int am, int c, T x,
                                              T y, T z, T& Y, T dY[3]) {
  Y = (T)0; dY[0] = dY[1] = dY[2] = (T)0;
  const int t0 = H.first[am - 3][c], t1 = H.first[am - 3][c + 1];
  for (int t = t0; t < t1; ++t) {
    const T cf = (T)H.coef[t];
    const int p = H.pow[t];
    const int i = p & 15, j = (p >> 4) & 15, k = (p >> 8) & 15;
    const T xi = oq_ipow(x, i), yj = oq_ipow(y, j), zk = oq_ipow(z, k);
    Y += cf * xi * yj * zk;
    if (i) dY[0] += cf * (T)i * oq_ipow(x, i - 1) * yj * zk;
    if (j) dY[1] += cf * (T)j * xi * oq_ipow(y, j - 1) * zk;
    if (k) dY[2] += cf * (T)k * xi * yj * oq_ipow(z, k - 1);
  }
}

// ---------------------------------------------------------------------------
// Cusp-corrected s orbital (value only and VGL), FP64.
// f = c0 (1-b) R + b q0 e^{-Zr} (c1 + sum_{k=2..7} c_k s^k), s = r/rc,
// b = 1 - 10 s^3 + 15 s^4 - 6 s^5 inside rc, 0 outside.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double oq_cusp_val(const OqSystem& S, int ia, double r,
                                              double R) {
  const double rc = S.rc[ia];
  const double* c = S.cc[ia];
  if (!(r < rc)) return c[0] * R;
  const double s = r / rc;
  const double s2 = s * s, s3 = s2 * s;
  const double b = 1.0 - 10.0 * s3 + 15.0 * s3 * s - 6.0 * s3 * s2;
  const double sl = S.q0[ia] * exp(-S.Z[ia] * r);
  double poly = c[7];
  for (int k = 6; k >= 2; --k) poly = poly * s + c[k];
  poly = poly * s2 + c[1];
  return c[0] * (1.0 - b) * R + b * sl * poly;
}

// (f, f'/r, f'' + 2 f'/r) given (R, R'/r, R'' + 2R'/r) of the plain s shell.
__device__ __forceinline__ void oq_cusp_vgl(const OqSystem& S, int ia, double r,
                                            double& R, double& Rp, double& Rl) {
  const double rc = S.rc[ia];
  const double* c = S.cc[ia];
  const double c0 = c[0];
  if (!(r < rc)) {
    R *= c0; Rp *= c0; Rl *= c0;
    return;
  }
  const double Z = S.Z[ia];
  const double s = r / rc, oms = 1.0 - s;
  const double s2 = s * s, s3 = s2 * s;
  const double b = 1.0 - 10.0 * s3 + 15.0 * s3 * s - 6.0 * s3 * s2;
  const double bp = -(30.0 / rc) * s2 * oms * oms;
  const double bp_r = -(30.0 / (rc * rc * rc)) * r * oms * oms;
  const double bpp = -(60.0 / (rc * rc)) * s * oms * (1.0 - 2.0 * s);
  const double BL = bpp + 2.0 * bp_r;
  const double Av = c0 * (1.0 - b) * R;
  const double Ag = c0 * (-bp_r * R + (1.0 - b) * Rp);
  const double Al = c0 * (-BL * R + (1.0 - b) * Rl - 2.0 * r * bp * Rp);
  const double Sl = S.q0[ia] * exp(-Z * r);
  // P = c1 + sum c_k s^k, P' and P'' in r
  double P = c[7], P1 = 7.0 * c[7], P2 = 42.0 * c[7];
  for (int k = 6; k >= 2; --k) {
    P = P * s + c[k];
    P1 = P1 * s + k * c[k];
    P2 = P2 * s + k * (k - 1) * c[k];
  }
  P = P * s2 + c[1];
  P1 = P1 * s / rc;
  P2 = P2 / (rc * rc);
  const double Q = b * Sl * P;
  const double Qp = bp * Sl * P - Z * b * Sl * P + b * Sl * P1;
  const double Qpp = bpp * Sl * P + Z * Z * b * Sl * P + b * Sl * P2 +
                     2.0 * (-Z * bp * Sl * P + bp * Sl * P1 - Z * b * Sl * P1);
  const double Qg = Qp / r;
  R = Av + Q;
  Rp = Ag + Qg;
  Rl = Al + Qpp + 2.0 * Qg;
}

// Padé u(r) = a r / (1 + b r) and (u'/r, u'' + 2u'/r)
template <typename T>
__device__ __forceinline__ T oq_pade(T a, T b, T r) { return a * r / ((T)1 + b * r); }

template <typename T>
__device__ __forceinline__ void oq_pade_vgl(T a, T b, T r, T& up_r, T& lap) {
  const T den = (T)1 + b * r;
  const T up = a / (den * den);
  const T upp = (T)-2 * a * b / (den * den * den);
  up_r = up / r;
  lap = upp + (T)2 * up / r;
}
