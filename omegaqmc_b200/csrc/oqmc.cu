// liboqmc_b200: C ABI over the sm_100a kernels of the GTO-VMC hot path.
// Host code: validation, the device system tables, launch configuration.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <map>
#include <vector>
#include <cuda_runtime.h>

#include "oqmc_launch.h"
#include "oqmc_rtc.h"
#include "oqmc_mlp_host.h"
#include "oqmc_mlp_sweep.cuh"
#include "../../include/oqmc_b200.h"

#include "oqmc_ctx.h"

static thread_local char g_create_err[512] = "";

static int set_err(oqmc_ctx* ctx, int code, const char* fmt, const char* extra = "") {
  char* dst = ctx ? ctx->err : g_create_err;
  snprintf(dst, 512, fmt, extra);
  return code;
}

#define OQ_CUDA(ctx, call)                                                    \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess) return set_err(ctx, OQ_ERR_CUDA, "CUDA error: %s", \
                                          cudaGetErrorString(_e));            \
  } while (0)

// ---------------------------------------------------------------------------
// f and g harmonics as monomial tables (am = 3, 4), the polynomials of
// _angular_cartesian (OmegaQMC/psi/gto.py:607-671).
// ---------------------------------------------------------------------------
static void build_harm_table(OqHarmTable& t) {
  memset(&t, 0, sizeof(t));
  struct Term { double c; int i, j, k; };
  const double cf1 = sqrt(2.5) * 0.5, cf2 = 3.0 * cf1, cf3 = sqrt(15.0),
               cf4 = sqrt(1.5) * 0.5, cf5 = sqrt(6.0), cf6 = 1.5, cf7 = cf3 * 0.5;
  const double cg1 = 2.9580398915498085, cg2 = 6.2749501990055672,
               cg3 = 2.0916500663351894, cg4 = 1.1180339887498949,
               cg5 = 6.7082039324993694, cg6 = 2.3717082451262845,
               cg7 = 3.1622776601683795, cg8 = 0.55901699437494745,
               cg9 = 3.3541019662496847, cg10 = 0.73950997288745213,
               cg11 = 4.4370598373247132;
  std::vector<std::vector<Term>> f = {
      {{cf2, 2, 1, 0}, {-cf1, 0, 3, 0}},
      {{cf3, 1, 1, 1}},
      {{cf5, 0, 1, 2}, {-cf4, 2, 1, 0}, {-cf4, 0, 3, 0}},
      {{1.0, 0, 0, 3}, {-cf6, 2, 0, 1}, {-cf6, 0, 2, 1}},
      {{cf5, 1, 0, 2}, {-cf4, 3, 0, 0}, {-cf4, 1, 2, 0}},
      {{cf7, 2, 0, 1}, {-cf7, 0, 2, 1}},
      {{-cf2, 1, 2, 0}, {cf1, 3, 0, 0}}};
  std::vector<std::vector<Term>> g = {
      {{cg1, 3, 1, 0}, {-cg1, 1, 3, 0}},
      {{cg2, 2, 1, 1}, {-cg3, 0, 3, 1}},
      {{-cg4, 3, 1, 0}, {-cg4, 1, 3, 0}, {cg5, 1, 1, 2}},
      {{-cg6, 2, 1, 1}, {-cg6, 0, 3, 1}, {cg7, 0, 1, 3}},
      {{0.375, 4, 0, 0}, {0.375, 0, 4, 0}, {0.75, 2, 2, 0}, {1.0, 0, 0, 4},
       {-3.0, 2, 0, 2}, {-3.0, 0, 2, 2}},
      {{-cg6, 3, 0, 1}, {-cg6, 1, 2, 1}, {cg7, 1, 0, 3}},
      {{-cg8, 4, 0, 0}, {cg8, 0, 4, 0}, {cg9, 2, 0, 2}, {-cg9, 0, 2, 2}},
      {{-cg2, 1, 2, 1}, {cg3, 3, 0, 1}},
      {{cg10, 4, 0, 0}, {cg10, 0, 4, 0}, {-cg11, 2, 2, 0}}};
  int n = 0;
  const std::vector<std::vector<Term>>* tabs[2] = {&f, &g};
  for (int a = 0; a < 2; ++a) {
    const auto& tab = *tabs[a];
    for (size_t c = 0; c < tab.size(); ++c) {
      t.first[a][c] = n;
      for (const Term& x : tab[c]) {
        t.coef[n] = x.c;
        t.pow[n] = x.i | (x.j << 4) | (x.k << 8);
        ++n;
      }
    }
    t.first[a][tab.size()] = n;
  }
}

static bool nocc_supported(int n) {
  switch (n) {
    case 1: case 2: case 3: case 4: case 5: case 6: case 7: case 8:
    case 10: case 12: case 14: case 16: return true;
    default: return false;
  }
}

// Switch over the instantiated determinant sizes; EXPR uses N.
#define OQ_CASE(N, EXPR) \
  case N: {              \
    EXPR(N);             \
  } break;
#define OQ_SWITCH(nocc, EXPR)                                                       \
  switch (nocc) {                                                                   \
    OQ_CASE(1, EXPR) OQ_CASE(2, EXPR) OQ_CASE(3, EXPR) OQ_CASE(4, EXPR)             \
    OQ_CASE(5, EXPR) OQ_CASE(6, EXPR) OQ_CASE(7, EXPR) OQ_CASE(8, EXPR)             \
    OQ_CASE(10, EXPR) OQ_CASE(12, EXPR) OQ_CASE(14, EXPR) OQ_CASE(16, EXPR)         \
    default: err = cudaErrorInvalidValue;                                           \
  }

static OqLaunch make_launch(const oqmc_ctx* ctx, void* stream, size_t smem) {
  OqLaunch L;
  L.sys = ctx->d_sys; L.split = ctx->d_split; L.C64 = ctx->d_C64; L.C32 = ctx->d_C32;
  L.flags = ctx->d_flags; L.stream = (cudaStream_t)stream; L.smem = smem;
  return L;
}

static void compute_split(oqmc_ctx* ctx) {
  OqSystem& S = ctx->hsys;
  for (int g = 0; g < OQ_MAX_GROUP; ++g) ctx->hsplit.r2[g] = 0.0;
  if (!(ctx->tight_alpha > 0.0)) return;
  for (int g = 0; g < S.ngroup; ++g) {
    double r2 = 0.0;
    for (int p = 0; p < S.g_n[g]; ++p) {
      const double a = S.alpha[S.g_off[g] + p];
      if (a > ctx->tight_alpha) r2 = fmax(r2, 25.0 / a);
    }
    ctx->hsplit.r2[g] = r2;
  }
}

// Record an error on a context (used by entry points in other files).

// Largest per-thread local memory (bytes) among the kernels that
// oqmc_refresh followed by oqmc_sweeps launch for this context and precision
// (the same dispatch as those two entry points).  Returns OQ_OK or an error.
int oq_ctx_sweep_local_bytes(oqmc_ctx* ctx, int precision, size_t* out) {
  const int mixed = precision == OQ_PREC_MIXED;
  size_t best = 0, v = 0;
  cudaError_t err = cudaSuccess;
  auto take = [&](int kind, int prop, int M) -> bool {
#define OQ_X(N) err = oq_local_bytes_##N(kind, mixed, prop, M, &v)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    if (err != cudaSuccess) return false;
    best = v > best ? v : best;
    return true;
  };
  auto take_rtc = [&](void* fn) -> bool {
    const int b = fn ? oq_rtc_local_bytes(fn) : -1;
    if (b < 0) return false;
    best = (size_t)b > best ? (size_t)b : best;
    return true;
  };
  bool ok = true;
  if (ctx->md) {
    ok = take(4, 0, ctx->md->M) && take(5, 0, ctx->md->M) && take(6, 0, ctx->md->M);
  } else {
    ok = take(0, 0, 0);
    if (ok) {
      if (ctx->move_kind == 1) ok = take(7, 0, 0);
      else if (ctx->mlp) ok = take_rtc(ctx->mlp_fn[ctx->mlp_groups == 4 ? 1 : 0]);
      else if (ctx->spec)
        ok = take_rtc(oq_spec_function(ctx->spec, (ctx->proposal == 1 ? 4 : 0) + mixed));
      else ok = take(1, ctx->proposal == 1 ? 1 : 0, 0);
    }
    if (ok) {
      if (mixed && ctx->use_tc) ok = take(3, 0, 0);
      else if (ctx->spec) ok = take_rtc(oq_spec_function(ctx->spec, 2 + mixed));
      else ok = take(2, 0, 0);
    }
  }
  if (!ok)
    return set_err(ctx, OQ_ERR_CUDA, "kernel attribute query failed: %s",
                   cudaGetErrorString(err != cudaSuccess ? err : cudaErrorInvalidValue));
  *out = best;
  return OQ_OK;
}

int oq_ctx_set_error(oqmc_ctx* ctx, int code, const char* msg) {
  return set_err(ctx, code, "%s", msg);
}

extern "C" {

const char* oqmc_version(void) { return "oqmc_b200 0.1.0 (sm_100a)"; }

const char* oqmc_last_error(const oqmc_ctx* ctx) { return ctx ? ctx->err : g_create_err; }

// Validate a descriptor and fill the device system tables (host side only).
static int fill_system(const oqmc_system_desc* d, OqSystem& S) {
  if (!d) return set_err(nullptr, OQ_ERR_ARG, "null argument%s");
  if (d->natm < 1 || d->natm > OQ_MAX_NUC)
    return set_err(nullptr, OQ_ERR_UNSUPPORTED, "natm out of range (1..16)%s");
  if (d->n_e != 2 * d->nocc)
    return set_err(nullptr, OQ_ERR_UNSUPPORTED, "only closed shells (n_e = 2 nocc)%s");
  if (!nocc_supported(d->nocc))
    return set_err(nullptr, OQ_ERR_UNSUPPORTED,
                   "nocc must be one of 1-8, 10, 12, 14, 16%s");
  if (d->nbf < d->nocc || d->nbf > OQ_MAX_BF)
    return set_err(nullptr, OQ_ERR_UNSUPPORTED, "nbf out of range%s");
  if (d->ngroup < 1 || d->ngroup > OQ_MAX_GROUP)
    return set_err(nullptr, OQ_ERR_UNSUPPORTED, "too many exponent groups%s");
  memset(&S, 0, sizeof(OqSystem));
  S.natm = d->natm; S.nbf = d->nbf; S.nocc = d->nocc; S.n_e = d->n_e;
  S.ngroup = d->ngroup; S.has_j1 = d->has_j1; S.has_j2 = d->has_j2; S.cusp = d->cusp;
  S.e_nn = d->e_nn;
  for (int i = 0; i < d->natm; ++i) {
    for (int c = 0; c < 3; ++c) S.nuc[i][c] = d->nuc[3 * i + c];
    S.Z[i] = d->Z[i];
    if (d->has_j1) { S.j1a[i] = d->j1[2 * i]; S.j1b[i] = d->j1[2 * i + 1]; }
    if (d->cusp) {
      S.rc[i] = d->cusp_rc[i]; S.q0[i] = d->cusp_q0[i];
      for (int k = 0; k < 8; ++k) S.cc[i][k] = d->cusp_coeff[8 * i + k];
    }
  }
  if (d->has_j2) for (int k = 0; k < 4; ++k) S.j2[k] = d->j2[k];
  int prim = 0, shell = 0, normo = 0, ao = 0;
  for (int g = 0; g < d->ngroup; ++g) {
    const int np = d->group_nprim[g], nc = d->group_ncol[g], am = d->group_am[g];
    const int ia = d->group_atom[g];
    if (np < 1 || nc < 1 || nc > OQ_MAX_COL || am < 0 || am > 4 || ia < 0 || ia >= d->natm ||
        prim + np > OQ_MAX_PRIM || shell + nc > OQ_MAX_SHELL || normo + np * nc > OQ_MAX_NORM)
      return set_err(nullptr, OQ_ERR_UNSUPPORTED, "basis group out of supported range%s");
    S.g_iat[g] = ia; S.g_off[g] = prim; S.g_n[g] = np; S.g_shell0[g] = shell;
    S.g_ncol[g] = nc; S.g_am[g] = am;
    for (int p = 0; p < np; ++p) S.alpha[prim + p] = d->alpha[prim + p];
    for (int k = 0; k < nc; ++k) {
      S.s_ao[shell + k] = ao;
      S.s_norm[shell + k] = normo;
      S.s_cusp[shell + k] = (d->cusp && am == 0) ? d->shell_cusp[shell + k] : 0;
      for (int p = 0; p < np; ++p) S.norm[normo + p] = d->norm[normo + p];
      normo += np;
      ao += 2 * am + 1;
    }
    prim += np;
    shell += nc;
  }
  S.nshell = shell;
  S.nprim_total = prim;
  if (ao != d->nbf) return set_err(nullptr, OQ_ERR_ARG, "group table does not add up to nbf AOs%s");
  if (d->has_bs2) {
    const int nl = d->bs2_ncoef_like, nu = d->bs2_ncoef_unlike;
    if (nl < 6 || nu < 6 || nl > OQ_MAX_BSC || nu > OQ_MAX_BSC || !(d->bs2_rcut > 0.0) ||
        !d->bs2_coef_like || !d->bs2_coef_unlike)
      return set_err(nullptr, OQ_ERR_ARG, "bad two-body B-spline table%s");
    S.has_bs2 = 1;
    S.bs2_n_like = nl - 4;
    S.bs2_n_unlike = nu - 4;
    S.bs2_rcut = d->bs2_rcut;
    S.bs2_dinv_like = (double)(nl - 3) / d->bs2_rcut;
    S.bs2_dinv_unlike = (double)(nu - 3) / d->bs2_rcut;
    for (int k = 0; k < nl; ++k) S.bs2_like[k] = d->bs2_coef_like[k];
    for (int k = 0; k < nu; ++k) S.bs2_unlike[k] = d->bs2_coef_unlike[k];
  }
  for (int i = 0; i < OQ_MAX_NUC; ++i) S.bs1_type[i] = -1;
  if (d->has_bs1) {
    if (d->bs1_ntype < 1 || d->bs1_ntype > OQ_MAX_BST || !d->bs1_type || !d->bs1_ncoef ||
        !d->bs1_rcut || !d->bs1_coef)
      return set_err(nullptr, OQ_ERR_ARG, "bad one-body B-spline table%s");
    S.has_bs1 = 1;
    int off = 0;
    for (int t = 0; t < d->bs1_ntype; ++t) {
      const int n = d->bs1_ncoef[t];
      if (n < 6 || n > OQ_MAX_BSC || !(d->bs1_rcut[t] > 0.0))
        return set_err(nullptr, OQ_ERR_ARG, "bad one-body B-spline table%s");
      S.bs1_n[t] = n - 4;
      S.bs1_rcut[t] = d->bs1_rcut[t];
      S.bs1_dinv[t] = (double)(n - 3) / d->bs1_rcut[t];
      for (int k = 0; k < n; ++k) S.bs1_c[t][k] = d->bs1_coef[off + k];
      off += n;
    }
    for (int i = 0; i < d->natm; ++i) {
      const int t = d->bs1_type[i];
      if (t < -1 || t >= d->bs1_ntype)
        return set_err(nullptr, OQ_ERR_ARG, "bad one-body B-spline atom type%s");
      S.bs1_type[i] = t;
    }
  }
  for (int i = 0; i < OQ_MAX_NUC; ++i) S.j3_type[i] = -1;
  if (d->has_j3) {
    if (d->j3_n_ei < 0 || d->j3_n_ei > 6 || d->j3_n_ee < 1 || d->j3_n_ee > 6 ||
        d->j3_ntype < 1 || d->j3_ntype > OQ_MAX_BST || !(d->j3_rcut > 0.0) || !d->j3_type ||
        !d->j3_on || !d->j3_gamma)
      return set_err(nullptr, OQ_ERR_ARG, "bad three-body Jastrow table%s");
    S.has_j3 = 1;
    S.j3_nI = d->j3_n_ei;
    S.j3_nE = d->j3_n_ee;
    S.j3_L = 0.5 * d->j3_rcut;
    S.j3_gamma = d->j3_gamma;     // host table; oqmc_create points it at a device copy
    for (int t = 0; t < d->j3_ntype; ++t)
      for (int b = 0; b < 2; ++b) S.j3_on[t][b] = d->j3_on[2 * t + b] ? 1 : 0;
    for (int i = 0; i < d->natm; ++i) {
      const int t = d->j3_type[i];
      if (t < -1 || t >= d->j3_ntype)
        return set_err(nullptr, OQ_ERR_ARG, "bad three-body Jastrow atom type%s");
      S.j3_type[i] = t;
    }
  }
  for (int i = 0; i < OQ_MAX_SHELL; ++i) S.s_spl[i] = -1;
  if (d->has_spl) {
    if (d->spl_npts < 3 || d->spl_ntab < 1 || !(d->spl_smin > 0.0) || !d->spl_shell ||
        !d->spl_knots || !d->spl_coef)
      return set_err(nullptr, OQ_ERR_ARG, "bad radial spline table%s");
    S.has_spl = 1;
    S.spl_npts = d->spl_npts;
    S.spl_smin = d->spl_smin;
    S.spl_knots = d->spl_knots;   // host tables; oqmc_create points them at device copies
    S.spl_coef = d->spl_coef;
    for (int i = 0; i < S.nshell; ++i) {
      const int t = d->spl_shell[i];
      if (t < -1 || t >= d->spl_ntab || (t >= 0 && S.s_cusp[i]))
        return set_err(nullptr, OQ_ERR_ARG, "bad radial spline shell table%s");
      S.s_spl[i] = t;
    }
  }
  build_harm_table(S.harm);
  return OQ_OK;
}

// Release a context's multi-determinant expansion.
static void md_free(oqmc_ctx* ctx) {
  OqMdHost* m = ctx->md;
  if (!m) return;
  cudaFree(m->d_C);
  cudaFree(m->d_coef);
  cudaFree(m->d_det);
  cudaFree(m->d_occ);
  cudaFree(m->d_scratch);
  delete m;
  ctx->md = nullptr;
}

// Doubles in the three-body Jastrow table of a descriptor.
static size_t j3_table_len(const oqmc_system_desc* d) {
  if (!d->has_j3) return 0;
  return (size_t)d->j3_ntype * 2 * (d->j3_n_ei + 1) * (d->j3_n_ei + 1) * (d->j3_n_ee + 1);
}

static_assert(sizeof(OqSystem) % 16 == 0, "OqSystem is copied in 16-byte chunks");

static void split_for(const OqSystem& S, double tight_alpha, OqSplit& sp) {
  for (int g = 0; g < OQ_MAX_GROUP; ++g) sp.r2[g] = 0.0;
  if (!(tight_alpha > 0.0)) return;
  for (int g = 0; g < S.ngroup; ++g) {
    double r2 = 0.0;
    for (int p = 0; p < S.g_n[g]; ++p) {
      const double a = S.alpha[S.g_off[g] + p];
      if (a > tight_alpha) r2 = fmax(r2, 25.0 / a);
    }
    sp.r2[g] = r2;
  }
}

}  // extern "C"

// Host-side system tables and split radii for a descriptor (used by the
// batch source generator); err receives the validation message.
int oq_fill_system_desc(const oqmc_system_desc* d, OqSystem* S, OqSplit* SP, int* nocc,
                        std::string* err) {
  const int rc = fill_system(d, *S);
  if (rc != OQ_OK) {
    *err = g_create_err;
    return rc;
  }
  split_for(*S, 50.0, *SP);
  *nocc = d->nocc;
  return OQ_OK;
}

extern "C" {

extern "C" int oqmc_spec_source_desc(const oqmc_system_desc* d, char* buf, size_t len) {
  OqSystem* S = new (std::nothrow) OqSystem();
  if (!S) return OQ_ERR_NOMEM;
  int rc = fill_system(d, *S);
  if (rc != OQ_OK) { delete S; return rc; }
  OqSplit sp;
  split_for(*S, 50.0, sp);
  const std::string src = oq_spec_source(*S, sp, d->C, d->nocc);
  delete S;
  if (buf && len) {
    const size_t n = src.size() < len - 1 ? src.size() : len - 1;
    memcpy(buf, src.data(), n);
    buf[n] = 0;
  }
  return (int)src.size();
}

extern "C" int oqmc_create(oqmc_ctx** out, const oqmc_system_desc* d) {
  if (!out || !d) return set_err(nullptr, OQ_ERR_ARG, "null argument%s");
  *out = nullptr;
  oqmc_ctx* ctx = new (std::nothrow) oqmc_ctx();
  if (!ctx) return set_err(nullptr, OQ_ERR_NOMEM, "out of host memory%s");
  {
    const int rc = fill_system(d, ctx->hsys);
    if (rc != OQ_OK) { delete ctx; return rc; }
  }
  OqSystem& S = ctx->hsys;
  ctx->nocc = d->nocc; ctx->n_e = d->n_e; ctx->nbf = d->nbf; ctx->natm = d->natm;
  ctx->tight_alpha = 50.0;
  ctx->proposal = 0;
  ctx->spec = nullptr;
  ctx->use_tc = 0;
  ctx->d_Btc = nullptr;
  ctx->h_C = new double[(size_t)d->nbf * d->nocc];
  memcpy(ctx->h_C, d->C, sizeof(double) * (size_t)d->nbf * d->nocc);
  ctx->scale_r0 = 1.0;
  ctx->scale_fmin = 0.05;
  compute_split(ctx);
  cudaGetDevice(&ctx->device);
  std::vector<float> c32((size_t)d->nbf * d->nocc);
  for (size_t i = 0; i < c32.size(); ++i) c32[i] = (float)d->C[i];
  cudaError_t e = cudaSuccess;
  e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_sys, sizeof(OqSystem)) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_split, sizeof(OqSplit)) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_C64, sizeof(double) * c32.size()) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_C32, sizeof(float) * c32.size()) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_flags, sizeof(unsigned)) : e;
  if (S.has_j3) {
    const size_t n3 = j3_table_len(d);
    e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_j3, sizeof(double) * n3) : e;
    e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_j3, d->j3_gamma, sizeof(double) * n3,
                                        cudaMemcpyHostToDevice) : e;
    S.j3_gamma = ctx->d_j3;
  }
  if (S.has_spl) {
    const size_t nk = (size_t)d->spl_ntab * d->spl_npts;
    const size_t nc = (size_t)d->spl_ntab * (d->spl_npts - 1) * 6;
    e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_spl_knots, sizeof(double) * nk) : e;
    e = (e == cudaSuccess) ? cudaMalloc(&ctx->d_spl_coef, sizeof(double) * nc) : e;
    e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_spl_knots, d->spl_knots, sizeof(double) * nk,
                                        cudaMemcpyHostToDevice) : e;
    e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_spl_coef, d->spl_coef, sizeof(double) * nc,
                                        cudaMemcpyHostToDevice) : e;
    S.spl_knots = ctx->d_spl_knots;
    S.spl_coef = ctx->d_spl_coef;
  }
  e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_sys, &S, sizeof(OqSystem), cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_split, &ctx->hsplit, sizeof(OqSplit), cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_C64, d->C, sizeof(double) * c32.size(), cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(ctx->d_C32, c32.data(), sizeof(float) * c32.size(), cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemset(ctx->d_flags, 0, sizeof(unsigned)) : e;
  if (e != cudaSuccess) {
    set_err(nullptr, OQ_ERR_CUDA, "CUDA error in create: %s", cudaGetErrorString(e));
    oqmc_destroy(ctx);
    return OQ_ERR_CUDA;
  }
  *out = ctx;
  return OQ_OK;
}

int oqmc_destroy(oqmc_ctx* ctx) {
  if (!ctx) return OQ_OK;
  oq_spec_destroy(ctx->spec);
  oq_rtc_unload(ctx->mlp_mod);
  cudaFree(ctx->d_Btc);
  delete[] ctx->h_C;
  cudaFree(ctx->d_sys);
  cudaFree(ctx->d_split);
  cudaFree(ctx->d_C64);
  cudaFree(ctx->d_C32);
  cudaFree(ctx->d_flags);
  cudaFree(ctx->d_j3);
  cudaFree(ctx->d_spl_knots);
  cudaFree(ctx->d_spl_coef);
  md_free(ctx);
  delete ctx;
  return OQ_OK;
}

int oqmc_set_multidet(oqmc_ctx* ctx, int ndet, int ncol, const double* C, const double* coef,
                      const int* occ_up, const int* occ_dn) {
  if (!ctx) return OQ_ERR_ARG;
  md_free(ctx);
  if (ndet == 0) return OQ_OK;
  const int N = ctx->nocc, nbf = ctx->nbf;
  if (ndet < 0 || ncol < N || !C || !coef || !occ_up || !occ_dn)
    return set_err(ctx, OQ_ERR_ARG, "bad multi-determinant arguments%s");
  // the orbital columns the expansion uses, in increasing order
  std::vector<int> slot(ncol, -1);
  for (int d = 0; d < ndet; ++d)
    for (int sp = 0; sp < 2; ++sp) {
      const int* o = (sp ? occ_dn : occ_up) + (size_t)d * N;
      for (int k = 0; k < N; ++k) {
        if (o[k] < 0 || o[k] >= ncol)
          return set_err(ctx, OQ_ERR_ARG, "orbital index out of range%s");
        for (int q = 0; q < k; ++q)
          if (o[q] == o[k])
            return set_err(ctx, OQ_ERR_ARG, "orbital repeated within a determinant%s");
        slot[o[k]] = 0;
      }
      if (!std::isfinite(coef[d]))
        return set_err(ctx, OQ_ERR_ARG, "non-finite CI coefficient%s");
    }
  int nused = 0;
  for (int c = 0; c < ncol; ++c)
    if (slot[c] == 0) slot[c] = nused++;
  if (nused > 16)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "multi-determinant expansions may use at most 16 orbitals%s");
  const int M = (nused <= 8 && N <= 8) ? 8 : 16;
  // unique spin determinants (orbital slots in the listed order)
  std::map<std::vector<int>, int> uniq[2];
  std::vector<std::vector<int>> lists[2];
  std::vector<int> det(2 * (size_t)ndet);
  for (int d = 0; d < ndet; ++d)
    for (int sp = 0; sp < 2; ++sp) {
      const int* o = (sp ? occ_dn : occ_up) + (size_t)d * N;
      std::vector<int> key(N);
      for (int k = 0; k < N; ++k) key[k] = slot[o[k]];
      auto it = uniq[sp].find(key);
      int idx;
      if (it == uniq[sp].end()) {
        idx = (int)lists[sp].size();
        uniq[sp][key] = idx;
        lists[sp].push_back(key);
      } else {
        idx = it->second;
      }
      det[2 * (size_t)d + sp] = idx;
    }
  const int nu0 = (int)lists[0].size(), nu1 = (int)lists[1].size();
  if (nu0 > OQ_MD_MAXU || nu1 > OQ_MD_MAXU)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "at most 64 distinct determinants per spin%s");
  for (int d = 0; d < ndet; ++d) det[2 * (size_t)d + 1] += nu0;
  std::vector<int> occ((size_t)(nu0 + nu1) * N);
  for (int u = 0; u < nu0; ++u)
    for (int k = 0; k < N; ++k) occ[(size_t)u * N + k] = lists[0][u][k];
  for (int u = 0; u < nu1; ++u)
    for (int k = 0; k < N; ++k) occ[(size_t)(nu0 + u) * N + k] = lists[1][u][k];
  std::vector<double> Cp((size_t)nbf * M, 0.0);
  for (int a = 0; a < nbf; ++a)
    for (int c = 0; c < ncol; ++c)
      if (slot[c] >= 0) Cp[(size_t)a * M + slot[c]] = C[(size_t)a * ncol + c];
  OqMdHost* m = new (std::nothrow) OqMdHost();
  if (!m) return set_err(ctx, OQ_ERR_NOMEM, "out of host memory%s");
  m->ndet = ndet; m->nu0 = nu0; m->nu1 = nu1; m->M = M;
  ctx->md = m;
  cudaError_t e = cudaSuccess;
  e = (e == cudaSuccess) ? cudaMalloc(&m->d_C, sizeof(double) * Cp.size()) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&m->d_coef, sizeof(double) * ndet) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&m->d_det, sizeof(int) * det.size()) : e;
  e = (e == cudaSuccess) ? cudaMalloc(&m->d_occ, sizeof(int) * occ.size()) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(m->d_C, Cp.data(), sizeof(double) * Cp.size(),
                                      cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(m->d_coef, coef, sizeof(double) * ndet,
                                      cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(m->d_det, det.data(), sizeof(int) * det.size(),
                                      cudaMemcpyHostToDevice) : e;
  e = (e == cudaSuccess) ? cudaMemcpy(m->d_occ, occ.data(), sizeof(int) * occ.size(),
                                      cudaMemcpyHostToDevice) : e;
  if (e != cudaSuccess) {
    md_free(ctx);
    return set_err(ctx, OQ_ERR_CUDA, "CUDA error in set_multidet: %s", cudaGetErrorString(e));
  }
  return OQ_OK;
}

int oqmc_multidet_info(const oqmc_ctx* ctx, int* ndet, int* nu_up, int* nu_dn, int* ncol) {
  if (!ctx) return OQ_ERR_ARG;
  const OqMdHost* m = ctx->md;
  if (ndet) *ndet = m ? m->ndet : 0;
  if (nu_up) *nu_up = m ? m->nu0 : 0;
  if (nu_dn) *nu_dn = m ? m->nu1 : 0;
  if (ncol) *ncol = m ? m->M : 0;
  return OQ_OK;
}

int oqmc_set_move_kind(oqmc_ctx* ctx, int kind) {
  if (!ctx) return OQ_ERR_ARG;
  if (kind != 0 && kind != 1) return set_err(ctx, OQ_ERR_ARG, "move kind must be 0 or 1%s");
  ctx->move_kind = kind;
  return OQ_OK;
}

int oqmc_set_proposal(oqmc_ctx* ctx, int kind, double r0, double fmin_frac) {
  if (!ctx) return OQ_ERR_ARG;
  if (kind < 0 || kind > 1 || (kind == 1 && (!(r0 > 0.0) || !(fmin_frac > 0.0) || fmin_frac > 1.0)))
    return set_err(ctx, OQ_ERR_ARG, "bad proposal parameters%s");
  ctx->proposal = kind;
  if (kind == 1) { ctx->scale_r0 = r0; ctx->scale_fmin = fmin_frac; }
  return OQ_OK;
}

int oqmc_set_mlp_proposal(oqmc_ctx* ctx, const oqmc_mlp* m) {
  if (!ctx) return OQ_ERR_ARG;
  if (!m) {
    ctx->mlp = nullptr;
    return OQ_OK;
  }
  if (!ctx->spec)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the learned proposal needs a specialised context (oqmc_specialize)%s");
  if (ctx->n_e > 32)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "the learned proposal handles up to 32 electrons%s");
  if (!ctx->mlp_fn[0]) {
    const std::string src = std::string("#include \"oqmc_mlp_sweep.cuh\"\n\n") +
                            oq_spec_basis_source(ctx->hsys, ctx->hsplit, ctx->h_C, ctx->nocc,
                                                 "OqSpecBasis");
    const std::string n = std::to_string(ctx->nocc);
    std::vector<void*> fns;
    std::string err;
    if (oq_rtc_build(src, {"k_moves_mlp<" + n + ", OqSpecBasis, 2>",
                           "k_moves_mlp<" + n + ", OqSpecBasis, 4>"},
                     &ctx->mlp_mod, &fns, &err) != 0)
      return set_err(ctx, OQ_ERR_UNSUPPORTED, "%s", err.c_str());
    ctx->mlp_fn[0] = fns[0];
    ctx->mlp_fn[1] = fns[1];
    if (ctx->mlp_groups != 4) ctx->mlp_groups = 2;
  }
  ctx->mlp = m;
  return OQ_OK;
}

int oqmc_set_mlp_groups(oqmc_ctx* ctx, int groups) {
  if (!ctx) return OQ_ERR_ARG;
  if (groups != 2 && groups != 4) return set_err(ctx, OQ_ERR_ARG, "groups must be 2 or 4%s");
  ctx->mlp_groups = groups;
  return OQ_OK;
}

// Jastrow-parameter derivatives, one thread per walker, FP64: d ln|psi|/dp
// and dE_L/dp for p = (J2 like a, like b, unlike a, unlike b, J1 a_I, b_I per
// atom), from the positions and the full gradient G of ln|psi| (oqmc_eval).
// For u = a r/(1+b r): du/da = r/den, du/db = -a r^2/den^2; u' = a/den^2,
// u'' = -2ab/den^3; E_L changes only through -1/2 sum_e (lap_e + |G_e|^2).
__device__ __forceinline__ void oq_pade_dp(double a, double b, double r, double du[2],
                                           double dup[2], double dL[2]) {
  const double den = 1.0 + b * r, id = 1.0 / den, id2 = id * id, id3 = id2 * id;
  du[0] = r * id;
  du[1] = -a * r * r * id2;
  dup[0] = id2;
  dup[1] = -2.0 * a * r * id3;
  const double dupp0 = -2.0 * b * id3, dupp1 = -2.0 * a * id3 + 6.0 * a * b * r * id3 * id;
  dL[0] = dupp0 + 2.0 * dup[0] / r;
  dL[1] = dupp1 + 2.0 * dup[1] / r;
}

// B-spline parameters: P_q is coefficient q+1 and coefficient 0 is
// P_1 - 2 dr cusp, so a term at distance r in knot interval i touches the
// parameters of coefficients i..i+3 (and P_1 through coefficient 0).
__device__ __forceinline__ void oq_bs_param_add(const OqSystem& S, const double* c, int n,
                                                double dinv, double rcut, double r, double gd,
                                                bool half, double* dl, double* de) {
  if (!(r < rcut)) return;
  double t;
  const int i = oq_bs_index<double>(r * dinv, n, t);
  const double t2 = t * t, t3 = t2 * t, s6 = 1.0 / 6.0;
  const double w[4] = {s6 * (-t3 + 3 * t2 - 3 * t + 1), s6 * (3 * t3 - 6 * t2 + 4),
                       s6 * (-3 * t3 + 3 * t2 + 3 * t + 1), s6 * t3};
  const double w1[4] = {s6 * dinv * (-3 * t2 + 6 * t - 3), s6 * dinv * (9 * t2 - 12 * t),
                        s6 * dinv * (-9 * t2 + 6 * t + 3), s6 * dinv * 3 * t2};
  const double w2[4] = {s6 * dinv * dinv * (-6 * t + 6), s6 * dinv * dinv * (18 * t - 12),
                        s6 * dinv * dinv * (-18 * t + 6), s6 * dinv * dinv * 6 * t};
  (void)c;
  for (int k = 0; k < 4; ++k) {
    const int idx = i + k;
    const int q = idx == 0 ? 1 : idx - 1;      // coefficient 0 depends on P_1
    if (q < 0 || q >= n) continue;
    const double dL = w2[k] + 2.0 * w1[k] / r;
    dl[q] += w[k];
    de[q] -= half ? 0.5 * (dL + 2.0 * w1[k] * gd) : dL + w1[k] * gd;
  }
}

__device__ void oq_param_derivs_bspline(const OqSystem& S, const double* x, const double* g,
                                        int n_e, double* dl, double* de) {
  int base = 4 + 2 * S.natm;
  if (S.has_bs2) {
    for (int i = 0; i < n_e; ++i)
      for (int j = i + 1; j < n_e; ++j) {
        const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1],
                     dz = x[3 * i + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double gd = ((g[3 * i] - g[3 * j]) * dx + (g[3 * i + 1] - g[3 * j + 1]) * dy +
                           (g[3 * i + 2] - g[3 * j + 2]) * dz) / r;
        const bool like = (i & 1) == (j & 1);
        if (like)
          oq_bs_param_add(S, S.bs2_like, S.bs2_n_like, S.bs2_dinv_like, S.bs2_rcut, r, gd, false,
                          dl + base, de + base);
        else
          oq_bs_param_add(S, S.bs2_unlike, S.bs2_n_unlike, S.bs2_dinv_unlike, S.bs2_rcut, r, gd,
                          false, dl + base + S.bs2_n_like, de + base + S.bs2_n_like);
      }
    base += S.bs2_n_like + S.bs2_n_unlike;
  }
  if (S.has_bs1) {
    int tbase[OQ_MAX_BST];
    for (int t = 0, b = base; t < OQ_MAX_BST; ++t) {
      tbase[t] = b;
      b += S.bs1_n[t];
    }
    for (int I = 0; I < S.natm; ++I) {
      const int ty = S.bs1_type[I];
      if (ty < 0) continue;
      for (int e = 0; e < n_e; ++e) {
        const double dx = x[3 * e] - S.nuc[I][0], dy = x[3 * e + 1] - S.nuc[I][1],
                     dz = x[3 * e + 2] - S.nuc[I][2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double gd = (g[3 * e] * dx + g[3 * e + 1] * dy + g[3 * e + 2] * dz) / r;
        oq_bs_param_add(S, S.bs1_c[ty], S.bs1_n[ty], S.bs1_dinv[ty], S.bs1_rcut[ty], r, gd, true,
                        dl + tbase[ty], de + tbase[ty]);
      }
    }
  }
}

// Unique gammas of one three-body block: (l, m, n) with l >= m, ordered
// m, then l, then n (the constraint map's order).
__host__ __device__ static inline int j3_unique(const OqSystem& S) {
  return (S.j3_nI + 1) * (S.j3_nI + 2) / 2 * (S.j3_nE + 1);
}

__device__ __forceinline__ double oq_ipow(double x, int k) {
  double v = 1.0;
  for (int i = 0; i < k; ++i) v *= x;
  return v;
}

// phi = r1^l r2^m r12^n (+ r1^m r2^l r12^n for l != m) and its partials
// with electron 1 moving: phi, d/dr1, d/dr12, d2/dr1^2, d2/dr12^2, d2/dr1dr12.
__device__ __forceinline__ void oq_j3_basis(int l, int m, int n, double r1, double r2, double r12,
                                            double f[6]) {
  for (int k = 0; k < 6; ++k) f[k] = 0.0;
  const double e0 = oq_ipow(r12, n), e1 = n >= 1 ? n * oq_ipow(r12, n - 1) : 0.0,
               e2 = n >= 2 ? n * (n - 1) * oq_ipow(r12, n - 2) : 0.0;
  for (int pass = 0; pass < (l != m ? 2 : 1); ++pass) {
    const int a = pass ? m : l, b = pass ? l : m;
    const double p0 = oq_ipow(r1, a), p1 = a >= 1 ? a * oq_ipow(r1, a - 1) : 0.0,
                 p2 = a >= 2 ? a * (a - 1) * oq_ipow(r1, a - 2) : 0.0, q = oq_ipow(r2, b);
    f[0] += p0 * q * e0;
    f[1] += p1 * q * e0;
    f[2] += p0 * q * e1;
    f[3] += p2 * q * e0;
    f[4] += p0 * q * e2;
    f[5] += p1 * q * e1;
  }
}

// d log|psi| / d gamma and d E_L / d gamma of the three-body Jastrow for the
// unique gammas of every present block (types in order, like then unlike),
// starting at raw slot `base`.  J3 = -sum u is linear in the gammas, so each
// gamma's derivative is the J3 value, gradient and Laplacian with that
// gamma's monomial in place of the polynomial.
__device__ void oq_param_derivs_j3(const OqSystem& S, const double* x, const double* g, int n_e,
                                   int base, double* dl, double* de) {
  const int NG = j3_unique(S);
  const double L = S.j3_L;
  int boff[OQ_MAX_BST][2];
  for (int t = 0, o = base; t < OQ_MAX_BST; ++t)
    for (int b = 0; b < 2; ++b) {
      boff[t][b] = S.j3_on[t][b] ? o : -1;
      if (S.j3_on[t][b]) o += NG;
    }
  for (int I = 0; I < S.natm; ++I) {
    const int ty = S.j3_type[I];
    if (ty < 0) continue;
    for (int i = 0; i < n_e; ++i)
      for (int j = i + 1; j < n_e; ++j) {
        const int blk = (i ^ j) & 1;
        const int off = boff[ty][blk];
        if (off < 0) continue;
        double di[3], dj[3], dij[3];
        for (int c = 0; c < 3; ++c) {
          di[c] = x[3 * i + c] - S.nuc[I][c];
          dj[c] = x[3 * j + c] - S.nuc[I][c];
          dij[c] = x[3 * i + c] - x[3 * j + c];
        }
        const double ri = sqrt(di[0] * di[0] + di[1] * di[1] + di[2] * di[2]);
        const double rj = sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
        if (!(ri < L) || !(rj < L)) continue;
        const double r12 = sqrt(dij[0] * dij[0] + dij[1] * dij[1] + dij[2] * dij[2]);
        // G_a . e_aI and G_a . e_ab for the two electrons, and the cosines
        double gi1 = 0, gie = 0, gj1 = 0, gje = 0, ci = 0, cj = 0;
        for (int c = 0; c < 3; ++c) {
          const double ei = di[c] / ri, ej = dj[c] / rj, e = dij[c] / r12;
          gi1 += g[3 * i + c] * ei;
          gie += g[3 * i + c] * e;
          gj1 += g[3 * j + c] * ej;
          gje -= g[3 * j + c] * e;
          ci += ei * e;
          cj -= ej * e;
        }
        // envelope (r_1I - L)^3 (r_2I - L)^3 in each electron's frame
        const double si = ri - L, sj = rj - L;
        const double E = si * si * si * sj * sj * sj;
        const double Ei1 = 3.0 * si * si * sj * sj * sj, Ei11 = 6.0 * si * sj * sj * sj;
        const double Ej1 = 3.0 * sj * sj * si * si * si, Ej11 = 6.0 * sj * si * si * si;
        int u = 0;
        for (int m = 0; m <= S.j3_nI; ++m)
          for (int l = m; l <= S.j3_nI; ++l)
            for (int n = 0; n <= S.j3_nE; ++n, ++u) {
              double fi[6], fj[6];
              oq_j3_basis(l, m, n, ri, rj, r12, fi);
              oq_j3_basis(l, m, n, rj, ri, r12, fj);
              // partials of f = phi * E with each electron as particle 1
              const double a1 = fi[1] * E + fi[0] * Ei1, ae = fi[2] * E;
              const double a11 = fi[3] * E + 2.0 * fi[1] * Ei1 + fi[0] * Ei11, aee = fi[4] * E;
              const double a1e = fi[5] * E + fi[2] * Ei1;
              const double b1 = fj[1] * E + fj[0] * Ej1, be = fj[2] * E;
              const double b11 = fj[3] * E + 2.0 * fj[1] * Ej1 + fj[0] * Ej11, bee = fj[4] * E;
              const double b1e = fj[5] * E + fj[2] * Ej1;
              // J3 = -sum f: d lap and G . dG of both electrons
              const double dlap_i = -(a11 + 2.0 * a1 / ri + aee + 2.0 * ae / r12 + 2.0 * a1e * ci);
              const double dlap_j = -(b11 + 2.0 * b1 / rj + bee + 2.0 * be / r12 + 2.0 * b1e * cj);
              const double gdg = -(a1 * gi1 + ae * gie) - (b1 * gj1 + be * gje);
              dl[off + u] -= fi[0] * E;
              de[off + u] -= 0.5 * (dlap_i + dlap_j + 2.0 * gdg);
            }
      }
  }
}

static int param_count_of(const OqSystem& S) {
  int n = 4 + 2 * S.natm;
  if (S.has_bs2) n += S.bs2_n_like + S.bs2_n_unlike;
  if (S.has_bs1)
    for (int t = 0; t < OQ_MAX_BST; ++t) n += S.bs1_n[t];
  if (S.has_j3)
    for (int t = 0; t < OQ_MAX_BST; ++t) n += j3_unique(S) * (S.j3_on[t][0] + S.j3_on[t][1]);
  return n;
}

__global__ void k_param_derivs(const OqSystem* __restrict__ gsys, const double* __restrict__ X,
                               const double* __restrict__ G, int W, int n_e,
                               double* __restrict__ dlog, double* __restrict__ del) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const OqSystem& S = *gsys;
  int n_raw = 4 + 2 * S.natm;
  if (S.has_bs2) n_raw += S.bs2_n_like + S.bs2_n_unlike;
  if (S.has_bs1)
    for (int t = 0; t < OQ_MAX_BST; ++t) n_raw += S.bs1_n[t];
  const int j3_base = n_raw;
  if (S.has_j3)
    for (int t = 0; t < OQ_MAX_BST; ++t) n_raw += j3_unique(S) * (S.j3_on[t][0] + S.j3_on[t][1]);
  const double* x = X + (size_t)w * n_e * 3;
  const double* g = G + (size_t)w * n_e * 3;
  double* dl = dlog + (size_t)w * n_raw;
  double* de = del + (size_t)w * n_raw;
  for (int k = 0; k < n_raw; ++k) { dl[k] = 0.0; de[k] = 0.0; }
  if (S.has_j2) {
    double al[4] = {0, 0, 0, 0}, ae[4] = {0, 0, 0, 0};
    for (int i = 0; i < n_e; ++i)
      for (int j = i + 1; j < n_e; ++j) {
        const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1],
                     dz = x[3 * i + 2] - x[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double gd = ((g[3 * i] - g[3 * j]) * dx + (g[3 * i + 1] - g[3 * j + 1]) * dy +
                           (g[3 * i + 2] - g[3 * j + 2]) * dz) / r;
        const int o = ((i & 1) == (j & 1)) ? 0 : 2;
        double du[2], dup[2], dL[2];
        oq_pade_dp(S.j2[o], S.j2[o + 1], r, du, dup, dL);
        for (int q = 0; q < 2; ++q) {
          al[o + q] += du[q];
          ae[o + q] -= dL[q] + dup[q] * gd;
        }
      }
    for (int k = 0; k < 4; ++k) { dl[k] = al[k]; de[k] = ae[k]; }
  }
  if (S.has_bs2 || S.has_bs1) oq_param_derivs_bspline(S, x, g, n_e, dl, de);
  if (S.has_j3) oq_param_derivs_j3(S, x, g, n_e, j3_base, dl, de);
  if (S.has_j1) {
    for (int I = 0; I < S.natm; ++I) {
      double sl0 = 0, sl1 = 0, se0 = 0, se1 = 0;
      for (int e = 0; e < n_e; ++e) {
        const double dx = x[3 * e] - S.nuc[I][0], dy = x[3 * e + 1] - S.nuc[I][1],
                     dz = x[3 * e + 2] - S.nuc[I][2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        const double gd = (g[3 * e] * dx + g[3 * e + 1] * dy + g[3 * e + 2] * dz) / r;
        double du[2], dup[2], dL[2];
        oq_pade_dp(S.j1a[I], S.j1b[I], r, du, dup, dL);
        sl0 += du[0]; sl1 += du[1];
        se0 -= 0.5 * (dL[0] + 2.0 * dup[0] * gd);
        se1 -= 0.5 * (dL[1] + 2.0 * dup[1] * gd);
      }
      dl[4 + 2 * I] = sl0; dl[5 + 2 * I] = sl1;
      de[4 + 2 * I] = se0; de[5 + 2 * I] = se1;
    }
  }
}

int oqmc_param_count(const oqmc_ctx* ctx) { return ctx ? param_count_of(ctx->hsys) : OQ_ERR_ARG; }

int oqmc_param_derivs(oqmc_ctx* ctx, const double* X, int W, const double* grad, double* dlogpsi,
                      double* dEL, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || (W > 0 && (!X || !grad || !dlogpsi || !dEL)))
    return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  k_param_derivs<<<(W + 127) / 128, 128, 0, (cudaStream_t)stream>>>(ctx->d_sys, X, grad, W,
                                                                     ctx->n_e, dlogpsi, dEL);
  OQ_CUDA(ctx, cudaGetLastError());
  return OQ_OK;
}

// TF32 rounding as cvt.rna (nearest, ties away from zero) and BF16 (nearest even)
static float host_tf32(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  memcpy(&f, &u, 4);
  return f;
}
static uint16_t host_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}

int oqmc_use_tensor_cores(oqmc_ctx* ctx, int enable) {
  if (ctx && enable && ctx->md)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the tensor-core local energy supports single determinants only%s");
  if (ctx && enable && ctx->hsys.has_spl)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the tensor-core local energy uses analytic radial functions only%s");
  if (ctx && enable && (ctx->hsys.has_bs1 || ctx->hsys.has_bs2 || ctx->hsys.has_j3))
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the tensor-core local energy supports Pade Jastrow terms only%s");
  if (!ctx) return OQ_ERR_ARG;
  if (!enable) { ctx->use_tc = 0; return OQ_OK; }
  if (ctx->nocc > 16 || 128 / ctx->n_e < 1)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "tensor-core local energy needs n_occ <= 16%s");
  const OqTcPlan P = oq_tc_plan(ctx->nbf);
  if (P.total > 227u * 1024u)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "basis too large for the tensor-core tile%s");
  if (!ctx->d_Btc) {
    std::vector<unsigned char> h(P.b_end - P.b_hi, 0);
    const int KC4 = (int)(P.K4 >> 2), KC2 = (int)(P.K2 >> 3);
    for (int n = 0; n < 16; ++n)
      for (int k = 0; k < ctx->nbf; ++k) {
        const float c = n < ctx->nocc ? (float)ctx->h_C[(size_t)k * ctx->nocc + n] : 0.0f;
        const float hi = host_tf32(c), lo = c - hi;
        const uint32_t o4 = (uint32_t)(((n >> 3) * KC4 + (k >> 2)) << 7) + ((n & 7) << 4) + ((k & 3) << 2);
        const uint32_t o2 = (uint32_t)(((n >> 3) * KC2 + (k >> 3)) << 7) + ((n & 7) << 4) + ((k & 7) << 1);
        memcpy(&h[(P.b_hi - P.b_hi) + o4], &hi, 4);
        memcpy(&h[(P.b_lo - P.b_hi) + o4], &lo, 4);
        const uint16_t bf = host_bf16(hi);
        memcpy(&h[(P.b_bf - P.b_hi) + o2], &bf, 2);
      }
    OQ_CUDA(ctx, cudaMalloc(&ctx->d_Btc, h.size()));
    OQ_CUDA(ctx, cudaMemcpy(ctx->d_Btc, h.data(), h.size(), cudaMemcpyHostToDevice));
  }
  ctx->use_tc = 1;
  return OQ_OK;
}

int oqmc_specialize(oqmc_ctx* ctx, int enable) {
  if (!ctx) return OQ_ERR_ARG;
  oq_spec_destroy(ctx->spec);
  ctx->spec = nullptr;
  if (!enable) return OQ_OK;
  if (ctx->hsys.has_spl)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "specialised kernels use analytic radial functions; the radial-spline "
                   "transform runs on the table-driven kernels%s");
  std::string err;
  OqSpecModule* m = nullptr;
  if (oq_spec_build(ctx->hsys, ctx->hsplit, ctx->h_C, ctx->nocc, &m, &err) != 0)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "specialisation unavailable: %s", err.c_str());
  ctx->spec = m;
  return OQ_OK;
}

int oqmc_spec_source(const oqmc_ctx* ctx, char* buf, size_t len) {
  if (!ctx) return OQ_ERR_ARG;
  const std::string s = oq_spec_source(ctx->hsys, ctx->hsplit, ctx->h_C, ctx->nocc);
  if (buf && len) {
    const size_t n = s.size() < len - 1 ? s.size() : len - 1;
    memcpy(buf, s.data(), n);
    buf[n] = 0;
  }
  return (int)s.size();
}

int oqmc_set_split(oqmc_ctx* ctx, double tight_alpha) {
  if (!ctx) return OQ_ERR_ARG;
  ctx->tight_alpha = tight_alpha;
  compute_split(ctx);
  if (ctx->spec) {   // the specialised kernels carry the split radii as literals
    const int rc = oqmc_specialize(ctx, 1);
    if (rc != OQ_OK) return rc;
  }
  if (ctx->mlp_mod) {   // so does the learned-proposal kernel: rebuild it
    oq_rtc_unload(ctx->mlp_mod);
    ctx->mlp_mod = ctx->mlp_fn[0] = ctx->mlp_fn[1] = nullptr;
    const oqmc_mlp* m = ctx->mlp;
    ctx->mlp = nullptr;
    if (m) {
      const int rc = oqmc_set_mlp_proposal(ctx, m);
      if (rc != OQ_OK) return rc;
    }
  }
  OQ_CUDA(ctx, cudaMemcpy(ctx->d_split, &ctx->hsplit, sizeof(OqSplit), cudaMemcpyHostToDevice));
  return OQ_OK;
}

static size_t smem_sys_c64(const oqmc_ctx* ctx) {
  return sizeof(OqSystem) + sizeof(double) * ctx->nbf * ctx->nocc;
}

static cudaError_t to_soa(const oqmc_ctx* ctx, const double* X, double* pos, int W,
                          cudaStream_t s);

static int md_eval(oqmc_ctx* ctx, const double* X, int W, double* logpsi, double* grad,
                   double* lap, double* eparts, void* stream);

int oqmc_eval(oqmc_ctx* ctx, const double* X, int W, double* logpsi, double* grad,
              double* lap, double* eparts, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || (W > 0 && (!X || !logpsi))) return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  if (ctx->md) return md_eval(ctx, X, W, logpsi, grad, lap, eparts, stream);
  const OqLaunch L = make_launch(ctx, stream, smem_sys_c64(ctx));
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_eval_##N(L, X, W, logpsi, grad, lap, eparts)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

int oqmc_log_psi(oqmc_ctx* ctx, const double* X, int W, double* logpsi, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || (W > 0 && (!X || !logpsi))) return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  if (ctx->md) return md_eval(ctx, X, W, logpsi, nullptr, nullptr, nullptr, stream);
  const OqLaunch L = make_launch(ctx, stream, smem_sys_c64(ctx));
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_logpsi_##N(L, X, W, logpsi)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

int oqmc_mo_values(oqmc_ctx* ctx, const double* X, int W, double* out, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || (W > 0 && (!X || !out))) return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  const OqLaunch L = make_launch(ctx, stream, smem_sys_c64(ctx));
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_movals_##N(L, X, W, out)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// Sampler state: [pos SoA 3*n_e*W doubles][ainv 2*nocc^2*W Real][logdet W doubles]
struct OqStatePtrs {
  double* pos;
  void* ainv;
  double* logdet;
};

static size_t real_size(int precision) {
  return precision == OQ_PREC_MIXED ? sizeof(float) : sizeof(double);
}

// Multi-determinant sampler state: [pos SoA][inverses (nu0+nu1) nocc^2 W]
// [log|det| (nu0+nu1) W][signs (nu0+nu1) W], all FP64.
static size_t md_state_bytes(const oqmc_ctx* ctx, int W) {
  const size_t nu = (size_t)ctx->md->nu0 + ctx->md->nu1;
  return align256((size_t)3 * ctx->n_e * W * sizeof(double)) +
         align256(nu * ctx->nocc * ctx->nocc * W * sizeof(double)) +
         2 * align256(nu * W * sizeof(double));
}

static OqMdState md_state(const oqmc_ctx* ctx, void* state, int W) {
  const size_t nu = (size_t)ctx->md->nu0 + ctx->md->nu1;
  OqMdState st;
  char* b = static_cast<char*>(state);
  st.pos = reinterpret_cast<double*>(b);
  b += align256((size_t)3 * ctx->n_e * W * sizeof(double));
  st.ainv = reinterpret_cast<double*>(b);
  b += align256(nu * ctx->nocc * ctx->nocc * W * sizeof(double));
  st.ldet = reinterpret_cast<double*>(b);
  b += align256(nu * W * sizeof(double));
  st.sgn = reinterpret_cast<double*>(b);
  st.W = W;
  st.pad = 0;
  return st;
}

static OqMdTables md_tables(const oqmc_ctx* ctx) {
  const OqMdHost* m = ctx->md;
  OqMdTables T;
  T.C = m->d_C; T.coef = m->d_coef; T.det = m->d_det; T.occ = m->d_occ;
  T.ndet = m->ndet; T.nu0 = m->nu0; T.nu1 = m->nu1; T.pad = 0;
  return T;
}

// Multi-determinant evaluation from scratch: FP64 refresh of a scratch state,
// then the local-energy kernel with the per-walker outputs.
static int md_eval(oqmc_ctx* ctx, const double* X, int W, double* logpsi, double* grad,
                   double* lap, double* eparts, void* stream) {
  OqMdHost* m = ctx->md;
  cudaStream_t s = (cudaStream_t)stream;
  if (m->scratch_w < W) {
    OQ_CUDA(ctx, cudaStreamSynchronize(s));
    cudaFree(m->d_scratch);
    m->d_scratch = nullptr;
    m->scratch_w = 0;
    OQ_CUDA(ctx, cudaMalloc(&m->d_scratch, md_state_bytes(ctx, W)));
    m->scratch_w = W;
  }
  const OqMdState st = md_state(ctx, m->d_scratch, W);
  const OqMdTables T = md_tables(ctx);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  const OqLaunch L = make_launch(ctx, stream, sizeof(OqSystem));
  OqElocArgs a;
  memset(&a, 0, sizeof(a));
  a.pos = st.pos; a.W = W; a.eparts = eparts; a.flags = ctx->d_flags;
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_md_refresh_##N(L, T, st, m->M)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
#define OQ_X(N) err = oq_md_local_##N(L, T, st, a, logpsi, grad, lap, m->M)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

size_t oqmc_state_bytes(const oqmc_ctx* ctx, int W, int precision) {
  if (!ctx || W < 0) return 0;
  if (ctx->md) return md_state_bytes(ctx, W);
  return align256((size_t)3 * ctx->n_e * W * sizeof(double)) +
         align256((size_t)2 * ctx->nocc * ctx->nocc * W * real_size(precision)) +
         align256((size_t)W * sizeof(double));
}

static OqStatePtrs state_ptrs(const oqmc_ctx* ctx, void* state, int W, int precision) {
  OqStatePtrs p;
  char* b = static_cast<char*>(state);
  p.pos = reinterpret_cast<double*>(b);
  b += align256((size_t)3 * ctx->n_e * W * sizeof(double));
  p.ainv = b;
  b += align256((size_t)2 * ctx->nocc * ctx->nocc * W * real_size(precision));
  p.logdet = reinterpret_cast<double*>(b);
  return p;
}

// (W, n3) row-major <-> [n3][W]
__global__ void k_aos_to_soa(const double* __restrict__ X, double* __restrict__ pos, int W,
                             int n3) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)W * n3) return;
  const int w = (int)(t / n3), k = (int)(t % n3);
  pos[(size_t)k * W + w] = X[t];
}

__global__ void k_soa_to_aos(const double* __restrict__ pos, double* __restrict__ X, int W,
                             int n3) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)W * n3) return;
  const int w = (int)(t / n3), k = (int)(t % n3);
  X[t] = pos[(size_t)k * W + w];
}

static cudaError_t to_soa(const oqmc_ctx* ctx, const double* X, double* pos, int W,
                          cudaStream_t s) {
  const long long n = (long long)W * 3 * ctx->n_e;
  k_aos_to_soa<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(X, pos, W, 3 * ctx->n_e);
  return cudaGetLastError();
}

static cudaError_t to_aos(const oqmc_ctx* ctx, const double* pos, double* X, int W,
                          cudaStream_t s) {
  const long long n = (long long)W * 3 * ctx->n_e;
  k_soa_to_aos<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(pos, X, W, 3 * ctx->n_e);
  return cudaGetLastError();
}

static bool valid_prec(int p) { return p == OQ_PREC_FP64 || p == OQ_PREC_MIXED; }

int oqmc_refresh(oqmc_ctx* ctx, const double* X, int W, void* state, int precision,
                 void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || (W > 0 && (!X || !state)) || !valid_prec(precision))
    return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (ctx->md) {
    if (precision != OQ_PREC_FP64)
      return set_err(ctx, OQ_ERR_UNSUPPORTED,
                     "multi-determinant trials are sampled in FP64 only%s");
    const OqMdState st = md_state(ctx, state, W);
    OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
    const OqLaunch L = make_launch(ctx, stream, sizeof(OqSystem));
    const OqMdTables T = md_tables(ctx);
    cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_md_refresh_##N(L, T, st, ctx->md->M)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    OQ_CUDA(ctx, err);
    return OQ_OK;
  }
  const OqStatePtrs st = state_ptrs(ctx, state, W, precision);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  const OqLaunch L = make_launch(ctx, stream, smem_sys_c64(ctx));
  const int mixed = precision == OQ_PREC_MIXED;
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_refresh_##N(L, st.pos, W, st.ainv, st.logdet, mixed)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

static size_t moves_smem(const oqmc_ctx* ctx, int wpb, int precision) {
  const size_t rs = real_size(precision);
  size_t b = sizeof(OqSystem) + sizeof(OqSplit);
  b += ((size_t)ctx->nbf * ctx->nocc * rs + 15) & ~(size_t)15;
  b += (size_t)3 * ctx->n_e * wpb * sizeof(double);
  b += (size_t)2 * ctx->nocc * ctx->nocc * wpb * rs;
  return b;
}

static size_t eloc_smem(const oqmc_ctx* ctx, int precision) {
  size_t b = sizeof(OqSystem) + sizeof(OqSplit);
  b += ((size_t)ctx->nbf * ctx->nocc * real_size(precision) + 15) & ~(size_t)15;
  b += (size_t)ctx->n_e * 4 * 32 * sizeof(double);
  return b;
}

static int pick_wpb(oqmc_ctx* ctx, int wpb, int precision, size_t* sm) {
  if (wpb == 0) wpb = 128;
  if (wpb != 32 && wpb != 64 && wpb != 128) return -1;
  *sm = moves_smem(ctx, wpb, precision);
  while (*sm > 227 * 1024 && wpb > 32) { wpb /= 2; *sm = moves_smem(ctx, wpb, precision); }
  if (*sm > 227 * 1024) return -2;
  return wpb;
}

static int launch_moves(oqmc_ctx* ctx, const OqMoveArgs& m, int wpb, size_t sm, int precision,
                        void* stream) {
  const int mixed = precision == OQ_PREC_MIXED;
  if (ctx->move_kind == 1 && m.mode == 0) {
    // all-electron steps: table-driven FP64 evaluation of the proposals
    const OqLaunch La = make_launch(ctx, stream, smem_sys_c64(ctx));
    cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_moves_alle_##N(La, m, mixed)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    OQ_CUDA(ctx, err);
    return OQ_OK;
  }
  const OqLaunch L = make_launch(ctx, stream, sm);
  if (ctx->mlp && m.mode == 0) {
    OqMoveArgs mm = m;
    const void* C = (const void*)ctx->d_C32;
    OqMlpWeights nw{ctx->mlp->wbf, ctx->mlp->theta};
    void* args[5] = {(void*)&L.sys, (void*)&L.split, (void*)&C, (void*)&mm, (void*)&nw};
    const int G = ctx->mlp_groups == 4 ? 4 : 2;
    if (oq_rtc_launch(ctx->mlp_fn[G == 4 ? 1 : 0], dim3((m.W + 128 * G - 1) / (128 * G)),
                      dim3(128 * G), oq_mlp_sweep_smem(G, ctx->n_e), L.stream, args) != 0)
      return set_err(ctx, OQ_ERR_CUDA, "learned-proposal move kernel launch failed%s");
    return OQ_OK;
  }
  if (ctx->spec && m.mode == 0) {
    OqMoveArgs mm = m;
    const void* C = mixed ? (const void*)ctx->d_C32 : (const void*)ctx->d_C64;
    void* args[4] = {(void*)&L.sys, (void*)&L.split, (void*)&C, (void*)&mm};
    const int which = (m.proposal == 1 ? 4 : 0) + (mixed ? 1 : 0);
    if (oq_spec_launch(ctx->spec, which, dim3((m.W + wpb - 1) / wpb), dim3(wpb), sm,
                       L.stream, args) != 0)
      return set_err(ctx, OQ_ERR_CUDA, "specialised move kernel launch failed%s");
    return OQ_OK;
  }
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_moves_##N(L, m, wpb, mixed)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

static int md_moves(oqmc_ctx* ctx, const OqMoveArgs& m, double* sgn, void* stream) {
  const OqLaunch L = make_launch(ctx, stream, sizeof(OqSystem));
  const OqMdTables T = md_tables(ctx);
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_md_moves_##N(L, T, m, sgn, ctx->md->M)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

// Sweeps with a multi-determinant Slater part (FP64; the same measurement
// layout as the single-determinant sweeps).
static int md_sweeps(oqmc_ctx* ctx, double* X, int W, void* state, int precision, int n_sweeps,
                     int measure_every, double step, uint64_t seed, uint64_t step_base,
                     double* sums, double* el_trace, double* eparts_last, void* stream) {
  if (precision != OQ_PREC_FP64)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "multi-determinant trials are sampled in FP64 only%s");
  if (ctx->mlp)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the learned proposal does not support multi-determinant trials%s");
  cudaStream_t s = (cudaStream_t)stream;
  const OqMdState st = md_state(ctx, state, W);
  const OqMdTables T = md_tables(ctx);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  OqMoveArgs m;
  memset(&m, 0, sizeof(m));
  m.pos = st.pos; m.ainv = st.ainv; m.logdet = st.ldet; m.W = W; m.mode = 0;
  m.step = step; m.seed = seed; m.flags = ctx->d_flags;
  m.proposal = ctx->proposal; m.scale_r0 = ctx->scale_r0; m.scale_fmin = ctx->scale_fmin;
  OqElocArgs el;
  memset(&el, 0, sizeof(el));
  el.pos = st.pos; el.W = W; el.flags = ctx->d_flags;
  const OqLaunch Le = make_launch(ctx, stream, sizeof(OqSystem));
  const int n_meas = n_sweeps / measure_every;
  int done = 0;
  for (int k = 0; k < n_meas; ++k) {
    m.n_steps = measure_every;
    m.step_base = step_base + done;
    m.acc_sum = sums + (size_t)k * OQ_NSUM + 5;
    int rc = md_moves(ctx, m, st.sgn, stream);
    if (rc != OQ_OK) return rc;
    done += measure_every;
    el.sums = sums + (size_t)k * OQ_NSUM;
    el.el_trace = el_trace ? el_trace + (size_t)k * W : nullptr;
    el.eparts = (k == n_meas - 1) ? eparts_last : nullptr;
    cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_md_local_##N(Le, T, st, el, nullptr, nullptr, nullptr, ctx->md->M)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    OQ_CUDA(ctx, err);
  }
  if (done < n_sweeps) {
    m.n_steps = n_sweeps - done;
    m.step_base = step_base + done;
    m.acc_sum = nullptr;
    int rc = md_moves(ctx, m, st.sgn, stream);
    if (rc != OQ_OK) return rc;
  }
  OQ_CUDA(ctx, to_aos(ctx, st.pos, X, W, s));
  return OQ_OK;
}

int oqmc_sweeps(oqmc_ctx* ctx, double* X, int W, void* state, int precision, int n_sweeps,
                int measure_every, double step, uint64_t seed, uint64_t step_base,
                double* sums, double* el_trace, double* eparts_last, int wpb,
                void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || n_sweeps < 0 || measure_every < 1 || !(step > 0.0) || !valid_prec(precision))
    return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0 || n_sweeps == 0) return OQ_OK;
  if (!X || !state || (n_sweeps >= measure_every && !sums))
    return set_err(ctx, OQ_ERR_ARG, "null buffer%s");
  if (ctx->mlp && precision != OQ_PREC_MIXED)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "the learned proposal runs in mixed precision only%s");
  if (ctx->mlp && ctx->move_kind == 1)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "the learned proposal moves one electron at a time%s");
  if (ctx->md && ctx->move_kind == 1)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "all-electron steps are built for single determinants%s");
  if (ctx->md)
    return md_sweeps(ctx, X, W, state, precision, n_sweeps, measure_every, step, seed, step_base,
                     sums, el_trace, eparts_last, stream);
  size_t sm;
  wpb = pick_wpb(ctx, wpb, precision, &sm);
  if (wpb == -1) return set_err(ctx, OQ_ERR_ARG, "walkers_per_block must be 32, 64 or 128%s");
  if (wpb < 0)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "system too large for the shared-memory move kernel%s");
  cudaStream_t s = (cudaStream_t)stream;
  const OqStatePtrs st = state_ptrs(ctx, state, W, precision);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  OqMoveArgs m;
  memset(&m, 0, sizeof(m));
  m.pos = st.pos; m.ainv = st.ainv; m.logdet = st.logdet; m.W = W; m.mode = 0;
  m.step = step; m.seed = seed; m.flags = ctx->d_flags;
  m.proposal = ctx->proposal; m.scale_r0 = ctx->scale_r0; m.scale_fmin = ctx->scale_fmin;
  OqElocArgs el;
  memset(&el, 0, sizeof(el));
  el.pos = st.pos; el.ainv = st.ainv; el.W = W; el.flags = ctx->d_flags;
  const OqLaunch Le = make_launch(ctx, stream, eloc_smem(ctx, precision));
  const int mixed = precision == OQ_PREC_MIXED;
  const int n_meas = n_sweeps / measure_every;
  int done = 0;
  for (int k = 0; k < n_meas; ++k) {
    m.n_steps = measure_every;
    m.step_base = step_base + done;
    m.acc_sum = sums + (size_t)k * OQ_NSUM + 5;
    int rc = launch_moves(ctx, m, wpb, sm, precision, stream);
    if (rc != OQ_OK) return rc;
    done += measure_every;
    el.sums = sums + (size_t)k * OQ_NSUM;
    el.el_trace = el_trace ? el_trace + (size_t)k * W : nullptr;
    el.eparts = (k == n_meas - 1) ? eparts_last : nullptr;
    if (mixed && ctx->use_tc) {
      cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_eloc_tc_##N(Le, el, ctx->d_Btc, ctx->nbf)
      OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
      OQ_CUDA(ctx, err);
      continue;
    }
    if (ctx->spec) {
      OqElocArgs ee = el;
      const void* C = mixed ? (const void*)ctx->d_C32 : (const void*)ctx->d_C64;
      void* args[4] = {(void*)&Le.sys, (void*)&Le.split, (void*)&C, (void*)&ee};
      if (oq_spec_launch(ctx->spec, mixed ? 3 : 2, dim3((W + 31) / 32), dim3(32, ctx->n_e),
                         Le.smem, Le.stream, args) != 0)
        return set_err(ctx, OQ_ERR_CUDA, "specialised local-energy kernel launch failed%s");
      continue;
    }
    cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_eloc_##N(Le, el, mixed)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    OQ_CUDA(ctx, err);
  }
  if (done < n_sweeps) {
    m.n_steps = n_sweeps - done;
    m.step_base = step_base + done;
    m.acc_sum = nullptr;
    int rc = launch_moves(ctx, m, wpb, sm, precision, stream);
    if (rc != OQ_OK) return rc;
  }
  OQ_CUDA(ctx, to_aos(ctx, st.pos, X, W, s));
  return OQ_OK;
}

// One step of the reference's step-size rule (_adapt_step_size,
// OmegaQMC/vmc_gto.py:121-126): with the acceptance ratio
// acc = (*accepted) * inv_moves of the sweep just made,
// log s <- log s + rate (acc - target).  Records the ratio in place of the
// count and the new width in step_trace (if set).  One thread.
__global__ void k_adapt_step(double* __restrict__ step, double* __restrict__ accepted,
                             double inv_moves, double rate, double target,
                             double* __restrict__ step_trace) {
  const double acc = *accepted * inv_moves;
  const double s = exp(log(*step) + rate * (acc - target));
  *step = s;
  *accepted = acc;
  if (step_trace) *step_trace = s;
}

int oqmc_equilibrate(oqmc_ctx* ctx, double* X, int W, void* state, int precision,
                     int n_steps, double* step, double target, double rate, uint64_t seed,
                     uint64_t step_base, int refresh_every, int since_refresh,
                     double* acc_trace, double* step_trace, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || n_steps < 0 || refresh_every < 1 || since_refresh < 0 || !valid_prec(precision))
    return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0 || n_steps == 0) return OQ_OK;
  if (!X || !state || !step || !acc_trace) return set_err(ctx, OQ_ERR_ARG, "null buffer%s");
  if (ctx->md || ctx->mlp || ctx->move_kind != 0)
    return set_err(ctx, OQ_ERR_UNSUPPORTED,
                   "device-side equilibration runs single-determinant, single-electron "
                   "Gaussian sweeps only%s");
  size_t sm;
  const int wpb = pick_wpb(ctx, 0, precision, &sm);
  if (wpb < 0)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "system too large for the shared-memory move kernel%s");
  cudaStream_t s = (cudaStream_t)stream;
  const OqStatePtrs st = state_ptrs(ctx, state, W, precision);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  OQ_CUDA(ctx, cudaMemsetAsync(acc_trace, 0, sizeof(double) * (size_t)n_steps, s));
  OqMoveArgs m;
  memset(&m, 0, sizeof(m));
  m.pos = st.pos; m.ainv = st.ainv; m.logdet = st.logdet; m.W = W; m.mode = 0;
  m.n_steps = 1; m.step = 0.0; m.step_dev = step; m.seed = seed; m.flags = ctx->d_flags;
  m.proposal = ctx->proposal; m.scale_r0 = ctx->scale_r0; m.scale_fmin = ctx->scale_fmin;
  const OqLaunch Lr = make_launch(ctx, stream, smem_sys_c64(ctx));
  const int mixed = precision == OQ_PREC_MIXED;
  const double inv_moves = 1.0 / ((double)W * ctx->n_e);
  int since = since_refresh;
  for (int t = 0; t < n_steps; ++t) {
    m.step_base = step_base + t;
    m.acc_sum = acc_trace + t;
    int rc = launch_moves(ctx, m, wpb, sm, precision, stream);
    if (rc != OQ_OK) return rc;
    k_adapt_step<<<1, 1, 0, s>>>(step, acc_trace + t, inv_moves, rate, target,
                                 step_trace ? step_trace + t : nullptr);
    OQ_CUDA(ctx, cudaGetLastError());
    if (++since >= refresh_every) {
      cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_refresh_##N(Lr, st.pos, W, st.ainv, st.logdet, mixed)
      OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
      OQ_CUDA(ctx, err);
      since = 0;
    }
  }
  OQ_CUDA(ctx, to_aos(ctx, st.pos, X, W, s));
  return OQ_OK;
}

int oqmc_state_eval(oqmc_ctx* ctx, const void* state, int W, int precision, double* logpsi,
                    double* grad, double* lap, double* eparts, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || !valid_prec(precision)) return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0) return OQ_OK;
  if (!state) return set_err(ctx, OQ_ERR_ARG, "null buffer%s");
  cudaStream_t s = (cudaStream_t)stream;
  if (ctx->md) {
    if (precision != OQ_PREC_FP64)
      return set_err(ctx, OQ_ERR_UNSUPPORTED,
                     "multi-determinant trials are sampled in FP64 only%s");
    // the expansion's local-energy kernel on the state's inverses
    const OqMdState st = md_state(ctx, const_cast<void*>(state), W);
    const OqMdTables T = md_tables(ctx);
    const OqLaunch L = make_launch(ctx, stream, sizeof(OqSystem));
    OqElocArgs a;
    memset(&a, 0, sizeof(a));
    a.pos = st.pos; a.W = W; a.eparts = eparts; a.flags = ctx->d_flags;
    cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_md_local_##N(L, T, st, a, logpsi, grad, lap, ctx->md->M)
    OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
    OQ_CUDA(ctx, err);
    return OQ_OK;
  }
  const OqStatePtrs st = state_ptrs(ctx, const_cast<void*>(state), W, precision);
  const int mixed = precision == OQ_PREC_MIXED;
  if (logpsi)
    OQ_CUDA(ctx, cudaMemcpyAsync(logpsi, st.logdet, sizeof(double) * (size_t)W,
                                 cudaMemcpyDeviceToDevice, s));
  OqElocArgs el;
  memset(&el, 0, sizeof(el));
  el.pos = st.pos; el.ainv = st.ainv; el.W = W; el.flags = ctx->d_flags;
  el.eparts = eparts; el.logpsi = logpsi; el.grad = grad; el.lap = lap;
  const OqLaunch Le = make_launch(ctx, stream, eloc_smem(ctx, precision));
  if (ctx->spec) {
    // the specialised kernel the sweeps use (the tensor-core form has no
    // per-electron outputs)
    const void* C = mixed ? (const void*)ctx->d_C32 : (const void*)ctx->d_C64;
    void* args[4] = {(void*)&Le.sys, (void*)&Le.split, (void*)&C, (void*)&el};
    if (oq_spec_launch(ctx->spec, mixed ? 3 : 2, dim3((W + 31) / 32), dim3(32, ctx->n_e),
                       Le.smem, Le.stream, args) != 0)
      return set_err(ctx, OQ_ERR_CUDA, "specialised local-energy kernel launch failed%s");
    return OQ_OK;
  }
  cudaError_t err = cudaSuccess;
#define OQ_X(N) err = oq_eloc_##N(Le, el, mixed)
  OQ_SWITCH(ctx->nocc, OQ_X)
#undef OQ_X
  OQ_CUDA(ctx, err);
  return OQ_OK;
}

int oqmc_basin(oqmc_ctx* ctx, double* X, int W, void* state, int precision, int n_steps,
               double sigma, uint64_t seed, uint64_t step_base, double* acc_sum,
               void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || n_steps < 0 || !(sigma > 0.0) || !valid_prec(precision))
    return set_err(ctx, OQ_ERR_ARG, "bad arguments%s");
  if (W == 0 || n_steps == 0) return OQ_OK;
  if (!X || !state) return set_err(ctx, OQ_ERR_ARG, "null buffer%s");
  if (ctx->md) {
    if (precision != OQ_PREC_FP64)
      return set_err(ctx, OQ_ERR_UNSUPPORTED,
                     "multi-determinant trials are sampled in FP64 only%s");
    cudaStream_t s = (cudaStream_t)stream;
    const OqMdState st = md_state(ctx, state, W);
    OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
    OqMoveArgs m;
    memset(&m, 0, sizeof(m));
    m.pos = st.pos; m.ainv = st.ainv; m.logdet = st.ldet; m.W = W; m.mode = 1;
    m.n_steps = n_steps; m.step = sigma; m.seed = seed; m.step_base = step_base;
    m.acc_sum = acc_sum; m.flags = ctx->d_flags;
    int rc = md_moves(ctx, m, st.sgn, stream);
    if (rc != OQ_OK) return rc;
    OQ_CUDA(ctx, to_aos(ctx, st.pos, X, W, s));
    return OQ_OK;
  }
  size_t sm;
  const int wpb = pick_wpb(ctx, 0, precision, &sm);
  if (wpb < 0)
    return set_err(ctx, OQ_ERR_UNSUPPORTED, "system too large for the shared-memory move kernel%s");
  cudaStream_t s = (cudaStream_t)stream;
  const OqStatePtrs st = state_ptrs(ctx, state, W, precision);
  OQ_CUDA(ctx, to_soa(ctx, X, st.pos, W, s));
  OqMoveArgs m;
  memset(&m, 0, sizeof(m));
  m.pos = st.pos; m.ainv = st.ainv; m.logdet = st.logdet; m.W = W; m.mode = 1;
  m.n_steps = n_steps; m.step = sigma; m.seed = seed; m.step_base = step_base;
  m.acc_sum = acc_sum; m.flags = ctx->d_flags;
  int rc = launch_moves(ctx, m, wpb, sm, precision, stream);
  if (rc != OQ_OK) return rc;
  OQ_CUDA(ctx, to_aos(ctx, st.pos, X, W, s));
  return OQ_OK;
}

int oqmc_get_flags(oqmc_ctx* ctx, unsigned* flags, int clear, void* stream) {
  if (!ctx || !flags) return OQ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned h = 0;
  OQ_CUDA(ctx, cudaMemcpyAsync(&h, ctx->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  OQ_CUDA(ctx, cudaStreamSynchronize(s));
  if (clear) OQ_CUDA(ctx, cudaMemsetAsync(ctx->d_flags, 0, sizeof(unsigned), s));
  *flags = h;
  return OQ_OK;
}

}  // extern "C"
