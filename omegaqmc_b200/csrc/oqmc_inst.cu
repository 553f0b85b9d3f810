// Kernel instantiations and launchers for one determinant size.
// Compile with -DOQ_N=<nocc>.
#include "oqmc_launch.h"

#ifndef OQ_N
#error "compile with -DOQ_N=<nocc>"
#endif

#define OQ_CAT2(a, b) a##_##b
#define OQ_CAT(a, b) OQ_CAT2(a, b)
#define OQ_FN(name) OQ_CAT(name, OQ_N)

// Dynamic shared memory above 48 KB needs an opt-in; every kernel also asks
// for the largest shared-memory carveout so several CTAs fit per SM.
template <typename K>
static cudaError_t oq_smem_attr(K kernel, size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                       (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  if (smem > 48 * 1024)
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

cudaError_t OQ_FN(oq_eval)(const OqLaunch& L, const double* X, int W, double* logpsi,
                           double* grad, double* lap, double* eparts) {
  const int tpb = 128, nb = (W + tpb - 1) / tpb;
  cudaError_t e = oq_smem_attr(k_eval<OQ_N>, L.smem);
  if (e != cudaSuccess) return e;
  k_eval<OQ_N><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, X, W, logpsi, grad, lap,
                                                eparts, L.flags);
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_logpsi)(const OqLaunch& L, const double* X, int W, double* logpsi) {
  const int tpb = 128, nb = (W + tpb - 1) / tpb;
  cudaError_t e = oq_smem_attr(k_logpsi<OQ_N>, L.smem);
  if (e != cudaSuccess) return e;
  k_logpsi<OQ_N><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, X, W, logpsi, L.flags);
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_movals)(const OqLaunch& L, const double* X, int W, double* out) {
  const int tpb = 128;
  const long long n = (long long)W * 2 * OQ_N;
  const int nb = (int)((n + tpb - 1) / tpb);
  cudaError_t e = oq_smem_attr(k_mo_values<OQ_N>, L.smem);
  if (e != cudaSuccess) return e;
  k_mo_values<OQ_N><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, X, W, out);
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_refresh)(const OqLaunch& L, const double* pos, int W, void* ainv,
                              double* logdet, int mixed) {
  const int tpb = 128, nb = (W + tpb - 1) / tpb;
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_refresh<OQ_N, float>, L.smem);
    if (e != cudaSuccess) return e;
    k_refresh<OQ_N, float><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, pos, W, (float*)ainv,
                                                           logdet, L.flags);
  } else {
    e = oq_smem_attr(k_refresh<OQ_N, double>, L.smem);
    if (e != cudaSuccess) return e;
    k_refresh<OQ_N, double><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, pos, W,
                                                            (double*)ainv, logdet, L.flags);
  }
  return cudaGetLastError();
}

template <int PROP>
static cudaError_t moves_prop(const OqLaunch& L, const OqMoveArgs& a, int wpb, int mixed) {
  const int nb = (a.W + wpb - 1) / wpb;
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_moves<OQ_N, float, float, PROP>, L.smem);
    if (e != cudaSuccess) return e;
    k_moves<OQ_N, float, float, PROP><<<nb, wpb, L.smem, L.stream>>>(L.sys, L.split, L.C32, a);
  } else {
    e = oq_smem_attr(k_moves<OQ_N, double, double, PROP>, L.smem);
    if (e != cudaSuccess) return e;
    k_moves<OQ_N, double, double, PROP><<<nb, wpb, L.smem, L.stream>>>(L.sys, L.split, L.C64, a);
  }
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_moves)(const OqLaunch& L, const OqMoveArgs& a, int wpb, int mixed) {
  if (a.mode == 1) return moves_prop<2>(L, a, wpb, mixed);
  if (a.proposal == 1) return moves_prop<1>(L, a, wpb, mixed);
  return moves_prop<0>(L, a, wpb, mixed);
}

cudaError_t OQ_FN(oq_eloc)(const OqLaunch& L, const OqElocArgs& a, int mixed) {
  const int nb = (a.W + 31) / 32;
  const dim3 block(32, 2 * OQ_N);
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_eloc<OQ_N, float, float>, L.smem);
    if (e != cudaSuccess) return e;
    k_eloc<OQ_N, float, float><<<nb, block, L.smem, L.stream>>>(L.sys, L.split, L.C32, a);
  } else {
    e = oq_smem_attr(k_eloc<OQ_N, double, double>, L.smem);
    if (e != cudaSuccess) return e;
    k_eloc<OQ_N, double, double><<<nb, block, L.smem, L.stream>>>(L.sys, L.split, L.C64, a);
  }
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_eloc_tc)(const OqLaunch& L, const OqElocArgs& a, const void* Bpack, int nbf) {
  constexpr int WB = 128 / (2 * OQ_N);
  const int nb = (a.W + WB - 1) / WB;
  const size_t smem = oq_tc_plan(nbf).total;
  cudaError_t e = oq_smem_attr(k_eloc_tc<OQ_N>, smem);
  if (e != cudaSuccess) return e;
  k_eloc_tc<OQ_N><<<nb, 128, smem, L.stream>>>(L.sys, L.split,
                                                static_cast<const unsigned char*>(Bpack), a);
  return cudaGetLastError();
}

// Multi-determinant kernels: M = 8 or 16 orbital columns (M >= OQ_N).
template <int M>
static cudaError_t md_refresh_m(const OqLaunch& L, const OqMdTables& T, const OqMdState& st) {
  cudaError_t e = oq_smem_attr(k_md_refresh<OQ_N, M>, L.smem);
  if (e != cudaSuccess) return e;
  k_md_refresh<OQ_N, M><<<(st.W + 127) / 128, 128, L.smem, L.stream>>>(L.sys, T, st, L.flags);
  return cudaGetLastError();
}

template <int M>
static cudaError_t md_moves_m(const OqLaunch& L, const OqMdTables& T, const OqMoveArgs& a,
                              double* sgn) {
  cudaError_t e = oq_smem_attr(k_md_moves<OQ_N, M>, L.smem);
  if (e != cudaSuccess) return e;
  k_md_moves<OQ_N, M><<<(a.W + 127) / 128, 128, L.smem, L.stream>>>(L.sys, T, a, sgn);
  return cudaGetLastError();
}

template <int M>
static cudaError_t md_local_m(const OqLaunch& L, const OqMdTables& T, const OqMdState& st,
                              const OqElocArgs& a, double* logpsi, double* grad, double* lap) {
  cudaError_t e = oq_smem_attr(k_md_local<OQ_N, M>, L.smem);
  if (e != cudaSuccess) return e;
  k_md_local<OQ_N, M><<<(st.W + 127) / 128, 128, L.smem, L.stream>>>(L.sys, T, st, a, logpsi,
                                                                       grad, lap);
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_md_refresh)(const OqLaunch& L, const OqMdTables& T, const OqMdState& st,
                                 int M) {
  if constexpr (OQ_N <= 8) {
    if (M == 8) return md_refresh_m<8>(L, T, st);
  }
  return M == 16 ? md_refresh_m<16>(L, T, st) : cudaErrorInvalidValue;
}

cudaError_t OQ_FN(oq_md_moves)(const OqLaunch& L, const OqMdTables& T, const OqMoveArgs& a,
                               double* sgn, int M) {
  if constexpr (OQ_N <= 8) {
    if (M == 8) return md_moves_m<8>(L, T, a, sgn);
  }
  return M == 16 ? md_moves_m<16>(L, T, a, sgn) : cudaErrorInvalidValue;
}

cudaError_t OQ_FN(oq_md_local)(const OqLaunch& L, const OqMdTables& T, const OqMdState& st,
                               const OqElocArgs& a, double* logpsi, double* grad, double* lap,
                               int M) {
  if constexpr (OQ_N <= 8) {
    if (M == 8) return md_local_m<8>(L, T, st, a, logpsi, grad, lap);
  }
  return M == 16 ? md_local_m<16>(L, T, st, a, logpsi, grad, lap) : cudaErrorInvalidValue;
}

cudaError_t OQ_FN(oq_moves_alle)(const OqLaunch& L, const OqMoveArgs& a, int mixed) {
  const int tpb = 128, nb = (a.W + tpb - 1) / tpb;
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_moves_alle<OQ_N, float>, L.smem);
    if (e != cudaSuccess) return e;
    k_moves_alle<OQ_N, float><<<nb, tpb, L.smem, L.stream>>>(
        L.sys, L.C64, a.pos, (float*)a.ainv, a.logdet, a.W, a.n_steps, a.step, a.seed,
        a.step_base, a.acc_sum, L.flags);
  } else {
    e = oq_smem_attr(k_moves_alle<OQ_N, double>, L.smem);
    if (e != cudaSuccess) return e;
    k_moves_alle<OQ_N, double><<<nb, tpb, L.smem, L.stream>>>(
        L.sys, L.C64, a.pos, (double*)a.ainv, a.logdet, a.W, a.n_steps, a.step, a.seed,
        a.step_base, a.acc_sum, L.flags);
  }
  return cudaGetLastError();
}

// Per-thread local memory (bytes) of one kernel this size launches: kind 0
// k_refresh, 1 k_moves (prop 0/1/2), 2 k_eloc, 3 k_eloc_tc, 4 k_md_refresh,
// 5 k_md_moves, 6 k_md_local (M = 8 or 16 columns), 7 k_moves_alle.
template <typename K>
static cudaError_t oq_lmem(K kernel, size_t* out) {
  cudaFuncAttributes a;
  const cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e == cudaSuccess) *out = a.localSizeBytes;
  return e;
}

template <int M>
static cudaError_t md_lmem(int kind, size_t* out) {
  if (kind == 4) return oq_lmem(k_md_refresh<OQ_N, M>, out);
  if (kind == 5) return oq_lmem(k_md_moves<OQ_N, M>, out);
  return oq_lmem(k_md_local<OQ_N, M>, out);
}

cudaError_t OQ_FN(oq_local_bytes)(int kind, int mixed, int prop, int M, size_t* out) {
  switch (kind) {
    case 0:
      return mixed ? oq_lmem(k_refresh<OQ_N, float>, out) : oq_lmem(k_refresh<OQ_N, double>, out);
    case 1:
      if (prop == 2)
        return mixed ? oq_lmem(k_moves<OQ_N, float, float, 2>, out)
                     : oq_lmem(k_moves<OQ_N, double, double, 2>, out);
      if (prop == 1)
        return mixed ? oq_lmem(k_moves<OQ_N, float, float, 1>, out)
                     : oq_lmem(k_moves<OQ_N, double, double, 1>, out);
      return mixed ? oq_lmem(k_moves<OQ_N, float, float, 0>, out)
                   : oq_lmem(k_moves<OQ_N, double, double, 0>, out);
    case 2:
      return mixed ? oq_lmem(k_eloc<OQ_N, float, float>, out)
                   : oq_lmem(k_eloc<OQ_N, double, double>, out);
    case 3:
      return oq_lmem(k_eloc_tc<OQ_N>, out);
    case 4:
    case 5:
    case 6:
      if constexpr (OQ_N <= 8) {
        if (M == 8) return md_lmem<8>(kind, out);
      }
      return M == 16 ? md_lmem<16>(kind, out) : cudaErrorInvalidValue;
    case 7:
      return mixed ? oq_lmem(k_moves_alle<OQ_N, float>, out)
                   : oq_lmem(k_moves_alle<OQ_N, double>, out);
  }
  return cudaErrorInvalidValue;
}
