// Kernel instantiations and launchers for one determinant size.
// Compile with -DOQ_N=<nocc>.
#include "oqmc_launch.h"

#ifndef OQ_N
#error "compile with -DOQ_N=<nocc>"
#endif

#define OQ_CAT2(a, b) a##_##b
#define OQ_CAT(a, b) OQ_CAT2(a, b)
#define OQ_FN(name) OQ_CAT(name, OQ_N)

template <typename K>
static cudaError_t oq_smem_attr(K kernel, size_t smem) {
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

cudaError_t OQ_FN(oq_refresh)(const OqLaunch& L, const double* X, int W, void* ainv,
                              double* logdet, int mixed) {
  const int tpb = 128, nb = (W + tpb - 1) / tpb;
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_refresh<OQ_N, float>, L.smem);
    if (e != cudaSuccess) return e;
    k_refresh<OQ_N, float><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, X, W, (float*)ainv,
                                                           logdet, L.flags);
  } else {
    e = oq_smem_attr(k_refresh<OQ_N, double>, L.smem);
    if (e != cudaSuccess) return e;
    k_refresh<OQ_N, double><<<nb, tpb, L.smem, L.stream>>>(L.sys, L.C64, X, W, (double*)ainv,
                                                            logdet, L.flags);
  }
  return cudaGetLastError();
}

cudaError_t OQ_FN(oq_sweeps)(const OqLaunch& L, const OqSweepArgs& a, int wpb, int mixed) {
  const int nb = (a.W + wpb - 1) / wpb;
  cudaError_t e;
  if (mixed) {
    e = oq_smem_attr(k_sweeps<OQ_N, float, float>, L.smem);
    if (e != cudaSuccess) return e;
    k_sweeps<OQ_N, float, float><<<nb, wpb, L.smem, L.stream>>>(L.sys, L.split, L.C32, a);
  } else {
    e = oq_smem_attr(k_sweeps<OQ_N, double, double>, L.smem);
    if (e != cudaSuccess) return e;
    k_sweeps<OQ_N, double, double><<<nb, wpb, L.smem, L.stream>>>(L.sys, L.split, L.C64, a);
  }
  return cudaGetLastError();
}
