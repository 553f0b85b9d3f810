// Host-side launchers, one set per determinant size NOCC.  Each set lives in
// its own translation unit (oqmc_inst.cu compiled with -DOQ_N=<NOCC>) so the
// template instantiations build in parallel.
#pragma once
#include <cuda_runtime.h>
#include "oqmc_eloc_tc.cuh"
#include "oqmc_multidet.cuh"

struct OqLaunch {
  const OqSystem* sys;
  const OqSplit* split;
  const double* C64;
  const float* C32;
  unsigned* flags;
  cudaStream_t stream;
  size_t smem;
};

#define OQ_DECL_LAUNCHERS(N)                                                          \
  cudaError_t oq_eval_##N(const OqLaunch& L, const double* X, int W, double* logpsi,  \
                          double* grad, double* lap, double* eparts);                 \
  cudaError_t oq_logpsi_##N(const OqLaunch& L, const double* X, int W, double* logpsi); \
  cudaError_t oq_movals_##N(const OqLaunch& L, const double* X, int W, double* out);  \
  cudaError_t oq_refresh_##N(const OqLaunch& L, const double* pos, int W, void* ainv, \
                             double* logdet, int mixed);                              \
  cudaError_t oq_moves_##N(const OqLaunch& L, const OqMoveArgs& a, int wpb, int mixed); \
  cudaError_t oq_moves_alle_##N(const OqLaunch& L, const OqMoveArgs& a, int mixed);     \
  cudaError_t oq_eloc_##N(const OqLaunch& L, const OqElocArgs& a, int mixed);           \
  cudaError_t oq_eloc_tc_##N(const OqLaunch& L, const OqElocArgs& a, const void* Bpack, \
                             int nbf);                                                \
  cudaError_t oq_md_refresh_##N(const OqLaunch& L, const OqMdTables& T,                \
                                const OqMdState& st, int M);                           \
  cudaError_t oq_md_moves_##N(const OqLaunch& L, const OqMdTables& T,                  \
                              const OqMoveArgs& a, double* sgn, int M);                \
  cudaError_t oq_md_local_##N(const OqLaunch& L, const OqMdTables& T,                  \
                              const OqMdState& st, const OqElocArgs& a, double* logpsi, \
                              double* grad, double* lap, int M);                \
  cudaError_t oq_local_bytes_##N(int kind, int mixed, int prop, int M, size_t* out);

#define OQ_NOCC_LIST(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(10) X(12) X(14) X(16)

OQ_NOCC_LIST(OQ_DECL_LAUNCHERS)
