// Arithmetic-throughput microkernels used as roofline denominators for the
// CUDA-core kernels: FP64 DFMA and FP32 FFMA issue rates and the FP32
// exponential (ex2.approx through __expf).  Each thread runs independent
// FMA chains so the pipe, not latency, bounds the rate.
#include <cuda_runtime.h>
#include "../../include/oqmc_b200.h"

template <typename T>
__global__ void k_fma_peak(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-1.2345) out[0] = s;  // keeps the chains live
}

__global__ void k_exp_peak(float* out, int iters, float a) {
  float x0 = threadIdx.x * 1e-6f, x1 = x0 + 1e-3f, x2 = x0 + 2e-3f, x3 = x0 + 3e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = __expf(x0 * a); x1 = __expf(x1 * a); x2 = __expf(x2 * a); x3 = __expf(x3 * a);
    }
  }
  const float s = x0 + x1 + x2 + x3;
  if (s == -1.2345f) out[0] = s;
}

extern "C" int oqmc_measure_peak(int kind, double* out_rate, void* stream) {
  if (!out_rate || kind < 0 || kind > 2) return OQ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int dev, sms;
  if (cudaGetDevice(&dev) != cudaSuccess) return OQ_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  void* buf;
  if (cudaMalloc(&buf, 64) != cudaSuccess) return OQ_ERR_CUDA;
  const int threads = 256, blocks = sms * 8;
  const int iters = kind == 0 ? 2048 : 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(e0, s);
    if (kind == 0)
      k_fma_peak<double><<<blocks, threads, 0, s>>>((double*)buf, iters, 0.999999, 1e-7);
    else if (kind == 1)
      k_fma_peak<float><<<blocks, threads, 0, s>>>((float*)buf, iters, 0.999999f, 1e-7f);
    else
      k_exp_peak<<<blocks, threads, 0, s>>>((float*)buf, iters, -0.5f);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  if (err != cudaSuccess) return OQ_ERR_CUDA;
  const double n = (double)blocks * threads * iters * 16.0;
  // FMA kinds: flops (2 per FMA, 8 chains); exp kind: exponentials (4 chains)
  const double ops = kind == 2 ? n * 4.0 : n * 8.0 * 2.0;
  *out_rate = ops / (best * 1e-3);
  return OQ_OK;
}
