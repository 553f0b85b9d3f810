// Internal: the learned-proposal network object behind the opaque oqmc_mlp
// handle (not part of the public ABI).
#pragma once
#include <cuda_runtime.h>

struct oqmc_mlp {
  int device = 0;
  float* theta = nullptr;        // FP32 master parameters (W1 b1 W2 b2 W3 b3 W4 b4)
  float* m = nullptr;            // Adam moments
  float* v = nullptr;
  float* grad = nullptr;         // accumulated gradient of the current step
  unsigned short* wbf = nullptr;   // BF16 weights, row-major [out][in]
  unsigned short* wtbf = nullptr;  // BF16 transposed weights, row-major [in][out]
  unsigned* d_flags = nullptr;
  int t = 0;                     // Adam step count
  char err[512] = "";
};

// OR of the device flags since creation; OQ_ERR_TIMEOUT if a wait timed out.
int oq_mlp_check_flags(oqmc_mlp* m, cudaStream_t s);
