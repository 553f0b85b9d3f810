// Run-time specialised kernels (see oqmc_rtc.cu).
#pragma once
#include <string>
#include <cuda_runtime.h>
#include "oqmc_sweep.cuh"

struct OqSpecModule;

// Generate, compile (NVRTC, sm_100a) and load the specialised move and
// local-energy kernels of one system.  Returns 0 or -1 with *err set.
int oq_spec_build(const OqSystem& S, const OqSplit& SP, const double* C, int nocc,
                  OqSpecModule** out, std::string* err);
void oq_spec_destroy(OqSpecModule* m);
// which: 0/1 = fixed-width moves FP64/mixed, 2/3 = local energy FP64/mixed,
// 4/5 = nucleus-scaled moves FP64/mixed
int oq_spec_launch(OqSpecModule* m, int which, dim3 grid, dim3 block, size_t smem,
                   cudaStream_t stream, void** args);
std::string oq_spec_source(const OqSystem& S, const OqSplit& SP, const double* C, int nocc);
