// Run-time specialised kernels (see oqmc_rtc.cu).
#pragma once
#include <string>
#include <vector>
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
// The CUfunction behind `which` (numbering as for oq_spec_launch).
void* oq_spec_function(OqSpecModule* m, int which);
std::string oq_spec_source(const OqSystem& S, const OqSplit& SP, const double* C, int nocc);

// The basis policy of one system as C++ source for a struct named `name`.
std::string oq_spec_basis_source(const OqSystem& S, const OqSplit& SP, const double* C, int nocc,
                                 const std::string& name);

// Generic run-time compilation: compile src (with the library's kernel
// headers available by name) for sm_100a, load it and resolve the kernels
// named by C++ name expressions.  Handles are CUmodule / CUfunction.
int oq_rtc_available(std::string* err);
// Compile only (thread-safe, no device work) / load a compiled image on the
// current device.
int oq_rtc_compile(const std::string& src, const std::vector<std::string>& names,
                   std::vector<char>* cubin, std::vector<std::string>* lowered,
                   std::string* err);
int oq_rtc_load(const std::vector<char>& cubin, const std::vector<std::string>& lowered,
                void** mod, std::vector<void*>* fns, std::string* err);
int oq_rtc_build(const std::string& src, const std::vector<std::string>& names, void** mod,
                 std::vector<void*>* fns, std::string* err);
void oq_rtc_unload(void* mod);
int oq_rtc_launch(void* fn, dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                  void** args);
// Resident CTAs per SM for a block size and dynamic shared memory (0: does not fit).
int oq_rtc_occupancy(void* fn, int block, size_t smem, int* nblk);
int oq_rtc_regs(void* fn);
int oq_rtc_local_bytes(void* fn);
