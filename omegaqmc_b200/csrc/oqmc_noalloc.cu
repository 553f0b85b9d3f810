// Allocation-free sampling entry point.
//
// Some callers cannot allocate device memory themselves: a host runtime that
// hands the GPU to a fixed arena owned by another allocator (a framework's
// caching pool, a JVM or Go binding under a hard device-memory budget) may
// forbid side allocations, and on latency-critical paths a cudaMalloc can
// synchronise the whole device.  oqmc_sweeps_noalloc serves them: it runs
// the same refresh and sweep kernels as oqmc_refresh + oqmc_sweeps, but
// keeps the walker state (walker-minor positions, inverse Slater matrices,
// log|det|) in a file-scope device array instead of a caller buffer.
//
// The array holds OQ_NOALLOC_SCRATCH_BYTES (16 MiB) on every GPU that loads
// the library, for as long as the library stays loaded.  Its device address
// is looked up once per device (cudaGetSymbolAddress, with that device
// current) by the first call on that device; make that first call before
// any stream capture.  All calls share the one array and it keeps the last
// call's contents, so calls that overlap on the GPU (different streams or
// contexts on one device) race with each other: serialise them.  Every call
// rewrites the whole state it uses from the caller's walkers before the first
// sweep, so nothing in it needs to start at zero.
//
// Two things outside this file can still allocate device memory on a call,
// and the entry point guards against or documents both:
//  * Local memory.  The driver reserves per-thread stack for every resident
//    thread at the size of the device's current stack limit and grows the
//    reservation when a launched kernel needs more.  Before launching, the
//    call compares the local memory of every kernel it would run with
//    cudaDeviceGetLimit(cudaLimitStackSize) and refuses (OQ_ERR_UNSUPPORTED)
//    rather than grow it.
//  * Module loading.  Under CUDA's default lazy loading a kernel's module is
//    loaded into device memory on its first use, so the first call on a
//    device may allocate for that.  Make one call (or one oqmc_sweeps call on
//    the same context) outside the memory-constrained region, or run with
//    CUDA_MODULE_LOADING=EAGER.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/oqmc_b200.h"

#define OQ_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_oq_scratch[OQ_NOALLOC_SCRATCH_BYTES];

static void* g_scratch_ptr[OQ_NOALLOC_MAX_DEVICES];
static std::mutex g_scratch_mu;

// Device address of g_oq_scratch on the current device (host code must not
// use the symbol itself: it is a host-side stand-in, not a device address).
static cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= OQ_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_oq_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

int oq_ctx_set_error(oqmc_ctx* ctx, int code, const char* msg);
int oq_ctx_sweep_local_bytes(oqmc_ctx* ctx, int precision, size_t* out);

extern "C" int oqmc_sweeps_noalloc(oqmc_ctx* ctx, double* walkers, int W, int precision,
                                   int n_sweeps, int measure_every, double step,
                                   uint64_t seed, uint64_t step_base, double* sums,
                                   double* el_trace, double* eparts_last, void* stream) {
  if (!ctx) return OQ_ERR_ARG;
  if (W < 0 || n_sweeps < 0 || (precision != OQ_PREC_FP64 && precision != OQ_PREC_MIXED))
    return oq_ctx_set_error(ctx, OQ_ERR_ARG, "bad arguments");
  if (W == 0 || n_sweeps == 0) return OQ_OK;
  // a kernel whose per-thread local memory exceeds the device's current
  // stack limit makes the driver grow its local-memory reservation at launch,
  // which is a device allocation (the all-electron step and the
  // multi-determinant kernels need more than the default 1 KiB)
  size_t lmem = 0, limit = 0;
  const int lrc = oq_ctx_sweep_local_bytes(ctx, precision, &lmem);
  if (lrc != OQ_OK) return lrc;
  const cudaError_t le = cudaDeviceGetLimit(&limit, cudaLimitStackSize);
  if (le != cudaSuccess) return oq_ctx_set_error(ctx, OQ_ERR_CUDA, cudaGetErrorString(le));
  if (lmem > limit) {
    char msg[256];
    snprintf(msg, sizeof(msg),
             "a kernel of this call needs %zu B of local memory per thread, above the "
             "device's current stack reservation of %zu B; growing it is an allocation: "
             "use oqmc_sweeps", lmem, limit);
    return oq_ctx_set_error(ctx, OQ_ERR_UNSUPPORTED, msg);
  }
  const size_t need = oqmc_state_bytes(ctx, W, precision);
  if (need > (size_t)OQ_NOALLOC_SCRATCH_BYTES)
    return oq_ctx_set_error(ctx, OQ_ERR_ARG,
                            "walker state exceeds the 16 MiB scratch of the "
                            "allocation-free entry point; use fewer walkers per call "
                            "or oqmc_sweeps with a caller buffer");
  void* scratch = nullptr;
  const cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) return oq_ctx_set_error(ctx, OQ_ERR_CUDA, cudaGetErrorString(e));
  int rc = oqmc_refresh(ctx, walkers, W, scratch, precision, stream);
  if (rc != OQ_OK) return rc;
  return oqmc_sweeps(ctx, walkers, W, scratch, precision, n_sweeps, measure_every, step, seed,
                     step_base, sums, el_trace, eparts_last, 0, stream);
}
