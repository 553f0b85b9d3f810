// Batched sampling of several molecules in one persistent launch (host side).
//
// oqmc_batch_create generates one module for the batch: the basis policy of
// every system (as oqmc_specialize does for one) and a persistent kernel
// k_batch that dispatches each tile to its system's code; NVRTC compiles it
// for sm_100a in a few register-budget variants, one program per variant on
// its own host thread.  The tile planner turns the walker counts and a tile
// configuration (threads per CTA, walkers per tile for each system, register
// variant) into a tile list ordered by decreasing cost, the shared-memory
// size and the persistent grid (resident CTAs per SM x SMs).
// oqmc_batch_tune searches that configuration space by timing short batched
// runs with CUDA events; oqmc_batch_capture records consecutive launches in
// a CUDA graph that oqmc_batch_replay replays.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <cuda_runtime.h>

#include "oqmc_batch.cuh"
#include "oqmc_ctx.h"
#include "oqmc_rtc.h"
#include "../../include/oqmc_b200.h"

namespace {

std::string lit(double v) {
  char b[40];
  snprintf(b, sizeof(b), "%.17g", v);
  return b;
}

// The nuclei and Jastrow constants of one system as a constant-memory
// OqJas with the values written in.
std::string jas_source(const OqSystem& S, const std::string& name) {
  std::string nuc, Z, a, b;
  for (int I = 0; I < S.natm; ++I) {
    const char* sep = I ? ", " : "";
    nuc += std::string(sep) + "{" + lit(S.nuc[I][0]) + ", " + lit(S.nuc[I][1]) + ", " +
           lit(S.nuc[I][2]) + "}";
    Z += sep + lit(S.Z[I]);
    a += sep + lit(S.j1a[I]);
    b += sep + lit(S.j1b[I]);
  }
  return "__constant__ OqJas " + name + " = {" + std::to_string(S.natm) + ", " +
         std::to_string(S.has_j1) + ", " + std::to_string(S.has_j2) + ", 0, " + lit(S.e_nn) +
         ", {" + nuc + "}, {" + Z + "}, {" + a + "}, {" + b + "}, {" + lit(S.j2[0]) + ", " +
         lit(S.j2[1]) + ", " + lit(S.j2[2]) + ", " + lit(S.j2[3]) + "}};\n";
}

struct Variant {
  int maxt, minb;
};
// register budgets: <= 255, <= 168 and <= 128 registers per thread
const Variant kVariants[] = {{256, 1}, {128, 3}, {256, 2}};
const int kNumVariants = 3;
const size_t kMaxSmem = 227 * 1024;   // opt-in shared memory per CTA on sm_100

// modes[k]: the move code compiled for molecule k (oq_batch_tile's MODE);
// empty = 0 for every molecule.
std::string batch_source(const std::vector<const OqSystem*>& S,
                         const std::vector<const OqSplit*>& SP,
                         const std::vector<const double*>& C, const std::vector<int>& nocc,
                         const std::vector<int>& modes = {}) {
  std::string src = "#include \"oqmc_batch.cuh\"\n\n";
  for (size_t k = 0; k < S.size(); ++k)
    src += oq_spec_basis_source(*S[k], *SP[k], C[k], nocc[k], "OqSpecBasis_" + std::to_string(k)) +
           "\n" + jas_source(*S[k], "oq_jas_" + std::to_string(k)) + "\n";
  src +=
      "template <typename T, typename Real, int MAXT, int MINB>\n"
      "__global__ void __launch_bounds__(MAXT, MINB) k_batch(OqBatchArgs a) {\n"
      "  extern __shared__ __align__(16) unsigned char smem[];\n"
      "  uint64_t step0, slot0;\n"
      "  oq_batch_counters(a, step0, slot0);\n"
      "  for (;;) {\n"
      "    const int k = oq_batch_next(a, smem);\n"
      "    if (k < 0) break;\n"
      "    const OqBatchTile tl = a.tiles[k];\n"
      "    const OqBatchSys d = a.systems[tl.sys];\n"
      "    switch (tl.sys) {\n";
  for (size_t k = 0; k < S.size(); ++k) {
    const std::string ks = std::to_string(k);
    const int mode = modes.empty() ? 0 : modes[k];
    src += "      case " + ks + ": oq_batch_tile<" + std::to_string(nocc[k]) +
           ", T, Real, OqSpecBasis_" + ks + ", " + std::to_string(mode) + ">(a, d, oq_jas_" +
           ks + ", tl.w0, step0, slot0, smem); break;\n";
  }
  src +=
      "      default: break;\n"
      "    }\n"
      "  }\n"
      "  oq_batch_finish(a);\n"
      "}\n";
  return src;
}

std::string kernel_name(int precision, int v) {
  const char* tr = precision == OQ_PREC_MIXED ? "float, float" : "double, double";
  return std::string("k_batch<") + tr + ", " + std::to_string(kVariants[v].maxt) + ", " +
         std::to_string(kVariants[v].minb) + ">";
}

// Shared memory of one tile (matches the carve-up in oq_batch_tile):
// positions and inverses (nt only sets the lanes per walker).
size_t tile_smem(int nocc, int wt, int nt, int precision) {
  (void)nt;
  const size_t real = precision == OQ_PREC_MIXED ? 4 : 8;
  return (size_t)6 * nocc * wt * 8 + (size_t)2 * nocc * nocc * wt * real;
}

}  // namespace

struct oqmc_batch {
  int device = 0, n = 0, precision = 0, n_sm = 0;
  std::vector<oqmc_ctx*> ctx;
  std::vector<void*> mods;       // one module per register variant
  std::vector<void*> fn;
  // module generated after tuning for the tuned shape only (each molecule's
  // move code fixed to one lane or several); used while that shape is set
  void* mod_final = nullptr;
  void* fn_final = nullptr;
  int final_threads = 0, final_variant = -1;
  std::vector<int> final_wt;
  std::vector<OqBatchSys> hsys;
  std::vector<double> cost;      // relative cost of one walker (orders the tiles)
  OqBatchSys* d_sys = nullptr;
  OqBatchTile* d_tiles = nullptr;
  int tiles_cap = 0, n_tiles = 0;
  OqBatchCtl* d_ctl = nullptr;
  unsigned long long* d_busy = nullptr;
  unsigned* d_flags = nullptr;
  bool bound = false, configured = false;
  int threads = 128, variant = 0, grid = 0;
  std::vector<int> wt;
  size_t smem = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  char err[512] = "";
};

static thread_local char g_batch_err[512] = "";

static int berr(oqmc_batch* b, int code, const std::string& msg) {
  snprintf(b ? b->err : g_batch_err, 512, "%s", msg.c_str());
  return code;
}

#define OQ_BCUDA(b, call)                                                               \
  do {                                                                                  \
    cudaError_t _e = (call);                                                            \
    if (_e != cudaSuccess) return berr(b, OQ_ERR_CUDA, std::string("CUDA error: ") +   \
                                                           cudaGetErrorString(_e));     \
  } while (0)

// The kernel for the current shape: the post-tuning module while the shape
// is the tuned one, else the general module of the register variant.
static void* kernel_fn(const oqmc_batch* b) {
  if (b->fn_final && b->threads == b->final_threads && b->variant == b->final_variant &&
      b->wt == b->final_wt)
    return b->fn_final;
  return b->fn[b->variant];
}

static void release_graph(oqmc_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
}

// Tile list, shared memory and grid for the current configuration.
static int plan(oqmc_batch* b) {
  if (!b->bound) return berr(b, OQ_ERR_ARG, "oqmc_batch_bind has not been called");
  const int nt = b->threads;
  const Variant& v = kVariants[b->variant];
  if (nt < 32 || nt % 32 || nt > v.maxt)
    return berr(b, OQ_ERR_ARG, "threads per CTA must be a multiple of 32 within the variant's limit");
  size_t smem = 0;
  for (int k = 0; k < b->n; ++k) {
    const int wt = b->wt[k];
    if (wt < 32 || wt % 32 || wt > nt || nt % wt)
      return berr(b, OQ_ERR_ARG, "walkers per tile must be a multiple of 32 dividing threads per CTA");
    smem = std::max(smem, tile_smem(b->ctx[k]->nocc, wt, nt, b->precision));
  }
  int occ = 0;
  if (oq_rtc_occupancy(kernel_fn(b), nt, smem, &occ) != 0)
    return berr(b, OQ_ERR_CUDA, "occupancy query failed");
  if (occ < 1) return berr(b, OQ_ERR_ARG, "tile configuration does not fit on an SM");
  // tiles, most expensive first
  struct T { double c; int sys, w0; };
  std::vector<T> t;
  for (int k = 0; k < b->n; ++k)
    for (int w0 = 0; w0 < b->hsys[k].W; w0 += b->wt[k])
      t.push_back({b->cost[k] * std::min(b->wt[k], b->hsys[k].W - w0), k, w0});
  std::stable_sort(t.begin(), t.end(), [](const T& x, const T& y) { return x.c > y.c; });
  std::vector<OqBatchTile> ht(t.size());
  for (size_t i = 0; i < t.size(); ++i) ht[i] = {t[i].sys, t[i].w0};
  if ((int)ht.size() > b->tiles_cap) {
    if (b->d_tiles) cudaFree(b->d_tiles);
    b->d_tiles = nullptr;
    b->tiles_cap = 0;
    OQ_BCUDA(b, cudaMalloc(&b->d_tiles, ht.size() * sizeof(OqBatchTile)));
    b->tiles_cap = (int)ht.size();
  }
  if (!ht.empty())
    OQ_BCUDA(b, cudaMemcpy(b->d_tiles, ht.data(), ht.size() * sizeof(OqBatchTile),
                           cudaMemcpyHostToDevice));
  for (int k = 0; k < b->n; ++k) b->hsys[k].wt = b->wt[k];
  OQ_BCUDA(b, cudaMemcpy(b->d_sys, b->hsys.data(), b->n * sizeof(OqBatchSys),
                         cudaMemcpyHostToDevice));
  b->n_tiles = (int)ht.size();
  b->smem = smem;
  b->grid = std::max(1, std::min(occ * b->n_sm, b->n_tiles));
  b->configured = true;
  return OQ_OK;
}

static int launch(oqmc_batch* b, int n_sweeps, int measure_every, uint64_t seed, int write_sums,
                  cudaStream_t s) {
  OqBatchArgs a;
  memset(&a, 0, sizeof(a));
  a.systems = b->d_sys;
  a.tiles = b->d_tiles;
  a.ctl = b->d_ctl;
  a.flags = b->d_flags;
  a.n_tiles = b->n_tiles;
  a.n_sweeps = n_sweeps;
  a.measure_every = measure_every;
  a.write_sums = write_sums;
  a.seed = seed;
  void* args[1] = {(void*)&a};
  if (oq_rtc_launch(kernel_fn(b), dim3(b->grid), dim3(b->threads), b->smem, s, args) != 0)
    return berr(b, OQ_ERR_CUDA, "batched kernel launch failed");
  return OQ_OK;
}

// Compile and load the batch kernel for the current shape with every
// molecule's move code fixed (one lane per walker, or several), in the
// current register variant only.
static int finalize_module(oqmc_batch* b) {
  std::vector<const OqSystem*> S;
  std::vector<const OqSplit*> SP;
  std::vector<const double*> C;
  std::vector<int> nocc, modes;
  for (int k = 0; k < b->n; ++k) {
    S.push_back(&b->ctx[k]->hsys);
    SP.push_back(&b->ctx[k]->hsplit);
    C.push_back(b->ctx[k]->h_C);
    nocc.push_back(b->ctx[k]->nocc);
    modes.push_back(b->threads / b->wt[k] > 1 ? 2 : 1);
  }
  std::vector<char> cubin;
  std::vector<std::string> lowered;
  std::string e;
  if (oq_rtc_compile(batch_source(S, SP, C, nocc, modes), {kernel_name(b->precision, b->variant)},
                     &cubin, &lowered, &e) != 0)
    return OQ_ERR_UNSUPPORTED;
  void* mod = nullptr;
  std::vector<void*> f;
  if (oq_rtc_load(cubin, lowered, &mod, &f, &e) != 0) return OQ_ERR_UNSUPPORTED;
  if (b->mod_final) oq_rtc_unload(b->mod_final);
  b->mod_final = mod;
  b->fn_final = f[0];
  b->final_threads = b->threads;
  b->final_variant = b->variant;
  b->final_wt = b->wt;
  return OQ_OK;
}

// Implemented in oqmc.cu (host-side system tables from a descriptor).
int oq_fill_system_desc(const oqmc_system_desc* d, OqSystem* S, OqSplit* SP, int* nocc,
                        std::string* err);

extern "C" {

const char* oqmc_batch_last_error(const oqmc_batch* b) { return b ? b->err : g_batch_err; }

int oqmc_batch_destroy(oqmc_batch* b) {
  if (!b) return OQ_OK;
  release_graph(b);
  if (b->d_sys) cudaFree(b->d_sys);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_ctl) cudaFree(b->d_ctl);
  if (b->d_busy) cudaFree(b->d_busy);
  if (b->d_flags) cudaFree(b->d_flags);
  for (void* m : b->mods) oq_rtc_unload(m);
  if (b->mod_final) oq_rtc_unload(b->mod_final);
  delete b;
  return OQ_OK;
}

int oqmc_batch_create(oqmc_batch** out, oqmc_ctx* const* ctxs, int n, int precision) {
  if (!out || !ctxs || n < 1 || n > 64) return berr(nullptr, OQ_ERR_ARG, "bad arguments");
  if (precision != OQ_PREC_FP64 && precision != OQ_PREC_MIXED)
    return berr(nullptr, OQ_ERR_ARG, "precision must be OQ_PREC_FP64 or OQ_PREC_MIXED");
  *out = nullptr;
  std::string e;
  if (!oq_rtc_available(&e))
    return berr(nullptr, OQ_ERR_UNSUPPORTED, "batched sampling needs NVRTC: " + e);
  for (int k = 0; k < n; ++k)
    if (!ctxs[k] || ctxs[k]->device != ctxs[0]->device)
      return berr(nullptr, OQ_ERR_ARG, "contexts must be non-null and on one device");
  oqmc_batch* b = new oqmc_batch();
  b->n = n;
  b->precision = precision;
  b->device = ctxs[0]->device;
  b->ctx.assign(ctxs, ctxs + n);
  cudaSetDevice(b->device);
  cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, b->device);
  std::vector<const OqSystem*> S;
  std::vector<const OqSplit*> SP;
  std::vector<const double*> C;
  std::vector<int> nocc;
  for (int k = 0; k < n; ++k) {
    S.push_back(&ctxs[k]->hsys);
    SP.push_back(&ctxs[k]->hsplit);
    C.push_back(ctxs[k]->h_C);
    nocc.push_back(ctxs[k]->nocc);
  }
  // one NVRTC program per register variant, compiled concurrently
  const std::string src = batch_source(S, SP, C, nocc);
  std::vector<std::vector<char>> cubin(kNumVariants);
  std::vector<std::vector<std::string>> lowered(kNumVariants);
  std::vector<std::string> cerr(kNumVariants);
  std::vector<int> crc(kNumVariants, 0);
  {
    std::vector<std::thread> th;
    for (int v = 0; v < kNumVariants; ++v)
      th.emplace_back([&, v] {
        crc[v] = oq_rtc_compile(src, {kernel_name(precision, v)}, &cubin[v], &lowered[v],
                                &cerr[v]);
      });
    for (auto& t : th) t.join();
  }
  for (int v = 0; v < kNumVariants; ++v) {
    void* mod = nullptr;
    std::vector<void*> f;
    if (crc[v] != 0 || oq_rtc_load(cubin[v], lowered[v], &mod, &f, &cerr[v]) != 0) {
      berr(nullptr, OQ_ERR_UNSUPPORTED, cerr[v]);
      oqmc_batch_destroy(b);
      return OQ_ERR_UNSUPPORTED;
    }
    b->mods.push_back(mod);
    b->fn.push_back(f[0]);
  }
  cudaError_t ce = cudaMalloc(&b->d_sys, n * sizeof(OqBatchSys));
  ce = ce == cudaSuccess ? cudaMalloc(&b->d_ctl, sizeof(OqBatchCtl)) : ce;
  ce = ce == cudaSuccess ? cudaMalloc(&b->d_busy, n * sizeof(unsigned long long)) : ce;
  ce = ce == cudaSuccess ? cudaMalloc(&b->d_flags, sizeof(unsigned)) : ce;
  ce = ce == cudaSuccess ? cudaMemset(b->d_flags, 0, sizeof(unsigned)) : ce;
  ce = ce == cudaSuccess ? cudaMemset(b->d_ctl, 0, sizeof(OqBatchCtl)) : ce;
  ce = ce == cudaSuccess ? cudaMemset(b->d_busy, 0, n * sizeof(unsigned long long)) : ce;
  if (ce != cudaSuccess) {
    berr(nullptr, OQ_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(ce));
    oqmc_batch_destroy(b);
    return OQ_ERR_CUDA;
  }
  b->hsys.resize(n);
  b->cost.resize(n);
  b->wt.assign(n, 128);
  for (int k = 0; k < n; ++k) {
    const OqSystem& s = ctxs[k]->hsys;
    // model cost of one walker-sweep: exponentials and MO accumulation per
    // electron move plus the pair terms
    b->cost[k] = (double)s.n_e * (s.nprim_total + 2.0 * s.nbf * s.nocc + s.n_e + s.natm);
  }
  *out = b;
  return OQ_OK;
}

int oqmc_batch_bind(oqmc_batch* b, const oqmc_batch_system* sys) {
  if (!b || !sys) return berr(b, OQ_ERR_ARG, "bad arguments");
  release_graph(b);
  for (int k = 0; k < b->n; ++k) {
    const oqmc_batch_system& in = sys[k];
    oqmc_ctx* c = b->ctx[k];
    if (in.W < 0 || !(in.step > 0.0) || (in.W > 0 && !in.walkers) || in.cap < 0 ||
        (in.cap > 0 && !in.sums) || (in.proposal != 0 && in.proposal != 1) ||
        (in.proposal == 1 && !(in.scale_r0 > 0.0 && in.scale_fmin > 0.0)))
      return berr(b, OQ_ERR_ARG, "bad system entry " + std::to_string(k));
    if (c->hsys.has_spl)
      return berr(b, OQ_ERR_UNSUPPORTED,
                  "system " + std::to_string(k) + " uses the radial-spline AO transform; the "
                  "batched kernel evaluates analytic radial functions");
    if (c->md)
      return berr(b, OQ_ERR_UNSUPPORTED,
                  "system " + std::to_string(k) + " has a multi-determinant trial; the "
                  "batched kernel samples single determinants");
    if (c->move_kind != 0)
      return berr(b, OQ_ERR_UNSUPPORTED,
                  "system " + std::to_string(k) + " is set to all-electron steps; the "
                  "batched kernel runs single-electron sweeps");
    OqBatchSys& d = b->hsys[k];
    memset(&d, 0, sizeof(d));
    d.sys = c->d_sys;
    d.split = c->d_split;
    d.C64 = c->d_C64;
    d.C32 = c->d_C32;
    d.walkers = in.walkers;
    d.sums = in.sums;
    d.busy_ns = b->d_busy + k;
    d.W = in.W;
    d.n_e = c->n_e;
    d.wt = b->wt[k];
    d.proposal = in.proposal;
    d.cap = in.cap;
    d.step = in.step;
    d.scale_r0 = in.scale_r0 > 0.0 ? in.scale_r0 : 1.0;
    d.scale_fmin = in.scale_fmin > 0.0 ? in.scale_fmin : 1.0;
  }
  b->bound = true;
  return plan(b);
}

int oqmc_batch_configure(oqmc_batch* b, int threads, const int* walkers_per_tile, int variant) {
  if (!b || !walkers_per_tile || variant < 0 || variant >= kNumVariants)
    return berr(b, OQ_ERR_ARG, "bad arguments");
  release_graph(b);
  const int old_t = b->threads, old_v = b->variant;
  const std::vector<int> old_wt = b->wt;
  b->threads = threads;
  b->variant = variant;
  b->wt.assign(walkers_per_tile, walkers_per_tile + b->n);
  const int rc = plan(b);
  if (rc != OQ_OK) {
    const std::string msg = b->err;
    b->threads = old_t;
    b->variant = old_v;
    b->wt = old_wt;
    if (b->bound) plan(b);
    berr(b, rc, msg);
  }
  return rc;
}

int oqmc_batch_get_config(const oqmc_batch* b, int* threads, int* walkers_per_tile, int* variant,
                          int* grid, size_t* smem, int* regs, int* local_bytes) {
  if (!b) return OQ_ERR_ARG;
  if (threads) *threads = b->threads;
  if (walkers_per_tile)
    for (int k = 0; k < b->n; ++k) walkers_per_tile[k] = b->wt[k];
  if (variant) *variant = b->variant;
  if (grid) *grid = b->grid;
  if (smem) *smem = b->smem;
  if (regs) *regs = oq_rtc_regs(kernel_fn(b));
  if (local_bytes) *local_bytes = oq_rtc_local_bytes(kernel_fn(b));
  return OQ_OK;
}

int oqmc_batch_reset(oqmc_batch* b, uint64_t step_base, void* stream) {
  if (!b) return OQ_ERR_ARG;
  OqBatchCtl c;
  memset(&c, 0, sizeof(c));
  c.step = step_base;
  cudaStream_t s = (cudaStream_t)stream;
  OQ_BCUDA(b, cudaMemcpyAsync(b->d_ctl, &c, sizeof(c), cudaMemcpyHostToDevice, s));
  OQ_BCUDA(b, cudaMemsetAsync(b->d_busy, 0, b->n * sizeof(unsigned long long), s));
  OQ_BCUDA(b, cudaStreamSynchronize(s));   // c lives on this stack frame
  return OQ_OK;
}

int oqmc_batch_run(oqmc_batch* b, int n_sweeps, int measure_every, uint64_t seed, void* stream) {
  if (!b) return OQ_ERR_ARG;
  if (n_sweeps < 1 || measure_every < 1) return berr(b, OQ_ERR_ARG, "bad arguments");
  if (!b->configured) return berr(b, OQ_ERR_ARG, "oqmc_batch_bind has not been called");
  return launch(b, n_sweeps, measure_every, seed, 1, (cudaStream_t)stream);
}

int oqmc_batch_capture(oqmc_batch* b, int n_launches, int n_sweeps, int measure_every,
                       uint64_t seed) {
  if (!b) return OQ_ERR_ARG;
  if (n_launches < 1 || n_sweeps < 1 || measure_every < 1)
    return berr(b, OQ_ERR_ARG, "bad arguments");
  if (!b->configured) return berr(b, OQ_ERR_ARG, "oqmc_batch_bind has not been called");
  release_graph(b);
  cudaStream_t cs;
  OQ_BCUDA(b, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t ce = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  int rc = OQ_OK;
  for (int i = 0; ce == cudaSuccess && rc == OQ_OK && i < n_launches; ++i)
    rc = launch(b, n_sweeps, measure_every, seed, 1, cs);
  cudaGraph_t g = nullptr;
  const cudaError_t ce2 = ce == cudaSuccess ? cudaStreamEndCapture(cs, &g) : ce;
  cudaStreamDestroy(cs);
  if (ce != cudaSuccess || ce2 != cudaSuccess || rc != OQ_OK) {
    if (g) cudaGraphDestroy(g);
    if (rc != OQ_OK) return rc;
    return berr(b, OQ_ERR_CUDA, std::string("graph capture failed: ") +
                                    cudaGetErrorString(ce != cudaSuccess ? ce : ce2));
  }
  b->graph = g;
  OQ_BCUDA(b, cudaGraphInstantiate(&b->gexec, g, 0));
  return OQ_OK;
}

int oqmc_batch_replay(oqmc_batch* b, void* stream) {
  if (!b) return OQ_ERR_ARG;
  if (!b->gexec) return berr(b, OQ_ERR_ARG, "no captured graph");
  OQ_BCUDA(b, cudaGraphLaunch(b->gexec, (cudaStream_t)stream));
  return OQ_OK;
}

int oqmc_batch_busy(oqmc_batch* b, unsigned long long* busy_ns, void* stream) {
  if (!b || !busy_ns) return OQ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  OQ_BCUDA(b, cudaMemcpyAsync(busy_ns, b->d_busy, b->n * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, s));
  OQ_BCUDA(b, cudaStreamSynchronize(s));
  return OQ_OK;
}

int oqmc_batch_get_flags(oqmc_batch* b, unsigned* flags, int clear, void* stream) {
  if (!b || !flags) return OQ_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  OQ_BCUDA(b, cudaMemcpyAsync(flags, b->d_flags, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  if (clear) OQ_BCUDA(b, cudaMemsetAsync(b->d_flags, 0, sizeof(unsigned), s));
  OQ_BCUDA(b, cudaStreamSynchronize(s));
  return OQ_OK;
}

// Autotuner.  Candidates: every register variant and CTA size (64, 128, 256
// threads, within the variant's limit); for each, walkers per tile start at
// the largest power of two <= threads whose tile fits a CTA's shared memory
// and are halved system by system
// (largest shared-memory footprint first) while that makes the batch faster.
// Each candidate is timed as the median of three launches of n_sweeps sweeps
// with local energies every n_sweeps / 2 sweeps (not accumulated).  The
// winner's per-walker cost, measured from the tiles' own timers, then orders
// the tile list.  The runs are ordinary Metropolis sweeps: they move the
// walkers and advance the sweep counter.
int oqmc_batch_tune(oqmc_batch* b, int n_sweeps, uint64_t seed, void* stream, float* best_ms) {
  if (!b) return OQ_ERR_ARG;
  if (n_sweeps < 2) return berr(b, OQ_ERR_ARG, "n_sweeps must be at least 2");
  if (!b->bound) return berr(b, OQ_ERR_ARG, "oqmc_batch_bind has not been called");
  release_graph(b);
  cudaStream_t s = (cudaStream_t)stream;
  cudaEvent_t e0, e1;
  OQ_BCUDA(b, cudaEventCreate(&e0));
  OQ_BCUDA(b, cudaEventCreate(&e1));
  const int me = n_sweeps / 2;
  auto time_it = [&](float* ms) -> int {
    float t[3];
    for (int r = 0; r < 3; ++r) {
      cudaEventRecord(e0, s);
      const int rc = launch(b, n_sweeps, me, seed, 0, s);
      if (rc != OQ_OK) return rc;
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) return berr(b, OQ_ERR_CUDA, "tuning run failed");
      cudaEventElapsedTime(&t[r], e0, e1);
    }
    std::sort(t, t + 3);
    *ms = t[1];
    return OQ_OK;
  };
  std::vector<int> order(b->n);
  for (int k = 0; k < b->n; ++k) order[k] = k;
  std::sort(order.begin(), order.end(), [&](int x, int y) {
    return tile_smem(b->ctx[x]->nocc, 32, 32, b->precision) >
           tile_smem(b->ctx[y]->nocc, 32, 32, b->precision);
  });
  float best = 1e30f;
  int best_t = b->threads, best_v = b->variant;
  std::vector<int> best_wt = b->wt;
  bool found = false;
  for (int v = 0; v < kNumVariants; ++v) {
    for (int nt : {64, 128, 256}) {
      if (nt > kVariants[v].maxt) continue;
      // start from the largest tile (walkers = threads at most) whose shared
      // memory fits one CTA
      std::vector<int> wt(b->n, 32);
      for (int k = 0; k < b->n; ++k)
        for (int c = nt; c >= 32; c /= 2)
          if (tile_smem(b->ctx[k]->nocc, c, nt, b->precision) <= kMaxSmem) {
            wt[k] = c;
            break;
          }
      float cur;
      if (oqmc_batch_configure(b, nt, wt.data(), v) != OQ_OK) continue;
      launch(b, 2, 2, seed, 0, s);   // first launch of this variant: module warm-up
      if (time_it(&cur) != OQ_OK) continue;
      for (int k : order) {
        for (int cand = wt[k] / 2; cand >= 32; cand /= 2) {
          std::vector<int> w2 = wt;
          w2[k] = cand;
          float t2;
          if (oqmc_batch_configure(b, nt, w2.data(), v) != OQ_OK) break;
          if (time_it(&t2) != OQ_OK) break;
          if (t2 < cur) {
            cur = t2;
            wt = w2;
          } else {
            break;
          }
        }
      }
      if (cur < best) {
        best = cur;
        best_t = nt;
        best_v = v;
        best_wt = wt;
        found = true;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!found) return berr(b, OQ_ERR_ARG, "no tile configuration fits");
  int rc = oqmc_batch_configure(b, best_t, best_wt.data(), best_v);
  if (rc != OQ_OK) return rc;
  // the module for the tuned shape alone (smaller code: each molecule keeps
  // only the move code of its lane count); the general one stays for other
  // shapes, and is used if this compilation fails.  Several molecules only:
  // one molecule's kernel gained nothing measurable for the extra compile
  if (b->n > 1 && finalize_module(b) == OQ_OK) {
    rc = plan(b);
    if (rc != OQ_OK) return rc;
  }
  // measured per-walker cost orders the tiles
  OQ_BCUDA(b, cudaMemsetAsync(b->d_busy, 0, b->n * sizeof(unsigned long long), s));
  rc = launch(b, n_sweeps, me, seed, 0, s);
  if (rc != OQ_OK) return rc;
  std::vector<unsigned long long> busy(b->n);
  OQ_BCUDA(b, cudaMemcpyAsync(busy.data(), b->d_busy, b->n * sizeof(unsigned long long),
                              cudaMemcpyDeviceToHost, s));
  OQ_BCUDA(b, cudaStreamSynchronize(s));
  for (int k = 0; k < b->n; ++k)
    if (b->hsys[k].W > 0 && busy[k] > 0) b->cost[k] = (double)busy[k] / b->hsys[k].W;
  rc = plan(b);
  if (rc != OQ_OK) return rc;
  OQ_BCUDA(b, cudaMemsetAsync(b->d_busy, 0, b->n * sizeof(unsigned long long), s));
  OQ_BCUDA(b, cudaStreamSynchronize(s));
  if (best_ms) *best_ms = best;
  return OQ_OK;
}

// Generated source of the batch kernel for descriptors (host only, no GPU):
// lets the run-time compilation be checked where no device is present.
int oqmc_batch_source_desc(const oqmc_system_desc* descs, int n, char* buf, size_t cap,
                           size_t* len) {
  if (!descs || n < 1) return berr(nullptr, OQ_ERR_ARG, "bad arguments");
  std::vector<OqSystem> S(n);
  std::vector<OqSplit> SP(n);
  std::vector<int> nocc(n);
  std::vector<const OqSystem*> pS;
  std::vector<const OqSplit*> pSP;
  std::vector<const double*> pC;
  for (int k = 0; k < n; ++k) {
    std::string e;
    const int rc = oq_fill_system_desc(&descs[k], &S[k], &SP[k], &nocc[k], &e);
    if (rc != OQ_OK) return berr(nullptr, rc, e);
    pS.push_back(&S[k]);
    pSP.push_back(&SP[k]);
    pC.push_back(descs[k].C);
  }
  const std::string src = batch_source(pS, pSP, pC, nocc);
  if (len) *len = src.size();
  if (buf && cap > 0) {
    const size_t m = std::min(cap - 1, src.size());
    memcpy(buf, src.data(), m);
    buf[m] = '\0';
  }
  return OQ_OK;
}

}  // extern "C"
