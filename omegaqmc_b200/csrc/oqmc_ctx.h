// Internal: the context object behind the opaque oqmc_ctx handle, shared by
// the library's translation units (not part of the public ABI).
#pragma once
#include "oqmc_sweep.cuh"

struct OqSpecModule;

// Multi-determinant expansion of a context (device tables and the scratch
// state the evaluation entry points use).
struct OqMdHost {
  int ndet, nu0, nu1, M;
  double* d_C;          // nbf x M
  double* d_coef;
  int* d_det;
  int* d_occ;
  void* d_scratch;      // evaluation state for up to scratch_w walkers
  int scratch_w;
};

struct oqmc_ctx {
  int device;
  int nocc, n_e, nbf, natm;
  OqSystem hsys;
  OqSplit hsplit;
  OqSystem* d_sys;
  OqSplit* d_split;
  double* d_C64;
  float* d_C32;
  unsigned* d_flags;
  double* d_j3;            // three-body Jastrow gamma blocks (or null)
  double* d_spl_knots;     // radial spline tables (or null)
  double* d_spl_coef;
  double tight_alpha;
  int proposal;           // 0 fixed-width Gaussian, 1 nucleus-scaled width
  int move_kind;          // 0 single-electron sweeps, 1 all-electron steps
  OqSpecModule* spec;     // run-time specialised kernels, or null
  int use_tc;             // mixed local energy on the tensor cores
  unsigned char* d_Btc;   // split MO-coefficient operands of k_eloc_tc
  double* h_C;            // host copy of the MO coefficients (for specialisation)
  double scale_r0, scale_fmin;
  const struct oqmc_mlp* mlp;   // learned proposal (borrowed), or null
  void* mlp_mod;                // its specialised sweep kernels (module; 2 and 4 groups)
  void* mlp_fn[2];
  int mlp_groups;               // walker groups per CTA of the learned-proposal sweep
  OqMdHost* md;                 // multi-determinant expansion, or null
  char err[512];
};

// Record an error message on a context and return code.
int oq_ctx_set_error(oqmc_ctx* ctx, int code, const char* msg);
