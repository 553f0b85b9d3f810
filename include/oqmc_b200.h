/*
 * oqmc_b200.h -- C ABI of liboqmc_b200.so, the B200 (sm_100a) kernels for
 * the GTO variational Monte Carlo hot path of OmegaQMC: Slater-Jastrow
 * wavefunction evaluation and single-electron Metropolis sweeps.
 *
 * Conventions
 *  - All array arguments are DEVICE pointers (plain memory the caller owns;
 *    the library borrows them for the duration of the enqueued work), except
 *    the oqmc_system_desc tables, which are host memory read at create time.
 *  - Walkers are (W, n_e, 3) FP64 arrays, electrons in the reference's spin
 *    layout: spin up at even positions, spin down at odd positions.
 *  - Work is enqueued on the caller's stream (cudaStream_t passed as void*;
 *    NULL = legacy default stream) and the call returns without waiting,
 *    except oqmc_get_flags, which synchronises the stream.
 *  - Every function returns 0 on success or a negative OQ_ERR_* code and
 *    never aborts; oqmc_last_error() describes the last failure.
 *  - A context is bound to the device that was current at create time and
 *    is not thread-safe: use one context per host thread / stream.
 *
 * The reference (myung-group/OmegaQMC) is Python/JAX with no native layer:
 * each entry point below replaces a jitted JAX function of the reference,
 * cited beside it as path:line within that project.
 */
#ifndef OQMC_B200_H
#define OQMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OQ_OK 0
#define OQ_ERR_ARG (-1)
#define OQ_ERR_CUDA (-2)
#define OQ_ERR_NAN (-3)
#define OQ_ERR_SINGULAR (-4)
#define OQ_ERR_TIMEOUT (-5)
#define OQ_ERR_UNSUPPORTED (-6)
#define OQ_ERR_NOMEM (-7)

/* kernel flag bits reported by oqmc_get_flags */
#define OQ_FLAG_NAN 1u
#define OQ_FLAG_SINGULAR 2u

/* precision of the sampler state and move arithmetic */
#define OQ_PREC_FP64 0   /* everything FP64 */
#define OQ_PREC_MIXED 1  /* FP32 AO/MO/inverse, FP64 refresh + accumulation */

typedef struct oqmc_ctx oqmc_ctx;

/*
 * Molecular system.  Basis functions are grouped by exponent list: group g
 * is one basis entry of one atom (OmegaQMC/psi/shell.py:150-256 read_shell,
 * psi/gto.py:890-913 _parse_shells) with nprim[g] exponents shared by
 * ncol[g] contracted shells (the columns of a general contraction).  Shells
 * are numbered group by group, column by column; AOs follow in the order of
 * _angular_cartesian (psi/gto.py:607-671), 2*am+1 per shell.
 */
typedef struct {
  int natm;              /* nuclei */
  int nbf;               /* spherical AOs */
  int nocc;              /* occupied orbitals per spin (n_up == n_dn) */
  int n_e;               /* electrons = 2 * nocc */
  const double* nuc;     /* natm*3, bohr */
  const double* Z;       /* natm nuclear charges */
  int ngroup;
  const int* group_atom;   /* ngroup */
  const int* group_am;     /* ngroup */
  const int* group_nprim;  /* ngroup */
  const int* group_ncol;   /* ngroup, 1..4 */
  const double* alpha;     /* sum(nprim) exponents, group-major */
  const double* norm;      /* sum(nprim*ncol): for g, for column, for prim */
  const int* shell_cusp;   /* sum(ncol) flags: cusp-corrected s shell */
  const double* C;         /* nbf*nocc occupied MO coefficients, row-major */
  int has_j1;
  const double* j1;        /* natm*2 Pade (a, b) per atom */
  int has_j2;
  const double* j2;        /* 4: like a, like b, unlike a, unlike b */
  int cusp;
  const double* cusp_rc;   /* natm */
  const double* cusp_q0;   /* natm */
  const double* cusp_coeff;/* natm*8 */
  double e_nn;             /* nuclear repulsion (eps-softened) */
  /* Cubic B-spline Jastrow terms (psi/gto.py:1657-1931), full coefficient
   * vectors c[0..N+3] (parameters N + 4, cusp and boundary coefficients
   * included) on knots k * r_cut / (N + 1). */
  int has_bs2;
  int bs2_ncoef_like, bs2_ncoef_unlike;   /* N + 4, at most 32 */
  double bs2_rcut;
  const double* bs2_coef_like;
  const double* bs2_coef_unlike;
  int has_bs1;
  int bs1_ntype;                           /* element types, at most 4 */
  const int* bs1_type;                     /* natm: type of each atom, -1 none */
  const int* bs1_ncoef;                    /* ntype */
  const double* bs1_rcut;                  /* ntype */
  const double* bs1_coef;                  /* ntype blocks of ncoef values */
  /* Three-body electron-electron-nucleus polynomial Jastrow (J3_eeI,
   * psi/gto.py:243-604, 1933-2196): per element type a like-spin and an
   * unlike-spin block of gammas g[l][m][n] (already expanded from the free
   * parameters, symmetric in l, m), zero beyond r_eI = j3_rcut / 2. */
  int has_j3;
  int j3_n_ei, j3_n_ee;                    /* orders: 0..6 and 1..6 */
  int j3_ntype;                            /* element types, at most 4 */
  double j3_rcut;
  const int* j3_type;                      /* natm: type of each atom, -1 none */
  const int* j3_on;                        /* ntype x 2: like / unlike block present */
  const double* j3_gamma;                  /* ntype x 2 x (n_ei+1)^2 x (n_ee+1) */
  /* Quintic radial splines of the AO transform (psi/gto.py:141-240): table
   * t holds knots in s = r^2 (spl_npts, knot 0 at s = 0, then a log grid
   * from spl_smin) and spl_npts - 1 segments of 6 power-form coefficients
   * (highest power first).  spl_shell: per shell (descriptor order) its
   * table, -1 for the analytic radial. */
  int has_spl;
  int spl_npts, spl_ntab;
  double spl_smin;
  const int* spl_shell;
  const double* spl_knots;                 /* ntab x npts */
  const double* spl_coef;                  /* ntab x (npts - 1) x 6 */
} oqmc_system_desc;

/* Library version string. */
const char* oqmc_version(void);

/* Build a context on the current device.  Replaces _PsiGTO.__init__
 * (OmegaQMC/psi/gto.py:820-844) / get_psi_fun (gto.py:2601-2621). */
int oqmc_create(oqmc_ctx** out, const oqmc_system_desc* desc);
int oqmc_destroy(oqmc_ctx* ctx);
/* Text of the last error of ctx (or of the last failed oqmc_create when
 * ctx is NULL). */
const char* oqmc_last_error(const oqmc_ctx* ctx);

/* Full FP64 evaluation of W walkers: log|psi| (W), grad log|psi| (W,n_e,3),
 * per-electron Laplacian of log|psi| (W,n_e) and local-energy parts (W,4:
 * ee, en, ke, total incl. e_nn).  grad/lap/eparts may be NULL.
 * Replaces vmap(log_trial_wavefunction) (psi/gto.py:2220-2254) together
 * with vmap(local_energy_ee/en/ke) (gto.py:2432-2451, 2506-2579) and
 * _local_energy_batch (OmegaQMC/vmc_gto.py:801-812). */
int oqmc_eval(oqmc_ctx* ctx, const double* walkers, int W, double* logpsi,
              double* grad, double* lap, double* eparts, void* stream);

/* log|psi| only (value path). Replaces _log_psi_batch
 * (OmegaQMC/vmc_gto.py:790-797). */
int oqmc_log_psi(oqmc_ctx* ctx, const double* walkers, int W, double* logpsi,
                 void* stream);

/* Occupied MO values (W, n_e, nocc) at every electron.  Replaces the
 * mo_val output of get_psi_mo (OmegaQMC/psi/gto.py:1058-1070). */
int oqmc_mo_values(oqmc_ctx* ctx, const double* walkers, int W, double* out,
                   void* stream);

/* Bytes of sampler state for W walkers at a precision: walker-minor
 * positions, inverse Slater matrices and log|det|.  The state is derived
 * from the walkers by oqmc_refresh; after changing walkers outside the
 * library, refresh before the next sweep. */
size_t oqmc_state_bytes(const oqmc_ctx* ctx, int W, int precision);

/* Full FP64 LU refresh of the sampler state from positions (the periodic
 * recompute that bounds Sherman-Morrison drift). */
int oqmc_refresh(oqmc_ctx* ctx, const double* walkers, int W, void* state,
                 int precision, void* stream);

/* Equilibration with the step adapted on the device: n_steps sweeps, each
 * followed by the reference's rule log s <- log s + rate (acc - target)
 * applied to the width at `step` (one device double, read by the next sweep
 * and left holding the final width); the equilibration_step scan of
 * OmegaQMC/vmc_gto.py:1338-1357 with _adapt_step_size (121-126), without
 * the host reading the acceptance between steps.  acc_trace (device,
 * n_steps) receives each sweep's acceptance ratio, step_trace (device,
 * n_steps, optional) the width after each adaptation.  The state is
 * refreshed (FP64 LU) whenever refresh_every sweeps have passed since the
 * last refresh, counting from since_refresh at entry.  Random numbers as
 * oqmc_sweeps (counter step_base + t).  Single-determinant, single-electron
 * Gaussian or nucleus-scaled sweeps; other contexts return
 * OQ_ERR_UNSUPPORTED. */
int oqmc_equilibrate(oqmc_ctx* ctx, double* walkers, int W, void* state, int precision,
                     int n_steps, double* step, double target, double rate, uint64_t seed,
                     uint64_t step_base, int refresh_every, int since_refresh,
                     double* acc_trace, double* step_trace, void* stream);

/* Per-walker outputs of the sampler state in its own precision: what the
 * sampler itself sees, for stating the error of each output of the mixed
 * path against the FP64 evaluation.  Counterparts: log_trial_wavefunction
 * (OmegaQMC/psi/gto.py:2220-2254) and the grad_flat / per-electron
 * Laplacian / local-energy parts of local_energy_ke (gto.py:2506-2579) and
 * local_energy_ee/en (gto.py:2406-2451).  logpsi (W) = the state's
 * Sherman-Morrison-tracked log|det| (FP64 sum of the accepted moves' ratio
 * logarithms since the last refresh) + the Jastrow in working precision;
 * grad (W x n_e x 3) and lap (W x n_e) from the state's inverse (FP32 in
 * the mixed state) and the working-precision orbitals and Jastrow; eparts
 * (W x 4) ee, en, ke, E_L.  Any output may be null.  Uses the specialised
 * local-energy kernel when the context is specialised; positions and state
 * are not changed. */
int oqmc_state_eval(oqmc_ctx* ctx, const void* state, int W, int precision,
                    double* logpsi, double* grad, double* lap, double* eparts,
                    void* stream);

/* n_sweeps single-electron Metropolis sweeps over all walkers (positions
 * updated in place), measuring the local energy after every
 * measure_every-th sweep.  sums: (n_sweeps/measure_every, 8) doubles that
 * are ACCUMULATED into (zero them first): sum ee, en, ke, E_L, E_L^2,
 * accepted moves, finite-E_L walkers.  el_trace: optional
 * (n_meas, W) per-walker E_L.  eparts_last: optional (W,4) parts of the
 * last measurement.  Random numbers: Philox4x32-10 keyed by seed, counter
 * (walker, step_base + sweep, electron).  walkers_per_block: CTA size (32,
 * 64 or 128; 0 = default).  Replaces the production scan body
 * (OmegaQMC/vmc_gto.py:985-1034) and metropolis_move_1w (841-905). */
int oqmc_sweeps(oqmc_ctx* ctx, double* walkers, int W, void* state,
                int precision, int n_sweeps, int measure_every, double step,
                uint64_t seed, uint64_t step_base, double* sums,
                double* el_trace, double* eparts_last, int walkers_per_block,
                void* stream);

/* n_steps basin relocations on every walker: one random electron is
 * proposed at N(R_J, sigma^2) around a random nucleus J and accepted with
 * the exact Metropolis-Hastings ratio including q(old)/q(new),
 * q(x) = sum_J exp(-|x - R_J|^2 / 2 sigma^2).  acc_sum: optional device
 * double that accumulates accepted moves.  Replaces basin_move_1w and
 * _thermalize_basins (OmegaQMC/vmc_gto.py:925-957, 1036-1053). */
int oqmc_basin(oqmc_ctx* ctx, double* walkers, int W, void* state, int precision,
               int n_steps, double sigma, uint64_t seed, uint64_t step_base,
               double* acc_sum, void* stream);

/* Size of the device array behind oqmc_sweeps_noalloc (every GPU that
 * loads the library holds it until the library is unloaded). */
#define OQ_NOALLOC_SCRATCH_BYTES (16u << 20)

/* Allocation-free sampling, for callers that cannot allocate device memory
 * (their device memory belongs to another allocator's arena or budget, or
 * a cudaMalloc would synchronise the device on their path).  No counterpart
 * in the reference.  Runs oqmc_refresh + oqmc_sweeps with the walker state
 * in a library-owned 16 MiB device array instead of a caller buffer: every
 * call refreshes the state from `walkers`, then runs the sweeps; the other
 * arguments mean what they mean for oqmc_sweeps.  W is limited to
 * oqmc_state_bytes(ctx, W, precision) <= OQ_NOALLOC_SCRATCH_BYTES (about
 * 25,000 FP64 H2O walkers); larger W returns OQ_ERR_ARG.  Calls no
 * allocating routine.  The first call on a device looks up the array's
 * device address; make it before any stream capture.  Under CUDA's default
 * lazy module loading that first call can also load the library's kernels
 * into device memory: make one call outside the memory-constrained region
 * (or set CUDA_MODULE_LOADING=EAGER).  A call whose kernels need more
 * per-thread local memory than the device's current stack limit
 * (cudaLimitStackSize) returns OQ_ERR_UNSUPPORTED instead of letting the
 * driver grow its local-memory reservation: at the default 1 KiB this
 * refuses all-electron steps and multi-determinant trials until an
 * allocating call has raised the limit.  All calls share the array: calls
 * that overlap on the GPU race, so serialise them. */
int oqmc_sweeps_noalloc(oqmc_ctx* ctx, double* walkers, int W, int precision,
                        int n_sweeps, int measure_every, double step,
                        uint64_t seed, uint64_t step_base, double* sums,
                        double* el_trace, double* eparts_last, void* stream);

/* Proposal of the single-electron moves of oqmc_sweeps: kind 0 (default)
 * is the reference's fixed-width Gaussian (metropolis_move_alle,
 * OmegaQMC/vmc_gto.py:815-839, applied per electron); kind 1 scales the width
 * with the distance to the nearest nucleus, sigma(x) = step *
 * clamp(r_near(x) / r0, fmin_frac, 1), and corrects the acceptance with the
 * exact proposal-density ratio, so the stationary distribution is unchanged
 * while core electrons move with core-sized steps. */
int oqmc_set_proposal(oqmc_ctx* ctx, int kind, double r0, double fmin_frac);
/* Move kind of oqmc_sweeps: 0 (default) single-electron
 * sweeps (n_e proposals per sweep, Sherman-Morrison updates); 1 the
 * reference's all-electron step (metropolis_move_alle + metropolis_move_1w,
 * OmegaQMC/vmc_gto.py:815-905): per "sweep" one proposal moving every
 * electron by step * N(0, 1), accepted on the ratio of |psi|^2 evaluated
 * afresh in FP64.  The proposal width setting (oqmc_set_proposal) applies
 * to single-electron sweeps only; the learned proposal, multi-determinant
 * trials and oqmc_batch_bind refuse kind 1.  The accepted-move sum counts
 * electron moves in both kinds: an accepted all-electron step adds n_e.
 * The all-electron kernel's per-thread stack exceeds the default local-memory
 * reservation, so oqmc_sweeps_noalloc refuses kind 1 on a device whose stack
 * limit has not been raised (see there). */
int oqmc_set_move_kind(oqmc_ctx* ctx, int kind);
/* Multi-determinant trial (the `trial` dict of get_psi_fun /
 * get_vmc_gto_func, OmegaQMC/psi/gto.py:846-863, 1312-1488):
 *   psi_S = sum_d coef[d] det(Phi_up[:, occ_up[d]]) det(Phi_dn[:, occ_dn[d]])
 * with Phi the orbitals of the ncol columns of C (nbf x ncol, row-major;
 * for UHF trials the alpha and beta columns side by side, occ_dn indexing
 * the beta half).  occ_up, occ_dn: ndet x nocc column indices in
 * determinant order.  At most 16 distinct columns and 64 distinct
 * determinants per spin.  Evaluation (oqmc_eval, oqmc_log_psi) and
 * sampling (oqmc_refresh, oqmc_sweeps, oqmc_basin) then use the expansion,
 * in FP64 only (oqmc_sweeps_noalloc included, under its local-memory rule);
 * the batched, learned-proposal
 * and tensor-core paths refuse it.  ndet = 0 returns to the single determinant
 * of the descriptor.  Sampler state sizes (oqmc_state_bytes) change with the
 * expansion.  With an expansion, oqmc_eval and oqmc_log_psi refresh a
 * scratch state kept on the context: it grows with cudaMalloc when a call
 * has more walkers than any before (synchronising that call's stream). */
int oqmc_set_multidet(oqmc_ctx* ctx, int ndet, int ncol, const double* C, const double* coef,
                      const int* occ_up, const int* occ_dn);
/* Terms, distinct up / down determinants and padded orbital columns of the
 * context's expansion (all 0 for a single determinant). */
int oqmc_multidet_info(const oqmc_ctx* ctx, int* ndet, int* nu_up, int* nu_dn, int* ncol);

/* Mixed-precision local energy with the MO contraction (the GEMM
 * AO(5 components) x C of get_psi_mo_vgl, OmegaQMC/psi/gto.py:1188-1214) on
 * the tcgen05 tensor cores: 128 (walker, electron) rows per CTA, split
 * TF32/BF16 operands for near-FP32 accuracy, FP32 accumulators in TMEM.
 * enable = 0 returns to the CUDA-core local-energy kernel. */
int oqmc_use_tensor_cores(oqmc_ctx* ctx, int enable);

/* Per-system specialisation (no counterpart in the reference, whose jit
 * unrolls the shell loop at trace time, OmegaQMC/psi/gto.py:1012-1186):
 * generate the AO->MO evaluation of this molecule as straight-line code with
 * exponents and coefficients compiled in, compile the move and local-energy
 * kernels with NVRTC for sm_100a and use them from then on (enable = 0
 * returns to the table-driven kernels).  Takes a few seconds; returns
 * OQ_ERR_UNSUPPORTED when NVRTC is not available. */
int oqmc_specialize(oqmc_ctx* ctx, int enable);

/* The generated specialisation source (of a context, or of a descriptor
 * without any device work): writes at most len-1 chars plus NUL into buf
 * and returns the full length (or a negative OQ_ERR_* code). */
int oqmc_spec_source(const oqmc_ctx* ctx, char* buf, size_t len);
int oqmc_spec_source_desc(const oqmc_system_desc* desc, char* buf, size_t len);

/* Exponent threshold above which an exponent group is evaluated in FP64
 * near its nucleus in the mixed build (default 50.0; <= 0 disables). */
int oqmc_set_split(oqmc_ctx* ctx, double tight_alpha);

/* Synchronise `stream`, return the OR of kernel flag bits since the last
 * clear in *flags and optionally clear them. */
int oqmc_get_flags(oqmc_ctx* ctx, unsigned* flags, int clear, void* stream);

/* Measured arithmetic throughput of the current GPU, the roofline
 * denominators of the CUDA-core kernels: kind 0 = FP64 FMA flop/s,
 * 1 = FP32 FMA flop/s, 2 = FP32 exponentials/s (SFU).  A measurement
 * utility with no counterpart in the reference. */
int oqmc_measure_peak(int kind, double* out_rate, void* stream);

/* Jastrow-parameter derivatives per walker, the inputs of the linear-method
 * optimiser (compute_walker_derivs, OmegaQMC/vmcopt_gto_linear.py:686-703,
 * which differentiates log_trial_wavefunction and the local energy with
 * jax.grad).  Raw parameters, oqmc_param_count(ctx) of them: J2 like a,
 * like b, unlike a, unlike b, then J1 a_I, b_I for every atom (Padé; absent
 * terms give zeros), then the B-spline parameters: J2 like, J2 unlike, then
 * J1 per element type (bs1_ncoef - 4 each, types in descriptor order), then
 * the three-body gammas: per J3 element type in descriptor order, the like
 * and then the unlike block when present, (n_ei+1)(n_ei+2)/2 (n_ee+1) unique
 * gammas g[l][m][n], l >= m, ordered by m, then l, then n (the caller maps
 * them onto the free parameters with the constraint matrix).  grad = the
 * (W, n_e, 3) gradient of ln|psi| that oqmc_eval returns for the same
 * walkers; outputs dlogpsi, dEL are (W, count), FP64. */
int oqmc_param_count(const oqmc_ctx* ctx);
int oqmc_param_derivs(oqmc_ctx* ctx, const double* walkers, int W, const double* grad,
                      double* dlogpsi, double* dEL, void* stream);

/* ------------------------------------------------------------------------
 * Batched sampling: several molecules (contexts) of different electron and
 * basis counts share one persistent launch.  No counterpart in the
 * reference, whose driver samples one molecule per run
 * (OmegaQMC/vmc_gto.py:1233-1617 VMCDriverGTO.__call__); per system a launch
 * does what oqmc_refresh followed by oqmc_sweeps does here
 * (_make_production_step, vmc_gto.py:985-1034, as single-electron sweeps),
 * with the same random-number counters, so the walkers it leaves are those
 * of the per-system path.
 * ---------------------------------------------------------------------- */
typedef struct oqmc_batch oqmc_batch;

/* One system of a batch. */
typedef struct {
  double* walkers;       /* (W, n_e, 3) device positions, updated in place */
  int W;
  int proposal;          /* 0 fixed-width Gaussian, 1 nucleus-scaled */
  double step;           /* Gaussian width (scale s of the scaled proposal) */
  double scale_r0;       /* nucleus-scaled width: step*clamp(r_near/r0, fmin, 1) */
  double scale_fmin;
  double* sums;          /* [cap][8] device measurement sums (as oqmc_sweeps),
                            accumulated; slot = measurement index since reset */
  int cap;
} oqmc_batch_system;

/* Generate and compile (NVRTC, sm_100a) the batch kernel for n contexts on
 * one device at a precision (tens of seconds for five cc-pVDZ molecules).
 * OQ_ERR_UNSUPPORTED without NVRTC. */
int oqmc_batch_create(oqmc_batch** out, oqmc_ctx* const* ctxs, int n, int precision);
int oqmc_batch_destroy(oqmc_batch* b);
const char* oqmc_batch_last_error(const oqmc_batch* b);
/* Attach walkers and proposal settings (n entries) and plan the tiles. */
int oqmc_batch_bind(oqmc_batch* b, const oqmc_batch_system* sys);
/* Tile shape: threads per CTA, walkers per tile of each system (multiples
 * of 32 dividing threads) and register variant (0: <= 255 registers per
 * thread, 1: <= 168 with at most 128 threads, 2: <= 128). */
int oqmc_batch_configure(oqmc_batch* b, int threads, const int* walkers_per_tile, int variant);
int oqmc_batch_get_config(const oqmc_batch* b, int* threads, int* walkers_per_tile,
                          int* variant, int* grid, size_t* smem, int* regs, int* local_bytes);
/* Autotune the tile shape by timing short batched runs (moves the walkers,
 * accumulates nothing); *best_ms = time of n_sweeps sweeps with the winner. */
int oqmc_batch_tune(oqmc_batch* b, int n_sweeps, uint64_t seed, void* stream, float* best_ms);
/* Sweep counter of the next launch = step_base, measurement slot = 0, tile
 * timers cleared (synchronises stream). */
int oqmc_batch_reset(oqmc_batch* b, uint64_t step_base, void* stream);
/* One persistent launch: FP64 refresh, then n_sweeps sweeps with a
 * measurement every measure_every sweeps, for every system. */
int oqmc_batch_run(oqmc_batch* b, int n_sweeps, int measure_every, uint64_t seed, void* stream);
/* Capture n_launches consecutive launches in a CUDA graph (the counters
 * advance on the device between them); oqmc_batch_replay launches it. */
int oqmc_batch_capture(oqmc_batch* b, int n_launches, int n_sweeps, int measure_every,
                       uint64_t seed);
int oqmc_batch_replay(oqmc_batch* b, void* stream);
/* Per-system sum of tile durations (ns) since the last reset (synchronises). */
int oqmc_batch_busy(oqmc_batch* b, unsigned long long* busy_ns, void* stream);
int oqmc_batch_get_flags(oqmc_batch* b, unsigned* flags, int clear, void* stream);
/* Generated batch source for descriptors (host only). */
int oqmc_batch_source_desc(const oqmc_system_desc* descs, int n, char* buf, size_t cap,
                           size_t* len);

/* ------------------------------------------------------------------------
 * Learned Metropolis proposal.  No counterpart in the reference, whose
 * proposal is the plain Gaussian random walk (metropolis_move_alle,
 * OmegaQMC/vmc_gto.py:815-839).  A per-electron MLP (32 features -> 128 ->
 * 128 -> 128 -> 48, ReLU, BF16 weights and activations, FP32 accumulation on
 * the tcgen05 tensor cores) outputs an 8-component isotropic Gaussian
 * mixture for the electron's displacement; moves are accepted with the
 * exact ratio |psi'|^2 q(x|x') / (|psi|^2 q(x'|x)) (the Metropolis-Hastings
 * form of metropolis_move_1w, vmc_gto.py:841-905, as the basin move uses it,
 * vmc_gto.py:925-957).  Parameters are a flat FP32 vector of
 * oqmc_mlp_num_params() values: W1[128][32] b1 W2[128][128] b2 W3[128][128]
 * b3 W4[48][128] b4.  Features of electron e: position relative to the
 * nearest and second-nearest nucleus (6), displacements to the 8 nearest
 * other electrons (24, nearest first), spin (+1 up / -1 down), 1.
 * Outputs: logits 0..7, means 8..31, sigma_c = 0.02 + softplus(out[32+c]).
 * ---------------------------------------------------------------------- */
typedef struct oqmc_mlp oqmc_mlp;

int oqmc_mlp_num_params(void);
/* Allocate on the current device with He-uniform weights (seeded). */
int oqmc_mlp_create(oqmc_mlp** out, uint64_t seed);
int oqmc_mlp_destroy(oqmc_mlp* m);
const char* oqmc_mlp_last_error(const oqmc_mlp* m);
/* FP32 parameters to/from host memory (set also resets the Adam state). */
int oqmc_mlp_get_params(oqmc_mlp* m, float* theta_host);
int oqmc_mlp_set_params(oqmc_mlp* m, const float* theta_host);
/* Training rows of walkers X0 (W, n_e, 3): BF16 features feat[W*n_e][32]
 * (row = walker * n_e + electron) and, when X1 (positions some sweeps
 * later) is given, the FP32 targets X1 - X0 in target[W*n_e][3]. */
int oqmc_mlp_features(oqmc_ctx* ctx, const double* X0, const double* X1, int W,
                      unsigned short* feat, float* target, void* stream);
/* Network outputs out[R][48] (FP32) of R feature rows. */
int oqmc_mlp_forward(oqmc_mlp* m, const unsigned short* feat, int R, float* out, void* stream);
/* Gradient of the mean negative log-likelihood of the targets over the R
 * rows (grad: device, num_params floats, overwritten) and the summed NLL
 * (loss_sum: device double, may be NULL). */
int oqmc_mlp_backward(oqmc_mlp* m, const unsigned short* feat, const float* target, int R,
                      float* grad, double* loss_sum, void* stream);
/* One Adam step (beta 0.9/0.999) on the mean NLL of the R rows. */
int oqmc_mlp_step(oqmc_mlp* m, const unsigned short* feat, const float* target, int R,
                  float lr, double* loss_sum, void* stream);
int oqmc_mlp_get_flags(oqmc_mlp* m, unsigned* flags, int clear, void* stream);
/* Use the network as the context's proposal in oqmc_sweeps (mixed
 * precision, specialised context; NULL restores the previous proposal).
 * The network is borrowed and must outlive its use. */
int oqmc_set_mlp_proposal(oqmc_ctx* ctx, const oqmc_mlp* m);
/* Walker groups of 128 per CTA of the learned-proposal sweep (2 or 4,
 * default 2): the groups share the weights in shared memory and overlap
 * each other's network and wavefunction work.  32,768 walkers make 256
 * groups, so 4 per CTA would leave most of the 148 SMs idle. */
int oqmc_set_mlp_groups(oqmc_ctx* ctx, int groups);

#ifdef __cplusplus
}
#endif
#endif /* OQMC_B200_H */
