/*
 * tups_b200 — B200 (sm_100a) implementation of the TUPS parquet loop hot path.
 *
 * C ABI: plain pointers, sizes and int status codes; no C++ or torch types.
 * Every complex array crossing this boundary is complex(dp) / double _Complex,
 * i.e. interleaved (re, im) doubles, passed as `double*` with 2*n entries, in
 * the reference's Fortran column-major layout, so a Fortran caller hands over
 * `c_loc(array)` without transposes.
 *
 * The reference keeps all state in module globals (SRC/parquet_ini.f90:67-285)
 * and its entry points take at most an iteration counter.  Here that state
 * lives on the GPU inside an opaque context; each entry point below replaces
 * the Fortran routine cited beside it and operates on the context's
 * device-resident state.  Host copies move only through tups_get_* /
 * tups_set_*.
 *
 * Threading: one context per process and thread; not re-entrant.
 * Status: 0 = ok, negative = error (TUPS_ERR_*); tups_last_error() gives
 * the message.  Nothing here aborts the process.
 */
#ifndef TUPS_B200_H
#define TUPS_B200_H

#include <stddef.h> /* size_t */

#ifdef __cplusplus
extern "C" {
#endif

#define TUPS_OK 0
#define TUPS_ERR_CUDA (-1)      /* a CUDA runtime call failed */
#define TUPS_ERR_OOM (-2)       /* device allocation failed */
#define TUPS_ERR_MU_NOCONV (-3) /* mu bisection exceeded its step cap */
#define TUPS_ERR_NAN (-4)       /* NaN/Inf in Sigma or a vertex */
#define TUPS_ERR_TIMEOUT (-5)   /* a bounded device wait ran out */
#define TUPS_ERR_BADDIM (-6)    /* unsupported or inconsistent sizes */
#define TUPS_ERR_BADARG (-7)    /* bad argument (NULL pointer, index range) */
#define TUPS_ERR_IO (-8)        /* input file unreadable or malformed */
#define TUPS_ERR_STATE (-9)     /* call order violated (e.g. PAE before PhiR) */
#define TUPS_ERR_COMM (-10)     /* a host exchange between ranks failed */

/* channel numbering as in the reference's select case(channel): d, m, s, t */
#define TUPS_CH_D 0
#define TUPS_CH_M 1
#define TUPS_CH_S 2
#define TUPS_CH_T 3

/* Input parameters: the 21-record prms file (SRC/parquet_ini.f90:300-322)
 * plus the extensions that the reference hard-codes (t', SRC/parquet_ini.f90:24)
 * or does not have (absolute convergence norm). */
typedef struct tups_params {
  double beta;          /* prms record 1 */
  double U;             /* 2 */
  double nParticle;     /* 3 */
  int Nx;               /* 4 (Ny = Nx) */
  int Nf;               /* 5, even */
  int neighbours;       /* 6 */
  int readinpick;       /* 7 */
  char pick_file[256];  /* 8 */
  int Ngrain;           /* 9 */
  int f_range;          /* 10 */
  double f_damping;     /* 11 */
  int ite_max;          /* 12 */
  int DGA;              /* 13: Lambda from fname_L + "_ph.init" / "_pp.init" (SRC/parquet_util.f90:317-346) */
  char fname_L[256];    /* 14 */
  int use_sig_dmft;     /* 15 */
  char fname_sig_dmft[256]; /* 16 */
  int use_U2;           /* 17 */
  int save_F;           /* 18 */
  int oneshot;          /* 19 */
  int old;              /* 20 (must be 0) */
  int SDE_old;          /* 21 (must be 0) */
  double tprime;        /* extension: -4 t' cos kx cos ky in the dispersion */
  double conv_abs;      /* extension: converged when max|dSigma| < conv_abs (0 = reference test) */
} tups_params;

/* Derived sizes (SRC/parquet_ini.f90:326-349, SRC/preprocessing.f90:127-133). */
typedef struct tups_dims {
  int Nx, Ny, Nf, Ngrain;
  int Nx_IBZ, NIBZ, Nred, Nc;
  int Nl, Nz, Nt, Nb, NR;
  int nbox;      /* (2*f_range+1)*Nf */
  int wperTask;  /* Nf/2 at one task */
} tups_dims;

/* Output of conv() (SRC/parquet_check.f90:39-150) */
typedef struct tups_conv_info {
  double rel_sig_max;   /* max |SigmaOld-Sigma|/|Sigma| */
  double rel_sig_av;    /* |sum(...)|/Nt */
  double dsigma_inf;    /* max |SigmaOld-Sigma| (extension norm) */
  double F_max[4];      /* max |F_r| */
  double rel_err[4];    /* |1 - max|F_r| / previous max|F_r|| */
  double mu;
  int bisection_steps;
  int converged;
} tups_conv_info;

typedef struct tups_ctx tups_ctx;

/* ---- setup ------------------------------------------------------------ */
/* set_parameters: parse the 21-record prms file (SRC/parquet_ini.f90:289-324).
 * t' and conv_abs come from the optional file `<path>.gpu` (`key = value`
 * lines, keys tprime and conv_abs, `!` or `#` comments), else 0; an unknown
 * key or a bad value there returns TUPS_ERR_IO. */
int tups_read_prms(const char* path, tups_params* out);
/* Initialization + FF_array + do_preprocessing's vertex init
 * (SRC/parquet_util.f90:14-478, SRC/parquet_formfactors.f90:11-90,
 * SRC/preprocessing.f90:100-133): builds all tables on the host, allocates and
 * fills device state on `device`. */
int tups_ctx_create(const tups_params* p, int device, tups_ctx** out);
int tups_ctx_destroy(tups_ctx* ctx);

/* Slot-sharded context: rank `rank` of `ntasks` holds the contiguous bosonic
 * slots [rank*Nb, (rank+1)*Nb), Nb = Nred/ntasks, as the reference's MPI ranks
 * do (`Nb = Nred/ntasks`, `id*Nb + idx_q`: SRC/parquet_ini.f90:336,
 * SRC/preprocessing.f90:98-116); ntasks must divide Nred, as the reference
 * requires (SRC/preprocessing.f90:95-98).  Vertices, chi and the BSE are
 * local; Phi(R), Sigma and mu are replicated.  The three steps that need
 * every slot call the exchange function set by tups_set_exchange: the
 * Phi(R) partial sums over the rank's momenta (communicatePhis /
 * FTPhis, SRC/parquet_PhiR.f90:114-258), the self-energy sum over slots
 * (SRC/parquet_SDE.f90:221-258) and max|F_r| of conv
 * (SRC/parquet_check.f90:109-117).  Iterations of a sharded context are not
 * replayed from CUDA graphs, and tups_readout needs an unsharded context. */
int tups_ctx_create_sharded(const tups_params* p, int device, int rank, int ntasks, tups_ctx** out);

/* Exchange between the ranks of a sharded context: combine `count` doubles
 * at device address `data` over all ranks, in place (op TUPS_XCH_SUM or
 * TUPS_XCH_MAX), and return 0, or nonzero on failure (the library then
 * returns TUPS_ERR_COMM).  `what` names the buffer: TUPS_XCH_PHIR + r for
 * Phi(R) of channel r (0..3), TUPS_XCH_SIGMAV, TUPS_XCH_FMAX.  The library
 * synchronises its stream before the call; the data must be complete in
 * device memory when the function returns.  Every rank makes the same calls
 * in the same order. */
typedef int (*tups_exchange_fn)(void* user, int what, double* data, size_t count, int op);
#define TUPS_XCH_SUM 0
#define TUPS_XCH_MAX 1
#define TUPS_XCH_PHIR 0
#define TUPS_XCH_SIGMAV 4
#define TUPS_XCH_FMAX 5
int tups_set_exchange(tups_ctx* ctx, tups_exchange_fn fn, void* user);
/* rank, ntasks and the first global slot of this context (0, 1, 0 unsharded) */
int tups_get_shard(const tups_ctx* ctx, int* rank, int* ntasks, int* slot0);
/* Host-only part of tups_ctx_create (no device needed): derived sizes and the
 * form-factor / symmetry / index tables in the layouts of tups_get_tables.
 * Lets a caller size its host arrays before creating a context. Any output
 * pointer may be NULL. */
int tups_host_tables(const tups_params* p, tups_dims* d, double* FF, double* FF_inv, int* signs, int* reps,
                     int* lsym, double* lfac, int* ibz);
/* The DGA branch of Initialization (SRC/parquet_util.f90:317-346) without a
 * device: reads `<fname_L>_ph.init` (Lambda_d, Lambda_m) and `_pp.init`
 * (Lambda_s, Lambda_t) into (Nf, Nf, Nf/2) complex arrays, the tables a DGA
 * context starts from.  Any output pointer may be NULL. */
int tups_read_lambda(const char* fname_L, int Nf, double* L_d, double* L_m, double* L_s, double* L_t);
int tups_get_dims(const tups_ctx* ctx, tups_dims* out);
const char* tups_last_error(const tups_ctx* ctx);
const char* tups_strerror(int status);

/* ---- module parquet_chi ---------------------------------------------- */
/* calc_Gkw_Grt(ite, Grt, cal_chi) (SRC/parquet_chi.f90:18-210): Sigma_H, mu
 * bisection (capped; TUPS_ERR_MU_NOCONV), G(r,tau) and G(k,nu).  The chi0
 * readout branch (:216-430) is not part of this call. */
int tups_calc_Gkw_Grt(tups_ctx* ctx, int ite, int cal_chi);
/* calc_chi(map_q, chi_ph_LL, chi_pp_LL) (SRC/parquet_chi.f90:438-523) for the
 * 1-based bosonic IBZ slot idx_q of this context (1..Nb; in a sharded context
 * global slot slot0 + idx_q, as the reference's id*Nb + idx_q); writes the
 * dense (Nz,Nz) matrices to host. */
int tups_calc_chi(tups_ctx* ctx, int idx_q, double* chi_ph_LL, double* chi_pp_LL);

/* ---- module Parquet_kernel ------------------------------------------- */
/* BSE(ite) (SRC/parquet_BSE.f90:19-135): on exit G_r holds Phi_r. */
int tups_BSE(tups_ctx* ctx, int ite);

/* ---- module parquet_PhiR --------------------------------------------- */
int tups_calculate_expSqR(tups_ctx* ctx);  /* SRC/parquet_PhiR.f90:360-395 */
int tups_calculate_expqSR(tups_ctx* ctx);  /* SRC/parquet_PhiR.f90:400-435 */
int tups_calc_PhiR(tups_ctx* ctx, int ite); /* SRC/parquet_PhiR.f90:35-109 */

/* ---- module parquet_EQMatrix (iteration 0) -------------------------- */
int tups_calc_M_phbar_to_ph(tups_ctx* ctx); /* SRC/parquet_EQMatrix.f90:21-123 */
int tups_calc_M_pp_to_ph(tups_ctx* ctx);    /* SRC/parquet_EQMatrix.f90:126-194 */
int tups_calc_M_ph_to_pp(tups_ctx* ctx);    /* SRC/parquet_EQMatrix.f90:198-271 */
int tups_calc_M_phbar_to_pp(tups_ctx* ctx); /* SRC/parquet_EQMatrix.f90:274-360 */

/* ---- module parquet_EQOuter / parquet_EQContribs -------------------- */
/* calculate_PAE (SRC/parquet_EQOuter.f90:16-118) with all crossing
 * contributions of SRC/parquet_EQContribs.f90:44-524; F_r is written once. */
int tups_calculate_PAE(tups_ctx* ctx);

/* ---- module parquet_SDE ---------------------------------------------- */
/* calc_SDE(ite, Grt) (SRC/parquet_SDE.f90:27-258); saves SigmaOld first,
 * as loop.f90:152 does. */
int tups_calc_SDE(tups_ctx* ctx, int ite);

/* ---- module parquet_check -------------------------------------------- */
/* conv() (SRC/parquet_check.f90:39-150); also SigmaOld = Sigma. */
int tups_conv(tups_ctx* ctx, tups_conv_info* info);

/* ---- loop.f90 --------------------------------------------------------- */
/* Gamma_r = F_r - Phi_r (SRC/loop.f90:219-222) */
int tups_vertex_update(tups_ctx* ctx);
/* the every-5-iterations readout's effect on the trajectory (SRC/loop.f90:195,
 * SRC/parquet_chi.f90:114-122): mu <- midpoint of [mu-U, mu+U] */
int tups_output_block(tups_ctx* ctx);
/* one pass of execute_loop (SRC/loop.f90:51-244) without the readout: on
 * output iterations only the readout's effect on mu is applied */
int tups_iteration(tups_ctx* ctx, int ite, tups_conv_info* info);
/* enable = 1: tups_iteration (from ite 1 on, phase timing off) replays the
 * iteration's device work from a CUDA graph captured on first use per
 * precision choice, with one host synchronisation per iteration.  No
 * counterpart in the reference. */
int tups_set_graph(tups_ctx* ctx, int enable);
/* execute_loop (SRC/loop.f90:29-249) including the readout of every output
 * iteration (SRC/loop.f90:181-213; results via tups_get_chi0/tups_get_sus);
 * *ite_out = iterations done */
int tups_execute_loop(tups_ctx* ctx, int* ite_out, int* converged);
/* One iteration of execute_loop with its output block (SRC/loop.f90:181-213):
 * at iterations ite % 5 == 0, ite_max - 1 and on convergence the readout
 * (tups_readout) runs after conv and before the vertex update, as in the
 * reference, and its results stay readable (tups_get_chi0, tups_get_sus)
 * until the next readout.  Unsharded contexts only. */
int tups_iteration_readout(tups_ctx* ctx, int ite, tups_conv_info* info);

/* ---- warm start and checkpoint ----------------------------------------------
 * Warm start at the reference's initialisation hook (SRC/preprocessing.f90:100-116,
 * SRC/parquet_util.f90:178-233): Sigma <- sigma (Nt complex, host); mu by
 * bisection for it; Gamma_r <- gamma_l1[r] (4 complex, host) on the (l=1,l=1)
 * nu-block and 0 elsewhere; F_r from ONE BSE solve in LU form,
 * F_r = (1 - 2 c_r/(beta Nx Ny) Gamma_r chi_r)^{-1} Gamma_r, i.e. the fixed
 * point of the reference's damped update for that Gamma_r.  Then continue
 * with tups_iteration. */
int tups_warm_start(tups_ctx* ctx, const double* sigma, const double* gamma_l1);
/* device-side copy of the loop state (Sigma, SigmaOld, mu, F_r, G_r, previous
 * vertex maxima): save = 1 stores it, save = 0 restores the stored copy */
int tups_checkpoint(tups_ctx* ctx, int save);

/* ---- split-precision BSE and ZGEMM ---------------------------------------------
 * No counterpart in the reference (its BSE GEMMs are FP64 ZGEMMs,
 * SRC/parquet_BSE.f90:72-128).  The complex GEMM is emulated with int8
 * slices on the tensor cores (tcgen05 kind::i8, exact int32 sums) and FP64
 * recombination: relative error about 10^(1.1 - 2 s) of max|A| max|B| K
 * for s slices per operand (s = 8: FP64 level).
 * tups_set_bse_precision: slices = 0 keeps the FP64 tensor-core GEMM;
 * 2..8 uses s slices in every BSE; ladder = 1 picks s per iteration from the
 * last relative Sigma change (3 slices before the first, 8 at the end). */
int tups_set_bse_precision(tups_ctx* ctx, int slices, int ladder);
/* slices the next BSE will use (0 = FP64) */
int tups_get_bse_slices(const tups_ctx* ctx);
/* Batched C_b = A_b B_b: A (M, K), B (K, N), C (M, N) column-major complex128,
 * batches packed contiguously, all DEVICE pointers; work: device buffer of
 * tups_zgemm_split_workspace() bytes.  Synchronises the stream. */
size_t tups_zgemm_split_workspace(int batch, int M, int N, int K, int slices);
int tups_zgemm_split(int batch, int M, int N, int K, const double* A, const double* B, double* C, int slices,
                     void* work, size_t work_bytes, void* stream);
/* Failure detection of the split GEMM's bounded device waits (its pipeline
 * barriers).  cycles > 0: a wait of the work loop gives up after that many SM
 * clock cycles (0 restores the default, about 2 s); the CTA then waits for
 * its copies and MMAs already in flight, frees its tensor memory and returns,
 * and the call (or the next conv/iteration of a context) reports
 * TUPS_ERR_TIMEOUT.  stall_test = 1: the next split GEMM launch first waits
 * on a barrier that nothing signals, so that wait runs out (a test of the
 * timeout path that faults nothing); later launches run normally.
 * Process-wide. */
int tups_set_split_wait(long long cycles, int stall_test);
/* Column tile of the split GEMM (real columns of [Re B | Im B] per CTA tile):
 * n_tile = 16, 32, ..., 128 fixes it, 0 restores the automatic choice (the
 * fewest tiles, then the widest).  Every tile shape gives the same bits (the
 * integer slice sums are exact and the FP64 folding order is fixed).
 * Process-wide; no counterpart in the reference. */
int tups_set_split_tile(int n_tile);
/* The split GEMM on CTA pairs: enable = 1 runs row counts >= 256 as
 * 256 x n_tile tiles over two SMs (tcgen05 cta_group::2, each SM staging
 * half of the B operand), 0 (default) as 128 x n_tile tiles on one SM each.
 * Both give the same bits.  Process-wide; no counterpart in the reference. */
int tups_set_split_cta_pairs(int enable);

/* ---- tile-shape tuner -------------------------------------------------------
 * No counterpart in the reference.  The first FP64 BSE GEMM and the first
 * crossing call of a context on a new shape time their candidate tilings on
 * the call's own operands (CUDA events on the library's stream; the BSE on
 * scratch copies of Gamma) and keep the fastest for that shape in this
 * process.  The candidates differ only in how output elements are spread over
 * CTAs and warps, never in the order of a sum, so results do not depend on
 * the choice.  Not run during a stream capture.  On by default; the
 * environment variable TUPS_AUTOTUNE=0 or enable = 0 fixes the default tiles. */
int tups_set_autotune(tups_ctx* ctx, int enable);
/* Real tensor-core products per complex multiply-add in the crossing GEMM of
 * tups_calculate_PAE: 3 (default; Gauss: Xr Mr, Xi Mi, (Xr + Xi)(Mr + Mi))
 * or 4, for 5 or more form factors.  Both agree with the reference's
 * crossing sums (parquet_EQContribs.f90:44-524) to rounding; the three-product
 * form rounds differently.  No counterpart in the reference. */
int tups_set_crossing_products(tups_ctx* ctx, int products);
/* The choices made so far in this process as text, one line per kernel and
 * shape: "<kernel> <shape> | choice <name> | <name>=<ms> ...".  Writes at
 * most len bytes (NUL-terminated) and returns the length the whole table
 * needs, NUL included; buf may be NULL with len 0 to ask for it. */
int tups_get_tuning(char* buf, size_t len);
/* Fix the candidate named `name` for every tuner key that starts with
 * key_prefix (e.g. "k_pae_mma(3M) Nl=5"), in this process, ahead of the
 * tuner and its cached choices; a key whose candidates do not include the
 * name keeps the tuner's choice.  name = NULL drops that prefix's entry;
 * key_prefix = NULL drops all.  Every candidate writes the same bits, so
 * this only selects a launch shape (for tests and profiling). */
int tups_set_tuning(const char* key_prefix, const char* name);

/* ---- multilayer perceptron of the learned warm start ------------------------
 * No counterpart in the reference.  FP32 network n_in -> n_hidden (x n_layers,
 * SiLU) -> n_out (linear), trained by Adam on the mean squared error.  Flat
 * parameters [W_0, b_0, W_1, b_1, ...], W_l (out, in) row-major.  Inputs,
 * targets and outputs are HOST row-major (batch, features) float arrays. */
typedef struct tups_mlp tups_mlp;
int tups_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, int max_batch, int device, tups_mlp** out);
int tups_mlp_destroy(tups_mlp* m);
const char* tups_mlp_last_error(const tups_mlp* m);
long long tups_mlp_num_params(const tups_mlp* m);
long long tups_mlp_kernel_launches(const tups_mlp* m);
/* set_params also resets the optimiser state */
int tups_mlp_set_params(tups_mlp* m, const float* host);
int tups_mlp_get_params(tups_mlp* m, float* host);
int tups_mlp_forward(tups_mlp* m, const float* x, int batch, float* y);
/* loss (mean squared error) and its gradient w.r.t. the flat parameters;
 * grad or loss may be NULL */
int tups_mlp_gradients(tups_mlp* m, const float* x, const float* t, int batch, float* grad, double* loss);
/* epochs of minibatch Adam (beta 0.9/0.999, eps 1e-8) over a resident copy of
 * (x, t), shuffled per epoch from seed; decoupled weight decay on W only;
 * loss_per_epoch (optional, host, epochs entries) = mean minibatch loss */
int tups_mlp_train(tups_mlp* m, const float* x, const float* t, int n_samples, int batch, int epochs, float lr,
                   float weight_decay, unsigned long long seed, double* loss_per_epoch);

/* ---- readout (SRC/loop.f90:181-213 without HDF5) -------------------------- */
/* calc_Gkw_Grt(ite, Grt, .true.) with the exact chi0 bubble
 * (SRC/parquet_chi.f90:216-430), calc_sus (SRC/parquet_sus.f90:18-643) and
 * symmetrize_sus (SRC/parquet_plot.f90:14-58).  Call between tups_conv and
 * tups_vertex_update, as the reference does. */
int tups_readout(tups_ctx* ctx, int ite);
/* chi0 of the last readout. bz = 0: IBZ arrays chi0_ph, chi0_pp (Nred) and
 * chi0_ph_FF, chi0_pp_FF (Nred, 4); bz = 1: the whole-BZ versions
 * (Nx*Ny*Nf/2) and (Nx*Ny*Nf/2, 4).  Any pointer may be NULL. */
int tups_get_chi0(tups_ctx* ctx, int bz, double* ph, double* pp, double* ph_FF, double* pp_FF);
/* sus_r of the last readout: bz = 0 sus_r_IBZ (Nred, 4), bz = 1 sus_r (Nx*Ny*Nf/2, 4) */
int tups_get_sus(tups_ctx* ctx, int channel, int bz, double* host);

/* ---- state in/out (host buffers, reference layouts) ------------------ */
int tups_get_sigma(tups_ctx* ctx, double* sigma);         /* (Nt) */
int tups_set_sigma(tups_ctx* ctx, const double* sigma);   /* (Nt) */
int tups_get_sigma_old(tups_ctx* ctx, double* sigma);     /* (Nt) */
int tups_get_Gkw(tups_ctx* ctx, double* gkw);             /* (Nt) */
int tups_get_Grt(tups_ctx* ctx, double* grt);             /* (Nx*Ng, Ny*Ng, Nf) */
int tups_get_mu(tups_ctx* ctx, double* mu);
int tups_set_mu(tups_ctx* ctx, double mu);
/* which: 0 = F_r (complete vertex), 1 = G_r (Gamma_r, or Phi_r between BSE
 * and the vertex update); layout (Nz, Nz, Nb) */
int tups_get_vertex(tups_ctx* ctx, int channel, int which, double* host);
int tups_set_vertex(tups_ctx* ctx, int channel, int which, const double* host);
/* the same for `count` consecutive slots from the 0-based local slot
 * `slot_begin` only: (Nz, Nz, count), the F_r/G_r columns a parity dump or the
 * reference's vertex output of save_F (write_F, SRC/parquet_plot.f90:237-276)
 * needs without moving the whole (Nz, Nz, Nb) array */
int tups_get_vertex_slots(tups_ctx* ctx, int channel, int which, int slot_begin, int count, double* host);
int tups_set_vertex_slots(tups_ctx* ctx, int channel, int which, int slot_begin, int count, const double* host);
int tups_get_PhiR(tups_ctx* ctx, int channel, double* host);  /* (Nz*Nz, Nf/2, NR) */
/* which: 0 phbar_to_ph, 1 pp_to_ph, 2 ph_to_pp, 3 phbar_to_pp;
 * layout (Nl, Nl, Nl, Nl, Nb, NR) as M_* of SRC/parquet_EQMatrix.f90:12-16 */
int tups_get_M(tups_ctx* ctx, int which, double* host);
int tups_get_expSqR(tups_ctx* ctx, double* host);   /* (NIBZ, NR, 8) */
int tups_get_expqSR(tups_ctx* ctx, double* host);   /* (Nc, NR, 8) */
/* form-factor tables: FF (Nx,Ny,Nl) and FF_inv (8,Nx,Ny,Nl) real; signs,
 * reps (Nl); l-space symmetry maps lsym (8,Nl) 1-based, lfac (8,Nl);
 * index_bosonic_IBZ (3,Nred) 1-based. Any pointer may be NULL. */
int tups_get_tables(tups_ctx* ctx, double* FF, double* FF_inv, int* signs, int* reps,
                    int* lsym, double* lfac, int* ibz);
/* SDE intermediates of the last calc_SDE: chi_aux_ph/pp (Nl*nbox, Nb) and
 * LChi, PhChi, PPChi (Nz, Nb); any pointer may be NULL */
int tups_get_sde_aux(tups_ctx* ctx, double* chi_aux_ph, double* chi_aux_pp,
                     double* LChi, double* PhChi, double* PPChi);
int tups_synchronize(tups_ctx* ctx);
/* number of this library's kernels launched since context creation */
long long tups_kernel_launches(const tups_ctx* ctx);

/* ---- LU form of the BSE, batched over instances of uneven size -------------
 * No counterpart in the reference (its BSE is the damped two-ordering update,
 * SRC/parquet_BSE.f90:72-128, whose fixed point this reproduces):
 *   F_i = (1 - scale_i Gamma_i chi_i)^{-1} Gamma_i   (want_phi: F_i - Gamma_i)
 * for n_inst instances of size n[i] = nl[i] * Nnu_i, in one persistent launch
 * (CTAs take instances largest first; partial-pivoting LU, panel 32, FP64
 * tensor-core trailing updates; n[i] right-hand sides).  n, nl, scale: host
 * arrays.  gamma, out, work: device, instances packed consecutively as
 * (n, n) column-major complex128; chi: device, packed (nl, nl, Nnu) blocks;
 * ipiv: device int, packed n[i].  status (host, optional): per instance 0, or
 * k+1 when column k had a zero pivot; when given, the call synchronises.
 * Allocates nothing; limit n_inst <= 16384. */
int tups_bse_lu_batched(int n_inst, const int* n, const int* nl, const double* scale, const double* gamma,
                        const double* chi, double* out, double* work, int* ipiv, int want_phi, int* status,
                        void* stream);

/* ---- LU form in split precision with FP64 iterative refinement ---------------
 * No counterpart in the reference (see tups_bse_lu_batched).  The same
 * F_i = (1 - scale_i Gamma_i chi_i)^{-1} Gamma_i (want_phi: F_i - Gamma_i)
 * with the arithmetic split: instances grouped by size; blocked LU with
 * partial pivoting whose 128-column panels are factored in FP64 and whose
 * trailing updates, like the off-diagonal updates of the triangular solves,
 * run on the int8 tensor cores with `slices` (2..8) int8 slices per operand
 * (error about 10^(1.1 - 2 slices) of the update's norm); then iterative
 * refinement: the residual R = Gamma - A X in FP64 (FP64 tensor cores) and,
 * until max|R| <= tol max|Gamma| for every instance of a size group or after
 * max_refine corrections, X += U^{-1} L^{-1} P R.  refinements and residual
 * (host, optional, n_inst entries): corrections applied and the final
 * max|R|/max|Gamma| of each instance; status as in tups_bse_lu_batched.  work: device buffer of tups_bse_lu_split_workspace()
 * bytes (the largest size group's five n x n matrices per instance, pivots and
 * the split-GEMM slices).  Synchronises the stream once per refinement step;
 * TUPS_ERR_TIMEOUT when a bounded wait of the int8 GEMM ran out. */
size_t tups_bse_lu_split_workspace(int n_inst, const int* n, int slices);
int tups_bse_lu_split_batched(int n_inst, const int* n, const int* nl, const double* scale, const double* gamma,
                              const double* chi, double* out, int want_phi, int slices, double tol, int max_refine,
                              void* work, size_t work_bytes, int* refinements, double* residual, int* status,
                              void* stream);

/* ---- BSE update without device allocation ----------------------------------
 * No counterpart in the reference.  For callers that may not allocate device
 * memory while they call this library (a host that gives all device memory
 * to its own arena at start-up, or a loop that must not trigger the implicit
 * synchronisation of cudaMalloc/cudaFree): the same update as BSE(ite) for
 * n_inst (q, channel) instances that the caller owns on the device,
 *   Phi = scale [(Gamma chi) F + F (chi Gamma)] + (1 - f_damping)(F - Gamma),
 * written over Gamma.  gamma_phi, F: n_inst consecutive (Nz, Nz) column-major
 * complex128 matrices; chi: n_inst consecutive (Nl, Nl, Nf) nu-diagonal blocks
 * (chi_LL[(l1,nu),(l2,nu)] at l1 + Nl*(l2 + Nl*nu)); scale = c_r f/(beta Nx Ny)
 * (c = 1/2, 1/2, -1/4, 1/4 for d, m, s, t); stream: a cudaStream_t or NULL.
 * Limit: Nz <= 1024.  The scratch is a fixed 32 MiB static device array that
 * every GPU loading the library holds until exit; the first call on a device
 * looks up its address (make it before any stream capture) and keeps it for
 * the life of the process, so do not call this on a device again after a
 * cudaDeviceReset of it; calls that overlap on the GPU race on it.  Allocates
 * nothing; returns after queueing. */
int tups_bse_noalloc(int n_inst, int Nz, int Nf, int Nl, double* gamma_phi, const double* F, const double* chi,
                     double scale, double f_damping, void* stream);

/* ---- instrumentation (the per-phase timings of SRC/loop.f90:64-178, taken
 * with CUDA events on the library's stream) ---------------------------------- */
#define TUPS_PHASE_GREEN 0     /* calc_Gkw_Grt */
#define TUPS_PHASE_CHI 1       /* calc_chi (all slots) */
#define TUPS_PHASE_BSE_PREP 2  /* Gamma chi, chi Gamma */
#define TUPS_PHASE_BSE_GEMM 3  /* the K = 2 Nz tensor-core GEMM */
#define TUPS_PHASE_PHIR 4      /* calc_PhiR */
#define TUPS_PHASE_M 5         /* calc_M_* */
#define TUPS_PHASE_PAE 6       /* calculate_PAE */
#define TUPS_PHASE_SDE 7       /* calc_SDE */
#define TUPS_PHASE_CONV 8      /* conv */
#define TUPS_PHASE_UPDATE 9    /* vertex update */
#define TUPS_NPHASE 10
/* enable (1) / disable (0) phase timing; enabling clears the accumulators */
int tups_set_timing(tups_ctx* ctx, int enable);
/* milliseconds accumulated per phase since timing was enabled, and the
 * number of timed launches of each (each array TUPS_NPHASE long; NULL ok) */
int tups_get_phase_times(tups_ctx* ctx, double* ms, int* count);
/* record a CUDA event on the library's stream in slot 0..7 */
int tups_record_event(tups_ctx* ctx, int slot);
/* milliseconds between two recorded slots (synchronizes on the later one) */
int tups_event_elapsed(tups_ctx* ctx, int slot_a, int slot_b, double* ms);

#ifdef __cplusplus
}
#endif
#endif /* TUPS_B200_H */
