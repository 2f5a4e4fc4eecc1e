// Internal declarations shared by the host runtime and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/tups_b200.h"

namespace tups {

constexpr int NS = 8;  // point-group operations of the square lattice

// complex128 as interleaved doubles on the device
typedef double2 cplx;

struct DeviceTables {
  double* FF = nullptr;       // (Nx, Ny, Nl) column-major
  double* FF_inv = nullptr;   // (8, Nx, Ny, Nl)
  double* Ek = nullptr;       // (Nx, Ny)
  double* Ekg = nullptr;      // (Ng, Ng, Nx, Ny)
  int* signs = nullptr;       // (Nl)
  int* lsym = nullptr;        // (8, Nl), 0-based target l
  double* lfac = nullptr;     // (8, Nl)
  int* ibz = nullptr;         // (Nred, 3): qx, qy, w (1-based)
  int* symlist = nullptr;     // (NIBZ, 8) 0/1
  int* symq = nullptr;        // (NIBZ, 8, 2): S(q) 1-based (qx, qy)
  cplx* L[4] = {};            // Lambda_r (Nf, Nf, Nf/2)
  cplx* expSqR = nullptr;     // (NIBZ, NR, 8)
  cplx* expqSR = nullptr;     // (Nc, NR, 8), k index (ky-1)*Nx+kx
  cplx* tw_tau = nullptr;     // (Nf tau, Nf nu) e^{-i nu_n tau_i}
  cplx* tw_x = nullptr;       // (Nx*Ng) e^{-2 pi i m / n1}
  cplx* tw_y = nullptr;       // (Ny*Ng)
  int4* pae_elems = nullptr;  // crossing: elements per (pair, family, W), see pae.cu
  int* pae_counts = nullptr;
};

struct DeviceState {
  cplx* Sigma = nullptr;      // (Nt)
  cplx* SigmaOld = nullptr;   // (Nt)
  cplx* SigmaH = nullptr;     // (Nx, Ny)
  cplx* Gkw = nullptr;        // (Nt)
  cplx* Grt = nullptr;        // (Nx*Ng, Ny*Ng, Nf)
  cplx* Grt_work = nullptr;   // same size, FFT scratch
  cplx* F[4] = {};            // (Nz, Nz, Nb)
  cplx* G[4] = {};            // (Nz, Nz, Nb)
  cplx* chi_ph = nullptr;     // (Nl, Nl, Nf, Nb) nu-diagonal blocks of chi_ph_LL
  cplx* chi_pp = nullptr;
  cplx* bse_A = nullptr;      // BSE scratch: Gamma*chi per instance of a chunk
  cplx* bse_B = nullptr;      // chi*Gamma
  size_t bse_chunk = 0;       // instances per chunk
  cplx* PhiR[4] = {};         // (Nz*Nz, Nf/2, NR)
  cplx* M[4] = {};            // (Nl^4, NIBZ, NR): 0 phbar_to_ph 1 pp_to_ph 2 ph_to_pp 3 phbar_to_pp
  cplx* chi_aux_ph = nullptr; // (Nl*nbox, Nb)
  cplx* chi_aux_pp = nullptr;
  cplx* LChi = nullptr;       // (Nb, Nz): slot fastest
  cplx* PhChi = nullptr;
  cplx* PPChi = nullptr;
  cplx* SigmaV = nullptr;     // (NIBZ*Nf)
  cplx* order2 = nullptr;     // (Nt)
  cplx* GGG = nullptr;        // (Nx*Ng, Ny*Ng, Nf) U^2 term after the FFT
  double* scal = nullptr;     // device scalars, see Scal
  double* red = nullptr;      // reduction scratch
};

// buffers of the every-5-iterations readout, allocated on its first use
struct ReadoutBufs {
  bool ready = false;
  double* sd = nullptr;     // FF_sdwave (Nx*Ny, 4), k = kx*Ny + ky
  double* sd2 = nullptr;    // its square
  cplx* pre = nullptr;      // pre-FFT G(k, tau) (n1, n2, Nf)
  cplx* ffg_in = nullptr;   // 4 x (n1, n2, Nf)
  cplx* ffg = nullptr;      // 4 x (n1, n2, Nf)
  cplx* prod = nullptr;     // 10 x (n1, n2, Nf)
  cplx* prod_ft = nullptr;  // 10 x (n1, n2, Nf)
  cplx* chi0 = nullptr;     // 10 x (Nred): ph, pp, ph_FF[4], pp_FF[4]
  cplx* chi0_bz = nullptr;  // 10 x (Nx*Ny*Nf/2)
  cplx* gph = nullptr;      // (Nl*nbox, Nb, 4)
  cplx* gpp = nullptr;
  cplx* sus = nullptr;      // (Nb, 4 ff, 4 channels)
  cplx* sus_bz = nullptr;   // 16 x (Nx*Ny*Nf/2)
};

// slots of DeviceState::scal
enum Scal {
  S_MU = 0,         // chemical potential
  S_T1 = 1,         // last particle number estimate
  S_STEPS = 2,      // bisection steps of the last calc_Gkw_Grt
  S_STATUS = 3,     // 0 ok, else a TUPS_ERR_* code set by a device routine
  S_RELSIG = 4,     // conv: max relative Sigma change
  S_RELSIGAV = 5,   // conv: |sum rel| / Nt
  S_DSIG = 6,       // conv: max |dSigma|
  S_FMAX = 7,       // conv: max|F_r|, 4 slots (7..10)
  S_NANFLAG = 11,   // conv: NaN/Inf seen
  S_SIGMAX = 12,    // conv: max |Sigma|
  S_COUNT = 16
};

}  // namespace tups

struct tups_ctx {
  tups_params p{};
  tups_dims d{};
  int device = 0;
  // slot sharding: this context holds global slots [slot0, slot0 + d.Nb)
  int rank = 0, ntasks = 1, slot0 = 0;
  tups_exchange_fn xfn = nullptr;
  void* xuser = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;
  // host tables
  std::vector<int> pick, bonds0, signs, reps, lsym, ibz, symlist, symq;
  std::vector<double> FF, FF_inv, lfac, Ek, Ekg;
  double aux = 1.0;         // 1/FF(1,1,1)^2
  // host copies of small state
  double F_max_prev[4] = {0, 0, 0, 0};
  bool have_exp = false, have_M = false, have_phir = false, have_green = false;
  int pae_max_tiles[2] = {0, 0};  // longest element list of each family
  tups::DeviceTables t;
  tups::DeviceState s;
  tups::ReadoutBufs rd;
  // warm start (LU workspace) and checkpoint, allocated on first use
  tups::cplx* lu_work = nullptr;
  int* lu_ipiv = nullptr;
  tups::cplx* ck_F[4] = {};
  tups::cplx* ck_G[4] = {};
  tups::cplx* ck_sigma = nullptr;
  tups::cplx* ck_sigma_old = nullptr;
  // split-precision BSE: slices per operand (0 = FP64 tensor cores), the
  // residual-driven ladder, and the int8 workspace (allocated on first use)
  int bse_slices = 0;
  bool precision_ladder = false;
  double last_dsigma_rel = -1.0;
  void* oz_work = nullptr;
  size_t oz_cap = 0;           // instances per split sub-chunk
  // slices of the BSE in flight, and the online tuner of the ladder: device
  // milliseconds of a whole BSE call (chi, prep, GEMM) per choice
  int cur_slices = 0;
  int tune_pending = -1;       // choice whose timing events are in flight
  cudaEvent_t tune_ev[2] = {nullptr, nullptr};
  double tune_ms[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};  // [0] FP64, [s] s slices
  // CUDA-graph iterations: one executable graph per (slices, SDE) choice;
  // in graph mode the tuner compares whole-iteration times (tune_graph_ms)
  bool use_graph = false;
  bool capturing = false;
  // tile-shape tuner (tune.cu): on by default, TUPS_AUTOTUNE=0 turns it off;
  // tile_tunings counts the tunings run by this context
  bool autotune = true;
  int pae_products = 3;        // real DMMA products per complex one in the crossing GEMM (3 or 4)
  long long tile_tunings = 0;
  cudaGraphExec_t graph_exec[18] = {};
  // second stream of a captured iteration: the SDE runs on it beside
  // Phi(R) and the crossing (created before the first capture)
  cudaStream_t side_stream = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  long long graph_launches[18] = {};
  double tune_graph_ms[9] = {-1, -1, -1, -1, -1, -1, -1, -1, -1};
  double ck_scal[16] = {};
  double ck_fmax[4] = {};
  bool ck_valid = false;
  std::vector<void*> allocations;
  // instrumentation: event pairs per phase, reused across calls
  bool timing = false;
  std::vector<cudaEvent_t> ev_begin[TUPS_NPHASE], ev_end[TUPS_NPHASE];
  int ev_used[TUPS_NPHASE] = {};
  double phase_ms[TUPS_NPHASE] = {};
  int phase_count[TUPS_NPHASE] = {};
  cudaEvent_t marks[8] = {};
};

namespace tups {
// bracket a phase with CUDA events on the library's stream when timing is on
void phase_begin(tups_ctx* ctx, int phase);
void phase_end(tups_ctx* ctx, int phase);
// fold recorded event pairs into phase_ms (synchronizes the stream)
void phase_collect(tups_ctx* ctx);
}  // namespace tups

namespace tups {

// ---- split-precision (int8 slice) complex GEMM, ozaki.cu ----
struct OzOperand {
  const cplx* p1;
  const cplx* p2;
  long long s1, s2;   // element strides between instances (ignored for BSE parts)
  int ld1, ld2;       // leading dimensions (column-major)
  int K1, K2;         // complex lengths of the two parts along K
  int bse2;           // 1: part 2 is F_r(q) of the BSE chunk (instance = 4 (q - q_begin) + r)
  int bse1;           // 1: part 1 is F_r(q)
  const cplx* F[4];
  int q_begin, Nz;
};

struct OzWork {
  int Kpad = 0;
  size_t a_bytes = 0, b_bytes = 0, rs_bytes = 0, cs_bytes = 0, acc_bytes = 0, total = 0;
};

struct OzRun {
  int batch = 0, M = 0, N = 0, s = 0;
  OzOperand A{}, B{};
  int8_t* a_slices = nullptr;
  int8_t* b_slices = nullptr;
  double* rscale = nullptr;
  double* cscale = nullptr;
  double* acc = nullptr;
  double* status = nullptr;   // receives status_code when a wait times out
  double status_code = 0.0;
  int epi = 0;         // 0: C = A B; 1: BSE update written over G; 2: C -= A B
  cplx* C = nullptr;
  int ldc = 0;              // epi 2: leading dimension of C and the complex
  long long c_stride = 0;   // stride between instances
  cplx* F[4] = {};
  cplx* G[4] = {};
  double scale[4] = {};
  double omf = 0.0;
  int q_begin = 0;
};

OzWork oz_work_layout(int batch, int M, int N, int K, int s);
// carve the workspace of oz_work_layout out of `base` into R
void oz_bind_work(OzRun& R, const OzWork& w, void* base);
int oz_run(OzRun& R, cudaStream_t stream, long long* launches);

int set_error(tups_ctx* ctx, int code, const std::string& msg);

// tile-shape tuner, tune.cu: process-wide choices keyed by kernel and shape
bool tune_get(const std::string& key, int* choice);
// index in names of the candidate fixed by tups_set_tuning for key, or -1
int tune_forced(const std::string& key, const std::vector<std::string>& names);
// false when the context has tuning off or its stream is being captured
bool tune_allowed(tups_ctx* ctx);
// time run(c) for c = 0..n_cand-1 (best of reps, CUDA events on the
// context's stream), store and return the fastest in *choice
int tune_pick(tups_ctx* ctx, const std::string& key, int n_cand, const std::vector<std::string>& names,
              const std::function<int(int)>& run, int reps, int* choice);
// sharded contexts: combine n doubles at device address dev over the ranks
// (no-op unsharded); synchronises the stream first
int exchange(tups_ctx* ctx, int what, double* dev, size_t n, int op);
// the ibz rows of this context's slots (local slot q -> global slot slot0 + q)
inline const int* ibz_local(const tups_ctx* ctx) { return ctx->t.ibz + 3 * (size_t)ctx->slot0; }
int cuda_check(tups_ctx* ctx, cudaError_t e, const char* what);
// record a kernel launch and check for launch errors
int after_launch(tups_ctx* ctx, const char* name);

// kernel drivers (each returns TUPS_OK or an error code)
int launch_sigma_hartree(tups_ctx* ctx);
int launch_bisection(tups_ctx* ctx, int cal_chi, int max_steps);
int launch_grt(tups_ctx* ctx);
int launch_gkw(tups_ctx* ctx);
int launch_chi(tups_ctx* ctx, int q_begin, int q_count);
int launch_bse_chunk(tups_ctx* ctx, int q_begin, int q_count);
// slices the next BSE call will use (0 = FP64), see bse.cu
int current_bse_slices(const tups_ctx* ctx);
// fold a finished BSE timing into the tuner (after the stream synchronised)
void bse_tune_collect(tups_ctx* ctx);
int launch_phir(tups_ctx* ctx);
int launch_M(tups_ctx* ctx, int which);
int launch_pae(tups_ctx* ctx);
int launch_sde(tups_ctx* ctx);
int launch_conv(tups_ctx* ctx);
int launch_vertex_update(tups_ctx* ctx);
// k_conv_sigma alone, and the vertex update fused with max|F_r| (the rest
// of launch_conv), for an iteration that runs both back to back
int launch_conv_sigma(tups_ctx* ctx);
int launch_vertex_update_fmax(tups_ctx* ctx);
int launch_output_mu(tups_ctx* ctx);
int launch_fft2d(tups_ctx* ctx, const cplx* in, cplx* out, int forward);
int launch_chi_aux(tups_ctx* ctx);
int launch_fill_lambda_block(tups_ctx* ctx, cplx* F, cplx* G, const cplx* L, double aux);
int launch_grt_pre(tups_ctx* ctx, cplx* out);
int launch_fft2d_batch(tups_ctx* ctx, const cplx* in, cplx* out, int nslices, int forward);
int launch_readout(tups_ctx* ctx);
int launch_set_l1_block(tups_ctx* ctx, cplx* G, double vr, double vi);

}  // namespace tups
