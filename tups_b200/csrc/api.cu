// C-ABI entry points: one per Fortran routine of the hot path, operating on
// the device-resident state of a context, plus the loop of SRC/loop.f90.
#include <cmath>
#include <cstring>
#include <vector>

#include "tups_internal.h"

using tups::cplx;

#define TRY(x)                      \
  do {                              \
    int _rc = (x);                  \
    if (_rc != TUPS_OK) return _rc; \
  } while (0)

namespace {

constexpr int kMuMaxSteps = 200;  // the reference's bisection has no cap

int set_dev(tups_ctx* ctx) { return tups::cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice"); }

int read_scalars(tups_ctx* ctx, double* out) {
  TRY(tups::cuda_check(ctx,
                       cudaMemcpyAsync(out, ctx->s.scal, tups::S_COUNT * sizeof(double), cudaMemcpyDeviceToHost,
                                       ctx->stream),
                       "read scalars"));
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

// surface a status left by a device routine (bisection cap) and clear it
int device_status(tups_ctx* ctx) {
  double sc[tups::S_COUNT];
  TRY(read_scalars(ctx, sc));
  int st = (int)sc[tups::S_STATUS];
  if (st != 0) {
    double z = 0.0;
    cudaMemcpy(ctx->s.scal + tups::S_STATUS, &z, sizeof(double), cudaMemcpyHostToDevice);
    if (st == TUPS_ERR_MU_NOCONV)
      return tups::set_error(ctx, st, "mu bisection exceeded " + std::to_string(kMuMaxSteps) + " steps");
    return tups::set_error(ctx, st, "device routine reported an error");
  }
  return TUPS_OK;
}

int copy_d2h(tups_ctx* ctx, void* host, const void* dev, size_t bytes) {
  if (!host) return tups::set_error(ctx, TUPS_ERR_BADARG, "NULL host buffer");
  TRY(tups::cuda_check(ctx, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream), "D2H"));
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

int copy_h2d(tups_ctx* ctx, void* dev, const void* host, size_t bytes) {
  if (!host) return tups::set_error(ctx, TUPS_ERR_BADARG, "NULL host buffer");
  TRY(tups::cuda_check(ctx, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream), "H2D"));
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

int green_async(tups_ctx* ctx, int cal_chi) {
  tups::phase_begin(ctx, TUPS_PHASE_GREEN);
  TRY(tups::launch_sigma_hartree(ctx));
  TRY(tups::launch_bisection(ctx, cal_chi, kMuMaxSteps));
  TRY(tups::launch_grt(ctx));
  TRY(tups::launch_gkw(ctx));
  tups::phase_end(ctx, TUPS_PHASE_GREEN);
  ctx->have_green = true;
  return TUPS_OK;
}

int bse_async(tups_ctx* ctx, int slices = -1) {
  if (!ctx->have_green) return tups::set_error(ctx, TUPS_ERR_STATE, "BSE before calc_Gkw_Grt");
  const int Nb = ctx->d.Nb;
  ctx->cur_slices = slices >= 0 ? slices : tups::current_bse_slices(ctx);
  // the tuner times whole BSE calls outside graphs; graph mode times the graph
  const bool tune = ctx->precision_ladder && !ctx->capturing && !ctx->use_graph;
  if (tune) {
    for (int i = 0; i < 2; i++)
      if (!ctx->tune_ev[i]) TRY(tups::cuda_check(ctx, cudaEventCreate(&ctx->tune_ev[i]), "event"));
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->tune_ev[0], ctx->stream), "event"));
  }
  const long long tunings = ctx->tile_tunings;
  const int chunk_q = (int)std::max<size_t>(1, ctx->s.bse_chunk / 4);
  for (int q0 = 0; q0 < Nb; q0 += chunk_q) {
    const int nq = std::min(chunk_q, Nb - q0);
    tups::phase_begin(ctx, TUPS_PHASE_CHI);
    TRY(tups::launch_chi(ctx, q0, nq));
    tups::phase_end(ctx, TUPS_PHASE_CHI);
    TRY(tups::launch_bse_chunk(ctx, q0, nq));
  }
  // a call that also timed tile shapes is no measure of the BSE itself
  if (tune && ctx->tile_tunings == tunings) {
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->tune_ev[1], ctx->stream), "event"));
    ctx->tune_pending = ctx->cur_slices;
  }
  return TUPS_OK;
}

int sde_async(tups_ctx* ctx) {
  if (!ctx->have_green) return tups::set_error(ctx, TUPS_ERR_STATE, "calc_SDE before calc_Gkw_Grt");
  const size_t bytes = (size_t)ctx->d.Nt * sizeof(cplx);
  TRY(tups::cuda_check(ctx,
                       cudaMemcpyAsync(ctx->s.SigmaOld, ctx->s.Sigma, bytes, cudaMemcpyDeviceToDevice, ctx->stream),
                       "SigmaOld = Sigma"));
  tups::phase_begin(ctx, TUPS_PHASE_SDE);
  TRY(tups::launch_sde(ctx));
  tups::phase_end(ctx, TUPS_PHASE_SDE);
  return TUPS_OK;
}

}  // namespace

extern "C" int tups_calc_Gkw_Grt(tups_ctx* ctx, int ite, int cal_chi) {
  (void)ite;
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  TRY(green_async(ctx, cal_chi));
  return device_status(ctx);
}

extern "C" int tups_calc_chi(tups_ctx* ctx, int idx_q, double* chi_ph_LL, double* chi_pp_LL) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  if (idx_q < 1 || idx_q > d.Nb) return tups::set_error(ctx, TUPS_ERR_BADARG, "idx_q out of range");
  if (!ctx->have_green) return tups::set_error(ctx, TUPS_ERR_STATE, "calc_chi before calc_Gkw_Grt");
  TRY(set_dev(ctx));
  TRY(tups::launch_chi(ctx, idx_q - 1, 1));
  const size_t nb = (size_t)d.Nl * d.Nl * d.Nf;
  std::vector<cplx> ph(nb), pp(nb);
  TRY(copy_d2h(ctx, ph.data(), ctx->s.chi_ph + nb * (idx_q - 1), nb * sizeof(cplx)));
  TRY(copy_d2h(ctx, pp.data(), ctx->s.chi_pp + nb * (idx_q - 1), nb * sizeof(cplx)));
  const size_t Nz = d.Nz;
  for (int which = 0; which < 2; which++) {
    double* out = which == 0 ? chi_ph_LL : chi_pp_LL;
    if (!out) continue;
    const std::vector<cplx>& src = which == 0 ? ph : pp;
    std::memset(out, 0, 2 * Nz * Nz * sizeof(double));
    for (int nu = 0; nu < d.Nf; nu++)
      for (int l2 = 0; l2 < d.Nl; l2++)
        for (int l1 = 0; l1 < d.Nl; l1++) {
          const cplx v = src[l1 + (size_t)d.Nl * (l2 + (size_t)d.Nl * nu)];
          const size_t o = (size_t)(l1 * d.Nf + nu) + Nz * (size_t)(l2 * d.Nf + nu);
          out[2 * o] = v.x;
          out[2 * o + 1] = v.y;
        }
  }
  return TUPS_OK;
}

extern "C" int tups_BSE(tups_ctx* ctx, int ite) {
  (void)ite;
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  TRY(bse_async(ctx));
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "BSE");
}

extern "C" int tups_calc_PhiR(tups_ctx* ctx, int ite) {
  (void)ite;
  if (!ctx) return TUPS_ERR_BADARG;
  if (!ctx->have_exp) return tups::set_error(ctx, TUPS_ERR_STATE, "calc_PhiR before calculate_expSqR");
  TRY(set_dev(ctx));
  tups::phase_begin(ctx, TUPS_PHASE_PHIR);
  TRY(tups::launch_phir(ctx));
  tups::phase_end(ctx, TUPS_PHASE_PHIR);
  ctx->have_phir = true;
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "calc_PhiR");
}

static int calc_M(tups_ctx* ctx, int which) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  tups::phase_begin(ctx, TUPS_PHASE_M);
  TRY(tups::launch_M(ctx, which));
  tups::phase_end(ctx, TUPS_PHASE_M);
  ctx->have_M = true;
  return TUPS_OK;
}
extern "C" int tups_calc_M_phbar_to_ph(tups_ctx* ctx) { return calc_M(ctx, 0); }
extern "C" int tups_calc_M_pp_to_ph(tups_ctx* ctx) { return calc_M(ctx, 1); }
extern "C" int tups_calc_M_ph_to_pp(tups_ctx* ctx) { return calc_M(ctx, 2); }
extern "C" int tups_calc_M_phbar_to_pp(tups_ctx* ctx) { return calc_M(ctx, 3); }

extern "C" int tups_calculate_PAE(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (!ctx->have_M || !ctx->have_phir)
    return tups::set_error(ctx, TUPS_ERR_STATE, "calculate_PAE before calc_PhiR / calc_M_*");
  TRY(set_dev(ctx));
  tups::phase_begin(ctx, TUPS_PHASE_PAE);
  TRY(tups::launch_pae(ctx));
  tups::phase_end(ctx, TUPS_PHASE_PAE);
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "calculate_PAE");
}

extern "C" int tups_calc_SDE(tups_ctx* ctx, int ite) {
  (void)ite;
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  TRY(sde_async(ctx));
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "calc_SDE");
}

// conv()'s host decision from the device scalars (SRC/parquet_check.f90:39-150)
static int conv_finish(tups_ctx* ctx, const double* sc, tups_conv_info* info) {
  tups_conv_info ci;
  std::memset(&ci, 0, sizeof(ci));
  ci.rel_sig_max = sc[tups::S_RELSIG];
  ci.rel_sig_av = sc[tups::S_RELSIGAV];
  ci.dsigma_inf = sc[tups::S_DSIG];
  ci.mu = sc[tups::S_MU];
  ci.bisection_steps = (int)sc[tups::S_STEPS];
  // f_sigma = f_vert = real(1e-8, 8) (SRC/parquet_ini.f90:31-32)
  const double f_tol = (double)1e-8f;
  bool ok = ci.rel_sig_max < f_tol;
  for (int r = 0; r < 4; r++) {
    ci.F_max[r] = sc[tups::S_FMAX + r];
    const double prev = ctx->F_max_prev[r];
    ci.rel_err[r] = prev != 0.0 ? std::fabs(1.0 - ci.F_max[r] / prev) : INFINITY;
    ok = ok && ci.rel_err[r] < f_tol;
    ctx->F_max_prev[r] = ci.F_max[r];
  }
  if (ctx->p.conv_abs > 0.0) ok = ci.dsigma_inf < ctx->p.conv_abs;
  ci.converged = ok ? 1 : 0;
  ctx->last_dsigma_rel = sc[tups::S_SIGMAX] > 0.0 ? ci.dsigma_inf / sc[tups::S_SIGMAX] : -1.0;
  tups::bse_tune_collect(ctx);  // the caller synchronised the stream
  if (info) *info = ci;
  if (sc[tups::S_NANFLAG] > 0.0 || !std::isfinite(ci.rel_sig_max))
    return tups::set_error(ctx, TUPS_ERR_NAN, "NaN or Inf in the self-energy or a vertex");
  return TUPS_OK;
}

static int copy_sigma_old(tups_ctx* ctx) {
  const size_t bytes = (size_t)ctx->d.Nt * sizeof(cplx);
  return tups::cuda_check(
      ctx, cudaMemcpyAsync(ctx->s.SigmaOld, ctx->s.Sigma, bytes, cudaMemcpyDeviceToDevice, ctx->stream),
      "SigmaOld = Sigma");
}

extern "C" int tups_conv(tups_ctx* ctx, tups_conv_info* info) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  tups::phase_begin(ctx, TUPS_PHASE_CONV);
  TRY(tups::launch_conv(ctx));
  tups::phase_end(ctx, TUPS_PHASE_CONV);
  double sc[tups::S_COUNT];
  TRY(read_scalars(ctx, sc));
  tups_conv_info ci;
  const int rc = conv_finish(ctx, sc, &ci);
  TRY(copy_sigma_old(ctx));
  if (info) *info = ci;
  return rc;
}

extern "C" int tups_vertex_update(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  tups::phase_begin(ctx, TUPS_PHASE_UPDATE);
  TRY(tups::launch_vertex_update(ctx));
  tups::phase_end(ctx, TUPS_PHASE_UPDATE);
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "vertex update");
}

extern "C" int tups_output_block(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  return tups::launch_output_mu(ctx);
}

// buffers of the readout, on first use
static int ensure_readout(tups_ctx* ctx) {
  auto& rd = ctx->rd;
  if (rd.ready) return TUPS_OK;
  const auto& d = ctx->d;
  const size_t ng = (size_t)d.Nx * d.Ngrain * d.Ny * d.Ngrain * d.Nf;
  const size_t nh = d.Nf / 2, nbz = (size_t)d.Nc * nh;
  auto alloc = [&](void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return tups::set_error(ctx, TUPS_ERR_OOM, "readout buffers");
    }
    ctx->allocations.push_back(*p);
    return TUPS_OK;
  };
  TRY(alloc((void**)&rd.sd, 4 * (size_t)d.Nc * sizeof(double)));
  TRY(alloc((void**)&rd.sd2, 4 * (size_t)d.Nc * sizeof(double)));
  TRY(alloc((void**)&rd.pre, ng * sizeof(cplx)));
  TRY(alloc((void**)&rd.ffg_in, 4 * ng * sizeof(cplx)));
  TRY(alloc((void**)&rd.ffg, 4 * ng * sizeof(cplx)));
  TRY(alloc((void**)&rd.prod, 10 * ng * sizeof(cplx)));
  TRY(alloc((void**)&rd.prod_ft, 10 * ng * sizeof(cplx)));
  TRY(alloc((void**)&rd.chi0, 10 * (size_t)d.Nred * sizeof(cplx)));
  TRY(alloc((void**)&rd.chi0_bz, 10 * nbz * sizeof(cplx)));
  TRY(alloc((void**)&rd.gph, 4 * (size_t)d.Nl * d.nbox * d.Nb * sizeof(cplx)));
  TRY(alloc((void**)&rd.gpp, 4 * (size_t)d.Nl * d.nbox * d.Nb * sizeof(cplx)));
  TRY(alloc((void**)&rd.sus, 16 * (size_t)d.Nb * sizeof(cplx)));
  TRY(alloc((void**)&rd.sus_bz, 16 * nbz * sizeof(cplx)));
  // fill_FF_sdwave (SRC/parquet_formfactors.f90:792-816), k = (kx-1)*Ny + ky-1
  std::vector<double> sd(4 * (size_t)d.Nc), sd2(4 * (size_t)d.Nc);
  for (int kx = 1; kx <= d.Nx; kx++)
    for (int ky = 1; ky <= d.Ny; ky++) {
      const double px = 2.0 / d.Nx * M_PI * (kx - 1), py = 2.0 / d.Ny * M_PI * (ky - 1);
      const double v[4] = {1.0, std::cos(px) - std::cos(py), std::sin(px), std::sin(px) * std::sin(py)};
      const size_t k = (size_t)(kx - 1) * d.Ny + (ky - 1);
      for (int f = 0; f < 4; f++) {
        sd[k + (size_t)d.Nc * f] = v[f];
        sd2[k + (size_t)d.Nc * f] = v[f] * v[f];
      }
    }
  TRY(copy_h2d(ctx, rd.sd, sd.data(), sd.size() * sizeof(double)));
  TRY(copy_h2d(ctx, rd.sd2, sd2.data(), sd2.size() * sizeof(double)));
  rd.ready = true;
  return TUPS_OK;
}

static int readout_async(tups_ctx* ctx) {
  TRY(ensure_readout(ctx));
  TRY(green_async(ctx, 1));
  return tups::launch_readout(ctx);
}

extern "C" int tups_readout(tups_ctx* ctx, int ite) {
  (void)ite;
  if (!ctx) return TUPS_ERR_BADARG;
  if (ctx->ntasks > 1) return tups::set_error(ctx, TUPS_ERR_STATE, "the readout needs every slot: use an unsharded context");
  TRY(set_dev(ctx));
  TRY(readout_async(ctx));
  TRY(device_status(ctx));
  return TUPS_OK;
}

extern "C" int tups_get_chi0(tups_ctx* ctx, int bz, double* ph, double* pp, double* ph_FF, double* pp_FF) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (!ctx->rd.ready) return tups::set_error(ctx, TUPS_ERR_STATE, "no readout yet");
  const size_t n = bz ? (size_t)ctx->d.Nc * (ctx->d.Nf / 2) : (size_t)ctx->d.Nred;
  const cplx* base = bz ? ctx->rd.chi0_bz : ctx->rd.chi0;
  if (ph) TRY(copy_d2h(ctx, ph, base, n * sizeof(cplx)));
  if (pp) TRY(copy_d2h(ctx, pp, base + n, n * sizeof(cplx)));
  if (ph_FF) TRY(copy_d2h(ctx, ph_FF, base + 2 * n, 4 * n * sizeof(cplx)));
  if (pp_FF) TRY(copy_d2h(ctx, pp_FF, base + 6 * n, 4 * n * sizeof(cplx)));
  return TUPS_OK;
}

extern "C" int tups_get_sus(tups_ctx* ctx, int channel, int bz, double* host) {
  if (!ctx || channel < 0 || channel > 3) return TUPS_ERR_BADARG;
  if (!ctx->rd.ready) return tups::set_error(ctx, TUPS_ERR_STATE, "no readout yet");
  const size_t n = bz ? (size_t)ctx->d.Nc * (ctx->d.Nf / 2) : (size_t)ctx->d.Nb;
  const cplx* base = bz ? ctx->rd.sus_bz : ctx->rd.sus;
  return copy_d2h(ctx, host, base + 4 * n * channel, 4 * n * sizeof(cplx));
}

static int iteration_impl(tups_ctx* ctx, int ite, tups_conv_info* info, bool with_readout);
static int iteration_graph(tups_ctx* ctx, int ite, tups_conv_info* info);

extern "C" int tups_iteration(tups_ctx* ctx, int ite, tups_conv_info* info) {
  // a sharded context calls the host exchange inside the iteration, which a
  // graph cannot hold
  if (ctx && ctx->use_graph && ite > 0 && ctx->have_exp && ctx->have_M && !ctx->timing && ctx->ntasks == 1)
    return iteration_graph(ctx, ite, info);
  return iteration_impl(ctx, ite, info, false);
}

// The device work of one iteration with no host synchronisation: Green's
// function, BSE, Phi(R), parquet equation, SDE, the conv kernels,
// SigmaOld = Sigma and the vertex update.  The output block only moves mu
// and does not touch the vertices, so it follows the update on the host;
// the update does not change F, so max|F_r| is taken in the update's own
// pass over F.  The SDE reads Phi (the BSE's output), the Green's function
// and the bubbles and writes only its own arrays and Sigma, none of which
// Phi(R) or the crossing read or write, so with a side stream it runs there
// beside them (its small kernels fill SMs the crossing's tail leaves idle)
// and joins before the conv kernels.
static int iteration_device(tups_ctx* ctx, int slices, bool do_sde) {
  TRY(green_async(ctx, 0));
  TRY(bse_async(ctx, slices));
  const bool fork = do_sde && ctx->side_stream && ctx->fork_ev && ctx->join_ev;
  if (fork) {
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->fork_ev, ctx->stream), "fork"));
    TRY(tups::cuda_check(ctx, cudaStreamWaitEvent(ctx->side_stream, ctx->fork_ev, 0), "fork"));
    cudaStream_t main = ctx->stream;
    ctx->stream = ctx->side_stream;
    const int rc = sde_async(ctx);
    ctx->stream = main;
    TRY(rc);
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->join_ev, ctx->side_stream), "join"));
  }
  TRY(tups::launch_phir(ctx));
  TRY(tups::launch_pae(ctx));
  if (do_sde && !fork) TRY(sde_async(ctx));
  if (fork) TRY(tups::cuda_check(ctx, cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0), "join"));
  TRY(tups::launch_conv_sigma(ctx));
  TRY(copy_sigma_old(ctx));
  return tups::launch_vertex_update_fmax(ctx);
}

// One iteration replayed from a CUDA graph captured on first use for each
// (slices, SDE) choice, then one read of the device scalars.
static int iteration_graph(tups_ctx* ctx, int ite, tups_conv_info* info) {
  TRY(set_dev(ctx));
  const int sl = tups::current_bse_slices(ctx);
  const bool do_sde = !ctx->p.oneshot || ite == ctx->p.ite_max - 1;
  const int key = sl * 2 + (do_sde ? 1 : 0);
  if (!ctx->graph_exec[key]) {
    if (!ctx->side_stream) {
      TRY(tups::cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking), "side stream"));
      TRY(tups::cuda_check(ctx, cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming), "fork event"));
      TRY(tups::cuda_check(ctx, cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming), "join event"));
    }
    const long long l0 = ctx->launches;
    TRY(tups::cuda_check(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed), "begin capture"));
    ctx->capturing = true;
    const int rc = iteration_device(ctx, sl, do_sde);
    ctx->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc;
    }
    TRY(tups::cuda_check(ctx, e, "end capture"));
    e = cudaGraphInstantiate(&ctx->graph_exec[key], g, 0);
    cudaGraphDestroy(g);
    TRY(tups::cuda_check(ctx, e, "graph instantiate"));
    ctx->graph_launches[key] = ctx->launches - l0;
    ctx->launches = l0;
  }
  const bool tune = ctx->precision_ladder;
  if (tune) {
    for (int i = 0; i < 2; i++)
      if (!ctx->tune_ev[i]) TRY(tups::cuda_check(ctx, cudaEventCreate(&ctx->tune_ev[i]), "event"));
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->tune_ev[0], ctx->stream), "event"));
  }
  TRY(tups::cuda_check(ctx, cudaGraphLaunch(ctx->graph_exec[key], ctx->stream), "graph launch"));
  ctx->launches += ctx->graph_launches[key];
  if (tune) {
    TRY(tups::cuda_check(ctx, cudaEventRecord(ctx->tune_ev[1], ctx->stream), "event"));
    ctx->tune_pending = sl;
  }
  double sc[tups::S_COUNT];
  TRY(read_scalars(ctx, sc));
  const int st = (int)sc[tups::S_STATUS];
  if (st != 0) {
    double z = 0.0;
    cudaMemcpy(ctx->s.scal + tups::S_STATUS, &z, sizeof(double), cudaMemcpyHostToDevice);
    return tups::set_error(ctx, st, st == TUPS_ERR_MU_NOCONV ? "mu bisection exceeded its step cap"
                                                             : "device routine reported an error");
  }
  tups_conv_info ci;
  const int rc = conv_finish(ctx, sc, &ci);
  if (info) *info = ci;
  if (rc) return rc;
  if (ite % 5 == 0 || ite == ctx->p.ite_max - 1 || ci.converged) TRY(tups::launch_output_mu(ctx));
  return TUPS_OK;
}

// one iteration with the readout of the output block at the reference's
// output iterations (every 5th, the last, on convergence), after conv and
// before the vertex update, as each step of tups_execute_loop does
extern "C" int tups_iteration_readout(tups_ctx* ctx, int ite, tups_conv_info* info) {
  if (ctx && ctx->ntasks > 1)
    return tups::set_error(ctx, TUPS_ERR_STATE, "the readout needs every slot: use an unsharded context");
  return iteration_impl(ctx, ite, info, true);
}

extern "C" int tups_set_graph(tups_ctx* ctx, int enable) {
  if (!ctx) return TUPS_ERR_BADARG;
  ctx->use_graph = enable != 0;
  return TUPS_OK;
}

static int iteration_impl(tups_ctx* ctx, int ite, tups_conv_info* info, bool with_readout) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  // SRC/loop.f90:67 .. 222, without the HDF5 output
  TRY(green_async(ctx, 0));
  TRY(bse_async(ctx));
  if (ite == 0 || !ctx->have_exp) {
    TRY(tups_calculate_expSqR(ctx));
    TRY(tups_calculate_expqSR(ctx));
  }
  tups::phase_begin(ctx, TUPS_PHASE_PHIR);
  TRY(tups::launch_phir(ctx));
  tups::phase_end(ctx, TUPS_PHASE_PHIR);
  ctx->have_phir = true;
  if (ite == 0 || !ctx->have_M)
    for (int w = 0; w < 4; w++) TRY(calc_M(ctx, w));
  tups::phase_begin(ctx, TUPS_PHASE_PAE);
  TRY(tups::launch_pae(ctx));
  tups::phase_end(ctx, TUPS_PHASE_PAE);
  if (!ctx->p.oneshot || ite == ctx->p.ite_max - 1) TRY(sde_async(ctx));
  TRY(device_status(ctx));
  tups_conv_info ci;
  int rc = tups_conv(ctx, &ci);
  if (info) *info = ci;
  if (rc) return rc;
  if (ite % 5 == 0 || ite == ctx->p.ite_max - 1 || ci.converged) {
    if (with_readout && ctx->ntasks == 1) TRY(readout_async(ctx));
    else TRY(tups::launch_output_mu(ctx));
  }
  tups::phase_begin(ctx, TUPS_PHASE_UPDATE);
  TRY(tups::launch_vertex_update(ctx));
  tups::phase_end(ctx, TUPS_PHASE_UPDATE);
  return TUPS_OK;
}

extern "C" int tups_execute_loop(tups_ctx* ctx, int* ite_out, int* converged) {
  if (!ctx) return TUPS_ERR_BADARG;
  int ite = 0, conv = 0;
  while (!conv && ite < ctx->p.ite_max) {
    tups_conv_info ci;
    int rc = iteration_impl(ctx, ite, &ci, true);
    if (rc) {
      if (ite_out) *ite_out = ite;
      return rc;
    }
    conv = ci.converged;
    ite++;
  }
  if (ite_out) *ite_out = ite;
  if (converged) *converged = conv;
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "execute_loop");
}

// ---- state in/out -----------------------------------------------------------
extern "C" int tups_get_sigma(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  return copy_d2h(ctx, h, ctx->s.Sigma, (size_t)ctx->d.Nt * sizeof(cplx));
}
extern "C" int tups_set_sigma(tups_ctx* ctx, const double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  return copy_h2d(ctx, ctx->s.Sigma, h, (size_t)ctx->d.Nt * sizeof(cplx));
}
extern "C" int tups_get_sigma_old(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  return copy_d2h(ctx, h, ctx->s.SigmaOld, (size_t)ctx->d.Nt * sizeof(cplx));
}
extern "C" int tups_get_Gkw(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  return copy_d2h(ctx, h, ctx->s.Gkw, (size_t)ctx->d.Nt * sizeof(cplx));
}
extern "C" int tups_get_Grt(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  return copy_d2h(ctx, h, ctx->s.Grt, (size_t)d.Nx * d.Ngrain * d.Ny * d.Ngrain * d.Nf * sizeof(cplx));
}
extern "C" int tups_get_mu(tups_ctx* ctx, double* mu) {
  if (!ctx || !mu) return TUPS_ERR_BADARG;
  return copy_d2h(ctx, mu, ctx->s.scal + tups::S_MU, sizeof(double));
}
extern "C" int tups_set_mu(tups_ctx* ctx, double mu) {
  if (!ctx) return TUPS_ERR_BADARG;
  return copy_h2d(ctx, ctx->s.scal + tups::S_MU, &mu, sizeof(double));
}
static cplx* vertex_ptr(tups_ctx* ctx, int channel, int which) {
  if (channel < 0 || channel > 3 || which < 0 || which > 1) return nullptr;
  return which == 0 ? ctx->s.F[channel] : ctx->s.G[channel];
}
extern "C" int tups_get_vertex(tups_ctx* ctx, int channel, int which, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  cplx* p = vertex_ptr(ctx, channel, which);
  if (!p) return tups::set_error(ctx, TUPS_ERR_BADARG, "channel/which out of range");
  const auto& d = ctx->d;
  return copy_d2h(ctx, h, p, (size_t)d.Nz * d.Nz * d.Nb * sizeof(cplx));
}
extern "C" int tups_set_vertex(tups_ctx* ctx, int channel, int which, const double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  cplx* p = vertex_ptr(ctx, channel, which);
  if (!p) return tups::set_error(ctx, TUPS_ERR_BADARG, "channel/which out of range");
  const auto& d = ctx->d;
  return copy_h2d(ctx, p, h, (size_t)d.Nz * d.Nz * d.Nb * sizeof(cplx));
}
// a run of `count` consecutive local slots starting at `slot_begin` (0-based)
static int slot_range(tups_ctx* ctx, int slot_begin, int count, size_t* off, size_t* bytes) {
  const auto& d = ctx->d;
  if (slot_begin < 0 || count < 1 || slot_begin > d.Nb - count)
    return tups::set_error(ctx, TUPS_ERR_BADARG, "slot range outside [0, Nb)");
  *off = (size_t)d.Nz * d.Nz * slot_begin;
  *bytes = (size_t)d.Nz * d.Nz * count * sizeof(cplx);
  return TUPS_OK;
}
extern "C" int tups_get_vertex_slots(tups_ctx* ctx, int channel, int which, int slot_begin, int count, double* h) {
  if (!ctx || !h) return TUPS_ERR_BADARG;
  cplx* p = vertex_ptr(ctx, channel, which);
  if (!p) return tups::set_error(ctx, TUPS_ERR_BADARG, "channel/which out of range");
  size_t off = 0, bytes = 0;
  TRY(slot_range(ctx, slot_begin, count, &off, &bytes));
  return copy_d2h(ctx, h, p + off, bytes);
}
extern "C" int tups_set_vertex_slots(tups_ctx* ctx, int channel, int which, int slot_begin, int count,
                                     const double* h) {
  if (!ctx || !h) return TUPS_ERR_BADARG;
  cplx* p = vertex_ptr(ctx, channel, which);
  if (!p) return tups::set_error(ctx, TUPS_ERR_BADARG, "channel/which out of range");
  size_t off = 0, bytes = 0;
  TRY(slot_range(ctx, slot_begin, count, &off, &bytes));
  return copy_h2d(ctx, p + off, h, bytes);
}
extern "C" int tups_get_PhiR(tups_ctx* ctx, int channel, double* h) {
  if (!ctx || channel < 0 || channel > 3) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  return copy_d2h(ctx, h, ctx->s.PhiR[channel], (size_t)d.Nz * d.Nz * (d.Nf / 2) * d.NR * sizeof(cplx));
}
extern "C" int tups_get_M(tups_ctx* ctx, int which, double* h) {
  if (!ctx || which < 0 || which > 3 || !h) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  const size_t nl4 = (size_t)d.Nl * d.Nl * d.Nl * d.Nl;
  std::vector<cplx> m(nl4 * d.NIBZ * d.NR);
  TRY(copy_d2h(ctx, m.data(), ctx->s.M[which], m.size() * sizeof(cplx)));
  cplx* out = reinterpret_cast<cplx*>(h);
  for (int R = 0; R < d.NR; R++)
    for (int q = 0; q < d.Nb; q++) {
      const int Qi = q / (d.Nf / 2);
      std::memcpy(out + nl4 * (q + (size_t)d.Nb * R), m.data() + nl4 * (Qi + (size_t)d.NIBZ * R), nl4 * sizeof(cplx));
    }
  return TUPS_OK;
}
extern "C" int tups_get_expSqR(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  return copy_d2h(ctx, h, ctx->t.expSqR, (size_t)d.NIBZ * d.NR * tups::NS * sizeof(cplx));
}
extern "C" int tups_get_expqSR(tups_ctx* ctx, double* h) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  return copy_d2h(ctx, h, ctx->t.expqSR, (size_t)d.Nc * d.NR * tups::NS * sizeof(cplx));
}
extern "C" int tups_get_sde_aux(tups_ctx* ctx, double* cph, double* cpp, double* lchi, double* phchi,
                                double* ppchi) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  const size_t na = (size_t)d.Nl * d.nbox * d.Nb * sizeof(cplx), nz = (size_t)d.Nz * d.Nb * sizeof(cplx);
  if (cph) TRY(copy_d2h(ctx, cph, ctx->s.chi_aux_ph, na));
  if (cpp) TRY(copy_d2h(ctx, cpp, ctx->s.chi_aux_pp, na));
  // the device keeps these slot-fastest (Nb, Nz); the caller gets (Nz, Nb)
  std::vector<cplx> tmp;
  const cplx* src[3] = {ctx->s.LChi, ctx->s.PhChi, ctx->s.PPChi};
  double* dst[3] = {lchi, phchi, ppchi};
  for (int a = 0; a < 3; a++) {
    if (!dst[a]) continue;
    tmp.resize((size_t)d.Nz * d.Nb);
    TRY(copy_d2h(ctx, tmp.data(), src[a], nz));
    cplx* out = reinterpret_cast<cplx*>(dst[a]);
    for (size_t q = 0; q < (size_t)d.Nb; q++)
      for (size_t i = 0; i < (size_t)d.Nz; i++) out[i + d.Nz * q] = tmp[q + d.Nb * i];
  }
  return TUPS_OK;
}
extern "C" int tups_synchronize(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "synchronize");
}

// ---- warm start and checkpoint ----------------------------------------------
static int dev_alloc(tups_ctx* ctx, void** p, size_t bytes, const char* what) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return tups::set_error(ctx, TUPS_ERR_OOM, what);
  }
  ctx->allocations.push_back(*p);
  return TUPS_OK;
}

extern "C" int tups_warm_start(tups_ctx* ctx, const double* sigma, const double* gamma_l1) {
  if (!ctx || !sigma || !gamma_l1) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  const auto& d = ctx->d;
  const size_t n2b = (size_t)d.Nz * d.Nz * d.Nb;
  if (!ctx->lu_work) {
    TRY(dev_alloc(ctx, (void**)&ctx->lu_work, n2b * sizeof(cplx), "warm-start LU workspace"));
    TRY(dev_alloc(ctx, (void**)&ctx->lu_ipiv, (size_t)d.Nz * d.Nb * sizeof(int), "warm-start pivots"));
  }
  TRY(copy_h2d(ctx, ctx->s.Sigma, sigma, (size_t)d.Nt * sizeof(cplx)));
  TRY(green_async(ctx, 0));
  TRY(tups::launch_chi(ctx, 0, d.Nb));
  TRY(device_status(ctx));
  const double a = 1.0 / (ctx->p.beta * d.Nx * d.Ny);
  const double c[4] = {0.5, 0.5, -0.25, 0.25};
  std::vector<int> n(d.Nb, d.Nz), nl(d.Nb, d.Nl), status(d.Nb, 0);
  for (int r = 0; r < 4; r++) {
    TRY(tups::launch_set_l1_block(ctx, ctx->s.G[r], gamma_l1[2 * r], gamma_l1[2 * r + 1]));
    std::vector<double> scale(d.Nb, 2.0 * c[r] * a);
    const tups::cplx* chi = r < 2 ? ctx->s.chi_ph : ctx->s.chi_pp;
    int rc = tups_bse_lu_batched(d.Nb, n.data(), nl.data(), scale.data(), (const double*)ctx->s.G[r],
                                 (const double*)chi, (double*)ctx->s.F[r], (double*)ctx->lu_work, ctx->lu_ipiv, 0,
                                 status.data(), ctx->stream);
    if (rc) return tups::set_error(ctx, rc, "warm-start BSE solve failed");
    for (int q = 0; q < d.Nb; q++)
      if (status[q]) return tups::set_error(ctx, TUPS_ERR_NAN, "warm-start BSE kernel singular");
    ctx->launches++;
  }
  for (int r = 0; r < 4; r++) ctx->F_max_prev[r] = 0.0;
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "warm start");
}

extern "C" int tups_checkpoint(tups_ctx* ctx, int save) {
  if (!ctx) return TUPS_ERR_BADARG;
  TRY(set_dev(ctx));
  const auto& d = ctx->d;
  const size_t vb = (size_t)d.Nz * d.Nz * d.Nb * sizeof(cplx), sb = (size_t)d.Nt * sizeof(cplx);
  if (!ctx->ck_sigma) {
    for (int r = 0; r < 4; r++) {
      TRY(dev_alloc(ctx, (void**)&ctx->ck_F[r], vb, "checkpoint"));
      TRY(dev_alloc(ctx, (void**)&ctx->ck_G[r], vb, "checkpoint"));
    }
    TRY(dev_alloc(ctx, (void**)&ctx->ck_sigma, sb, "checkpoint"));
    TRY(dev_alloc(ctx, (void**)&ctx->ck_sigma_old, sb, "checkpoint"));
  }
  if (!save && !ctx->ck_valid) return tups::set_error(ctx, TUPS_ERR_STATE, "no checkpoint stored");
  auto cp = [&](void* dst, const void* src, size_t b) {
    return tups::cuda_check(ctx, cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToDevice, ctx->stream), "checkpoint");
  };
  for (int r = 0; r < 4; r++) {
    TRY(save ? cp(ctx->ck_F[r], ctx->s.F[r], vb) : cp(ctx->s.F[r], ctx->ck_F[r], vb));
    TRY(save ? cp(ctx->ck_G[r], ctx->s.G[r], vb) : cp(ctx->s.G[r], ctx->ck_G[r], vb));
  }
  TRY(save ? cp(ctx->ck_sigma, ctx->s.Sigma, sb) : cp(ctx->s.Sigma, ctx->ck_sigma, sb));
  TRY(save ? cp(ctx->ck_sigma_old, ctx->s.SigmaOld, sb) : cp(ctx->s.SigmaOld, ctx->ck_sigma_old, sb));
  if (save) {
    TRY(read_scalars(ctx, ctx->ck_scal));
    for (int r = 0; r < 4; r++) ctx->ck_fmax[r] = ctx->F_max_prev[r];
    ctx->ck_valid = true;
  } else {
    TRY(copy_h2d(ctx, ctx->s.scal, ctx->ck_scal, tups::S_COUNT * sizeof(double)));
    for (int r = 0; r < 4; r++) ctx->F_max_prev[r] = ctx->ck_fmax[r];
  }
  return tups::cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "checkpoint");
}

extern "C" int tups_set_bse_precision(tups_ctx* ctx, int slices, int ladder) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (slices < 0 || slices > 8 || slices == 1) return tups::set_error(ctx, TUPS_ERR_BADARG, "slices must be 0 or 2..8");
  ctx->bse_slices = slices;
  ctx->precision_ladder = ladder != 0;
  ctx->cur_slices = slices;
  return TUPS_OK;
}

extern "C" int tups_get_bse_slices(const tups_ctx* ctx) { return ctx ? tups::current_bse_slices(ctx) : -1; }
