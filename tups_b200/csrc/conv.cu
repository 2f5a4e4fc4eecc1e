// Convergence check conv() (SRC/parquet_check.f90:39-150) and the vertex
// update Gamma_r = F_r - Phi_r (SRC/loop.f90:219-222).
#include "tups_device.cuh"

namespace tups {

// Sigma part of conv(): max and mean of |SigmaOld - Sigma|/|Sigma|, max
// |SigmaOld - Sigma|, NaN/Inf flag.  One CTA.
__global__ void __launch_bounds__(1024) k_conv_sigma(const cplx* __restrict__ S, const cplx* __restrict__ So,
                                                     double* scal, int Nt) {
  __shared__ double sh[32];
  double mx = 0.0, sum = 0.0, dmx = 0.0, bad = 0.0, smax = 0.0;
  for (int i = threadIdx.x; i < Nt; i += blockDim.x) {
    const cplx a = S[i], b = So[i];
    const double dx = b.x - a.x, dy = b.y - a.y;
    const double d = sqrt(dx * dx + dy * dy);
    const double as = sqrt(a.x * a.x + a.y * a.y);
    const double rel = d / as;
    if (!isfinite(a.x) || !isfinite(a.y)) bad = 1.0;
    mx = fmax(mx, rel);
    dmx = fmax(dmx, d);
    smax = fmax(smax, as);
    sum += rel;
  }
  mx = warp_max(mx);
  dmx = warp_max(dmx);
  bad = warp_max(bad);
  smax = warp_max(smax);
  __shared__ double smx[32], sdm[32], sbd[32], ssm[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    smx[wid] = mx;
    sdm[wid] = dmx;
    sbd[wid] = bad;
    ssm[wid] = smax;
  }
  sum = block_sum(sum, sh);
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0, e = 0.0;
    for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) {
      a = fmax(a, smx[w]);
      b = fmax(b, sdm[w]);
      c = fmax(c, sbd[w]);
      e = fmax(e, ssm[w]);
    }
    scal[S_RELSIG] = a;
    scal[S_RELSIGAV] = fabs(sum / Nt);
    scal[S_DSIG] = b;
    scal[S_NANFLAG] = c;
    scal[S_SIGMAX] = e;
    for (int r = 0; r < 4; r++) scal[S_FMAX + r] = 0.0;
  }
}

// max |F_r| for the four channels; grid-stride, atomic max of per-CTA maxima
__global__ void k_fmax(const cplx* __restrict__ F0, const cplx* __restrict__ F1, const cplx* __restrict__ F2,
                       const cplx* __restrict__ F3, size_t n, double* scal) {
  const cplx* F = blockIdx.y == 0 ? F0 : (blockIdx.y == 1 ? F1 : (blockIdx.y == 2 ? F2 : F3));
  double mx = 0.0, bad = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cplx v = F[i];
    const double a2 = v.x * v.x + v.y * v.y;
    if (!isfinite(a2)) bad = 1.0;
    mx = fmax(mx, a2);
  }
  mx = warp_max(mx);
  bad = warp_max(bad);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(&scal[S_FMAX + blockIdx.y], sqrt(mx));
    if (bad > 0.0) atomic_max_nonneg(&scal[S_NANFLAG], 1.0);
  }
}

// G_r = F_r - G_r for the four channels
__global__ void k_vertex_update(cplx* __restrict__ G0, cplx* __restrict__ G1, cplx* __restrict__ G2,
                                cplx* __restrict__ G3, const cplx* __restrict__ F0, const cplx* __restrict__ F1,
                                const cplx* __restrict__ F2, const cplx* __restrict__ F3, size_t n) {
  cplx* G = blockIdx.y == 0 ? G0 : (blockIdx.y == 1 ? G1 : (blockIdx.y == 2 ? G2 : G3));
  const cplx* F = blockIdx.y == 0 ? F0 : (blockIdx.y == 1 ? F1 : (blockIdx.y == 2 ? F2 : F3));
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    G[i] = csub(F[i], G[i]);
}

// Both of the above in one pass over F: G_r = F_r - G_r, max |F_r| and the
// NaN flag (k_conv_sigma has reset the maxima before it).  The maxima are
// exact, so they do not depend on the order of the atomics.
__global__ void k_vertex_update_fmax(cplx* __restrict__ G0, cplx* __restrict__ G1, cplx* __restrict__ G2,
                                     cplx* __restrict__ G3, const cplx* __restrict__ F0,
                                     const cplx* __restrict__ F1, const cplx* __restrict__ F2,
                                     const cplx* __restrict__ F3, size_t n, double* scal) {
  cplx* G = blockIdx.y == 0 ? G0 : (blockIdx.y == 1 ? G1 : (blockIdx.y == 2 ? G2 : G3));
  const cplx* F = blockIdx.y == 0 ? F0 : (blockIdx.y == 1 ? F1 : (blockIdx.y == 2 ? F2 : F3));
  double mx = 0.0, bad = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const cplx v = F[i];
    const double a2 = v.x * v.x + v.y * v.y;
    if (!isfinite(a2)) bad = 1.0;
    mx = fmax(mx, a2);
    G[i] = csub(v, G[i]);
  }
  mx = warp_max(mx);
  bad = warp_max(bad);
  if ((threadIdx.x & 31) == 0) {
    atomic_max_nonneg(&scal[S_FMAX + blockIdx.y], sqrt(mx));
    if (bad > 0.0) atomic_max_nonneg(&scal[S_NANFLAG], 1.0);
  }
}

// F = G = aux * Lambda(:, :, w) on the (l=1, l=1) nu-block of every slot, w
// the slot's bosonic index (SRC/preprocessing.f90:102-116)
__global__ void k_fill_lambda_block(cplx* __restrict__ F, cplx* __restrict__ G, const cplx* __restrict__ L,
                                    const int* __restrict__ ibz, int Nz, int Nf, int Nb, double aux) {
  const size_t n = (size_t)Nf * Nf * Nb;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % Nf), j = (int)((e / Nf) % Nf);
    const size_t q = e / ((size_t)Nf * Nf);
    const int w = ibz[3 * q + 2];
    const cplx l = L[i + (size_t)Nf * (j + (size_t)Nf * (w - 1))];
    const size_t idx = i + (size_t)Nz * (j + (size_t)Nz * q);
    F[idx] = cmk(l.x * aux, l.y * aux);
    G[idx] = cmk(l.x * aux, l.y * aux);
  }
}

int launch_fill_lambda_block(tups_ctx* ctx, cplx* F, cplx* G, const cplx* L, double aux) {
  const auto& d = ctx->d;
  const size_t n = (size_t)d.Nf * d.Nf * d.Nb;
  k_fill_lambda_block<<<(unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 256, 0, ctx->stream>>>(
      F, G, L, ibz_local(ctx), d.Nz, d.Nf, d.Nb, aux);
  return after_launch(ctx, "k_fill_lambda_block");
}

// G = 0 except value on the (l=1, l=1) nu-block of every slot
__global__ void k_set_l1_block(cplx* __restrict__ G, int Nz, int Nf, int Nb, double vr, double vi) {
  const size_t n = (size_t)Nz * Nz * Nb;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % Nz), j = (int)((e / Nz) % Nz);
    G[e] = (i < Nf && j < Nf) ? cmk(vr, vi) : cmk(0.0, 0.0);
  }
}

int launch_set_l1_block(tups_ctx* ctx, cplx* G, double vr, double vi) {
  const auto& d = ctx->d;
  const size_t n = (size_t)d.Nz * d.Nz * d.Nb;
  k_set_l1_block<<<(unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 256, 0, ctx->stream>>>(G, d.Nz, d.Nf, d.Nb, vr,
                                                                                           vi);
  return after_launch(ctx, "k_set_l1_block");
}

int launch_conv_sigma(tups_ctx* ctx) {
  k_conv_sigma<<<1, 1024, 0, ctx->stream>>>(ctx->s.Sigma, ctx->s.SigmaOld, ctx->s.scal, ctx->d.Nt);
  return after_launch(ctx, "k_conv_sigma");
}

int launch_conv(tups_ctx* ctx) {
  const auto& d = ctx->d;
  int rc = launch_conv_sigma(ctx);
  if (rc) return rc;
  const size_t n = (size_t)d.Nz * d.Nz * d.Nb;
  dim3 grid((unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 4);
  k_fmax<<<grid, 256, 0, ctx->stream>>>(ctx->s.F[0], ctx->s.F[1], ctx->s.F[2], ctx->s.F[3], n, ctx->s.scal);
  rc = after_launch(ctx, "k_fmax");
  if (rc) return rc;
  // max|F_r| (4 values) and the NaN flag over the ranks of a sharded context
  static_assert(S_NANFLAG == S_FMAX + 4, "exchanged as one range");
  return exchange(ctx, TUPS_XCH_FMAX, ctx->s.scal + S_FMAX, 5, TUPS_XCH_MAX);
}

int launch_vertex_update(tups_ctx* ctx) {
  const auto& d = ctx->d;
  const size_t n = (size_t)d.Nz * d.Nz * d.Nb;
  dim3 grid((unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 4);
  k_vertex_update<<<grid, 256, 0, ctx->stream>>>(ctx->s.G[0], ctx->s.G[1], ctx->s.G[2], ctx->s.G[3], ctx->s.F[0],
                                                 ctx->s.F[1], ctx->s.F[2], ctx->s.F[3], n);
  return after_launch(ctx, "k_vertex_update");
}

int launch_vertex_update_fmax(tups_ctx* ctx) {
  const auto& d = ctx->d;
  const size_t n = (size_t)d.Nz * d.Nz * d.Nb;
  dim3 grid((unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 4);
  k_vertex_update_fmax<<<grid, 256, 0, ctx->stream>>>(ctx->s.G[0], ctx->s.G[1], ctx->s.G[2], ctx->s.G[3],
                                                      ctx->s.F[0], ctx->s.F[1], ctx->s.F[2], ctx->s.F[3], n,
                                                      ctx->s.scal);
  int rc = after_launch(ctx, "k_vertex_update_fmax");
  if (rc) return rc;
  return exchange(ctx, TUPS_XCH_FMAX, ctx->s.scal + S_FMAX, 5, TUPS_XCH_MAX);
}

}  // namespace tups
