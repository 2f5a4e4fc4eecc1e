// Schwinger-Dyson equation: calc_SDE (SRC/parquet_SDE.f90:27-258) with
// calc_LChi/PhChi/PPChi (:439-574), the Sigma_V accumulation (:116-221),
// symmetrize_array (SRC/parquet_util.f90:1215-1272) and the U^2 term
// calc_order_2nd (:264-338) with FDfit/nfourier (SRC/MATH_mod.f90:95-212).
#include "tups_device.cuh"

namespace tups {

int launch_chi_aux(tups_ctx* ctx);  // chi.cu

struct SdePtrs {
  const cplx* Phi[4];  // G arrays hold Phi_r during the SDE
  const cplx* L[4];
};

// pick index of fillpickNu_range (SRC/parquet_SDE.f90:659-675); j 0-based in
// the extended box, result 1-based in 1..Nf
__device__ __forceinline__ int pick_range(int j, int Nf, int fr) {
  const int nu = j + 1;
  if (nu <= fr * Nf) return 1;
  if (nu < (fr + 1) * Nf + 1) return nu - fr * Nf;
  return Nf;
}

// LChi, PhChi, PPChi stored slot-fastest, (Nb, Nz): element (i, q) at
// q + Nb i, so that k_sde_sigma's lanes (consecutive slots) read
// consecutive addresses.  32 rows x 8 column groups per CTA, one slot q
__global__ void k_sde_chis(SdePtrs P, const cplx* __restrict__ cph, const cplx* __restrict__ cpp,
                           const int* __restrict__ ibz, cplx* __restrict__ LChi, cplx* __restrict__ PhChi,
                           cplx* __restrict__ PPChi, int Nz, int Nf, int Nl, int fr, int use_U2, double U,
                           double ff2) {
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  const int q = blockIdx.y;
  const bool active = i0 < Nz;
  const int i = active ? i0 : Nz - 1;  // idle rows load row Nz-1 and store nothing
  const int nbox = (2 * fr + 1) * Nf;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* cph_q = cph + (size_t)Nl * nbox * q;
  const cplx* cpp_q = cpp + (size_t)Nl * nbox * q;
  const int W = ibz[3 * q + 2];
  // Lambda contribution, only the l3 = l4 = 1 block
  cplx lc = cmk(0.0, 0.0);
  if (i < Nf && threadIdx.y == 0) {
    for (int j = 0; j < nbox; j++) {
      const int l40 = j - fr * Nf + 1;
      const cplx c = cph_q[j];
      if (l40 > 0 && l40 < Nf + 1) {
        const size_t li = (size_t)i + (size_t)Nf * ((l40 - 1) + (size_t)Nf * (W - 1));
        lc = cadd(lc, cmul(cscale(P.L[0][li], ff2), c));
        lc = csub(lc, cmul(cscale(P.L[1][li], ff2), c));
        if (use_U2) lc = csub(lc, cscale(c, 2.0 * U * ff2));
      } else if (!use_U2) {
        lc = cadd(lc, cscale(c, 2.0 * U * ff2));
      }
    }
  }
  // the (l4, j) columns are split over the 8 thread rows of the CTA
  // (blockDim = 32 x 8): 8x the parallelism of one thread per row
  cplx ph = cmk(0.0, 0.0), pp = cmk(0.0, 0.0);
  const cplx* Pd = P.Phi[0] + n2 * q;
  const cplx* Pm = P.Phi[1] + n2 * q;
  const cplx* Ps = P.Phi[2] + n2 * q;
  const cplx* Pt = P.Phi[3] + n2 * q;
  const int ncol = Nl * nbox;
  for (int c = threadIdx.y; c < ncol; c += blockDim.y) {
    const int l4 = c / nbox, j = c % nbox;
    const size_t col = (size_t)(l4 * Nf + pick_range(j, Nf, fr) - 1);
    const size_t idx = (size_t)i + (size_t)Nz * col;
    const cplx a = cph_q[l4 * nbox + j], b = cpp_q[l4 * nbox + j];
    ph = cfma(Pd[idx], a, ph);
    ph = csub(ph, cmul(cscale(Pm[idx], 3.0), a));
    pp = cfma(Ps[idx], b, pp);
    pp = cfma(Pt[idx], b, pp);
  }
  __shared__ cplx red_ph[8][32], red_pp[8][32];
  red_ph[threadIdx.y][threadIdx.x] = ph;
  red_pp[threadIdx.y][threadIdx.x] = pp;
  __syncthreads();
  if (threadIdx.y != 0 || !active) return;
  for (int y = 1; y < (int)blockDim.y; y++) {
    ph = cadd(ph, red_ph[y][threadIdx.x]);
    pp = cadd(pp, red_pp[y][threadIdx.x]);
  }
  const size_t o = (size_t)q + (size_t)gridDim.y * i;  // gridDim.y = Nb
  LChi[o] = lc;
  PhChi[o] = ph;
  PPChi[o] = pp;
}

// get_green (SRC/parquet_util.f90:1278-1299): 0-based momentum, 1-based nu
__device__ __forceinline__ cplx get_green(const cplx* __restrict__ Gkw, const cplx* __restrict__ SigmaH,
                                          const double* __restrict__ Ek, int kx, int ky, int iw, int Nx, int Ny,
                                          int Nf, double beta, double mu) {
  if (iw >= 1 && iw <= Nf) return Gkw[((size_t)kx * Ny + ky) * Nf + iw - 1];
  const cplx s = SigmaH[kx + Nx * ky];
  return crecip(cmk(0.0 - Ek[kx + Nx * ky] + mu - s.x, matsubara(iw, Nf, beta) - s.y));
}

// Sigma_V(k_IBZ, nu): one CTA per (k_IBZ, nu), threads over bosonic slots
__global__ void __launch_bounds__(256) k_sde_sigma(const cplx* __restrict__ Gkw, const cplx* __restrict__ SigmaH,
                                                   const double* __restrict__ Ek, const double* __restrict__ FFinv,
                                                   const int* __restrict__ signs, const int* __restrict__ ibz,
                                                   const int* __restrict__ symlist, const int* __restrict__ symq,
                                                   const cplx* __restrict__ LChi, const cplx* __restrict__ PhChi,
                                                   const cplx* __restrict__ PPChi, const double* __restrict__ scal,
                                                   cplx* __restrict__ SigmaV, int Nx, int Ny, int Nf, int Nl, int Nz,
                                                   int Nb, int slot0, double beta, double pref) {
  __shared__ double sh[32];
  const int ik = blockIdx.x, k0 = blockIdx.y + 1;
  const int nh = Nf / 2;
  const int kx = ibz[3 * ik * nh] - 1, ky = ibz[3 * ik * nh + 1] - 1;  // 0-based IBZ point
  const double mu = scal[S_MU];
  const int mkx = (Nx - kx) % Nx, mky = (Ny - ky) % Ny;
  double sre = 0.0, sim = 0.0;
  for (int q = threadIdx.x; q < Nb; q += blockDim.x) {
    // local slot q of this context is global slot slot0 + q
    const int w = ibz[3 * (slot0 + q) + 2];
    const int Qi = (slot0 + q) / nh;
    // row i of slot q at q + Nb i
    const cplx* Lq = LChi + q;
    const cplx* Pq = PhChi + q;
    const cplx* Qq = PPChi + q;
    cplx acc = cmk(0.0, 0.0);
    for (int s = 0; s < NS; s++) {
      if (!symlist[NS * Qi + s]) continue;
      const int sx = symq[2 * (NS * Qi + s)] - 1, sy = symq[2 * (NS * Qi + s) + 1] - 1;
      const int kqx = (kx + sx) % Nx, kqy = (ky + sy) % Ny;
      const cplx gkq = get_green(Gkw, SigmaH, Ek, kqx, kqy, k0 + w - 1, Nx, Ny, Nf, beta, mu);
      const int qmkx = (mkx + sx) % Nx, qmky = (mky + sy) % Ny, qmkw = (Nf + 1 - k0) + w - 1;
      const cplx gqmk = get_green(Gkw, SigmaH, Ek, qmkx, qmky, qmkw, Nx, Ny, Nf, beta, mu);
      const cplx gkmq =
          get_green(Gkw, SigmaH, Ek, (Nx - qmkx) % Nx, (Ny - qmky) % Ny, -qmkw + Nf + 1, Nx, Ny, Nf, beta, mu);
      for (int l3 = 0; l3 < Nl; l3++) {
        const double ffi = FFinv[s + NS * (kx + Nx * (ky + Ny * l3))];
        const size_t i3 = (size_t)Nb * (l3 * Nf + k0 - 1);
        acc = cadd(acc, cscale(cmul(gkq, Lq[i3]), ffi));
        acc = cadd(acc, cscale(cmul(gkq, Pq[i3]), ffi));
        acc = cadd(acc, cscale(cmul(gqmk, Qq[i3]), ffi));
        if (w == 1) continue;
        const size_t i3m = (size_t)Nb * (l3 * Nf + Nf - k0);
        const double fs = ffi * (double)signs[l3];
        acc = cadd(acc, cscale(cmul(gkmq, cconj(Lq[i3m])), fs));
        acc = cadd(acc, cscale(cmul(gkmq, cconj(Pq[i3m])), fs));
        acc = cadd(acc, cscale(cmul(cconj(gkq), cconj(Qq[i3m])), fs));
      }
    }
    sre += acc.x;
    sim += acc.y;
  }
  sre = block_sum(sre, sh);
  sim = block_sum(sim, sh);
  if (threadIdx.x == 0) SigmaV[(size_t)ik * Nf + k0 - 1] = cmk(-pref * sre, -pref * sim);
}

// Sigma(BZ) from Sigma_V(IBZ) (symmetrize_array) plus the U^2 term; one
// thread per frequency does the whole scatter for it, in the reference's order
__global__ void k_symmetrize(const cplx* __restrict__ SigmaV, const cplx* __restrict__ order2,
                             const int* __restrict__ ibz, const int* __restrict__ symlist, const int* __restrict__ symq,
                             cplx* __restrict__ Sigma, int Nx, int Ny, int Nf, int nxibz, int use_U2) {
  // one thread per output (k, nu): the sum, in the reference's (ip, s) loop
  // order, of the IBZ values whose star images land on k (one per k on an
  // even lattice), plus the U^2 term
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)Nx * Ny * Nf) return;
  const int nu = (int)(e % Nf), k = (int)(e / Nf);
  const int kx = k / Ny + 1, ky = k % Ny + 1;
  cplx acc = cmk(0.0, 0.0);
  int ip = 0;
  for (int qx = 1; qx <= nxibz; qx++)
    for (int qy = 1; qy <= qx; qy++, ip++)
      for (int s = 0; s < NS; s++) {
        if (!symlist[NS * ip + s]) continue;
        if (symq[2 * (NS * ip + s)] == kx && symq[2 * (NS * ip + s) + 1] == ky)
          acc = cadd(acc, SigmaV[(size_t)ip * Nf + nu]);
      }
  if (use_U2) acc = cadd(acc, order2[e]);
  Sigma[e] = acc;
  (void)ibz;
}

// GGG(r, tau) = G(r,tau)^2 G(-r, beta-tau) U^2 (SRC/parquet_SDE.f90:297-305)
__global__ void k_ggg(const cplx* __restrict__ Grt, cplx* __restrict__ out, int n1, int n2, int Nf, double U) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n1 * n2 * Nf) return;
  const int x = (int)(e % n1), y = (int)((e / n1) % n2), t = (int)(e / ((size_t)n1 * n2));
  const int xm = x == 0 ? 0 : n1 - x, ym = y == 0 ? 0 : n2 - y;
  const cplx g = Grt[e];
  const cplx gm = Grt[xm + (size_t)n1 * (ym + (size_t)n2 * (Nf - 1 - t))];
  out[e] = cscale(cscale(cmul(cmul(g, g), gm), U), U);
}

// FDfit + nfourier (cubic spline with clamped end slopes, integrated exactly
// against e^{i om tau}) for one k per CTA; writes order_2nd(k, nu).  Thread 0
// solves the tridiagonal spline system, the others then sum over intervals.
__global__ void k_nfourier(const cplx* __restrict__ GGG, cplx* __restrict__ order2, int Nx, int Ny, int Ng, int Nf,
                           double beta) {
  extern __shared__ double sp[];
  double* r = sp;
  double* qv = sp + Nf;
  double* u = sp + 2 * Nf;
  double* xm = sp + 3 * Nf;
  const int k = blockIdx.x;
  const int kx = k / Ny, ky = k % Ny;
  const int n1 = Nx * Ng, n2 = Ny * Ng;
  const int kxc = kx * Ng, kyc = ky * Ng;
  const int L = Nf - 1;
  const double delta = beta / L;
  for (int t = threadIdx.x; t < Nf; t += blockDim.x) r[t] = GGG[kxc + (size_t)n1 * (kyc + (size_t)n2 * t)].x;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dt = beta / (Nf - 1);
    // FDfit (SRC/MATH_mod.f90:95-107)
    const double fd1 = (-25.0 * r[0] + 48.0 * r[1] - 36.0 * r[2] + 16.0 * r[3] - 3.0 * r[4]) / 12.0 / dt;
    const double fd2 =
        (25.0 * r[L] - 48.0 * r[L - 1] + 36.0 * r[L - 2] - 16.0 * r[L - 3] + 3.0 * r[L - 4]) / 12.0 / dt;
    // spline second derivatives (SRC/MATH_mod.f90:140-168)
    qv[0] = -0.5;
    u[0] = (3.0 / delta) * ((r[1] - r[0]) / delta - fd1);
    for (int kk = 2; kk <= L; kk++) {
      const double p = qv[kk - 2] / 2.0 + 2.0;
      qv[kk - 1] = -1.0 / 2.0 / p;
      u[kk - 1] = 3.0 / (delta * delta) * (r[kk] + r[kk - 2] - 2.0 * r[kk - 1]);
      u[kk - 1] = (u[kk - 1] - u[kk - 2] / 2.0) / p;
    }
    qv[L] = 0.5;
    u[L] = (3.0 / delta) * (fd2 - (r[L] - r[L - 1]) / delta);
    xm[L] = (u[L] - qv[L] * u[L - 1]) / (qv[L] * qv[L - 1] + 1.0);
    for (int kk = L; kk >= 1; kk--) xm[kk - 1] = qv[kk - 1] * xm[kk] + u[kk - 1];
  }
  __syncthreads();
  const size_t base = (size_t)k * Nf;
  for (int i = threadIdx.x + 1; i <= Nf / 2; i += blockDim.x) {
    const double om = (2.0 * i - 1.0) * M_PI / beta;
    const double om2 = om * om, om3 = om2 * om, om4 = om3 * om;
    double cr = 0.0, ci = 0.0;
    for (int j = 1; j <= L; j++) {
      const double a = r[j - 1], c = xm[j - 1] / 2.0;
      const double b = (r[j] - r[j - 1]) / delta - (2.0 * xm[j - 1] + xm[j]) * delta / 6.0;
      const double d = (xm[j] - xm[j - 1]) / (6.0 * delta);
      double sp1, cp1, sm1, cm1;
      sincos(om * delta * j, &sp1, &cp1);
      sincos(om * delta * (j - 1), &sm1, &cm1);
      // explus*(p1r + i p1i) + ex*(p2r + i p2i), SRC/MATH_mod.f90:200-207
      const double p1r = (-6.0 * d) / om4 + (b + 2.0 * delta * c + 3.0 * delta * delta * d) / om2;
      const double p1i =
          (2.0 * c + 6.0 * delta * d) / om3 + (-a - delta * b - delta * delta * c - delta * delta * delta * d) / om;
      const double p2r = 6.0 * d / om4 - b / om2;
      const double p2i = -2.0 * c / om3 + a / om;
      cr += cp1 * p1r - sp1 * p1i + cm1 * p2r - sm1 * p2i;
      ci += cp1 * p1i + sp1 * p1r + cm1 * p2i + sm1 * p2r;
    }
    // SRC/parquet_SDE.f90:325-330
    const int nu = Nf / 2 + 1 - i;
    order2[base + nu - 1] = cmk(cr, -ci);
    order2[base + Nf - nu] = cmk(cr, ci);
  }
}

int launch_sde(tups_ctx* ctx) {
  const auto& d = ctx->d;
  int rc = launch_chi_aux(ctx);
  if (rc) return rc;
  SdePtrs P;
  for (int r = 0; r < 4; r++) {
    P.Phi[r] = ctx->s.G[r];
    P.L[r] = ctx->t.L[r];
  }
  const double ff2 = 1.0 / (ctx->FF[0] * ctx->FF[0]);
  dim3 g1(cdiv(d.Nz, 32), d.Nb);
  k_sde_chis<<<g1, dim3(32, 8), 0, ctx->stream>>>(P, ctx->s.chi_aux_ph, ctx->s.chi_aux_pp, ibz_local(ctx), ctx->s.LChi,
                                          ctx->s.PhChi, ctx->s.PPChi, d.Nz, d.Nf, d.Nl, ctx->p.f_range,
                                          ctx->p.use_U2, ctx->p.U, ff2);
  if ((rc = after_launch(ctx, "k_sde_chis"))) return rc;
  const double pref = ctx->p.U / ctx->p.beta / ctx->p.beta / d.Nc / d.Nc / 2.0;
  dim3 g2(d.NIBZ, d.Nf);
  k_sde_sigma<<<g2, 256, 0, ctx->stream>>>(ctx->s.Gkw, ctx->s.SigmaH, ctx->t.Ek, ctx->t.FF_inv, ctx->t.signs,
                                           ctx->t.ibz, ctx->t.symlist, ctx->t.symq, ctx->s.LChi, ctx->s.PhChi,
                                           ctx->s.PPChi, ctx->s.scal, ctx->s.SigmaV, d.Nx, d.Ny, d.Nf, d.Nl, d.Nz,
                                           d.Nb, ctx->slot0, ctx->p.beta, pref);
  if ((rc = after_launch(ctx, "k_sde_sigma"))) return rc;
  // a sharded context summed its own slots: Sigma_V over all ranks
  if ((rc = exchange(ctx, TUPS_XCH_SIGMAV, reinterpret_cast<double*>(ctx->s.SigmaV), 2 * (size_t)d.NIBZ * d.Nf,
                     TUPS_XCH_SUM)))
    return rc;
  if (ctx->p.use_U2) {
    const int n1 = d.Nx * d.Ngrain, n2 = d.Ny * d.Ngrain;
    const size_t n = (size_t)n1 * n2 * d.Nf;
    k_ggg<<<cdiv(n, 256), 256, 0, ctx->stream>>>(ctx->s.Grt, ctx->s.Grt_work, n1, n2, d.Nf, ctx->p.U);
    if ((rc = after_launch(ctx, "k_ggg"))) return rc;
    if ((rc = launch_fft2d(ctx, ctx->s.Grt_work, ctx->s.GGG, 0))) return rc;
    k_nfourier<<<d.Nc, 64, 4 * (size_t)d.Nf * sizeof(double), ctx->stream>>>(ctx->s.GGG, ctx->s.order2, d.Nx, d.Ny,
                                                                            d.Ngrain, d.Nf, ctx->p.beta);
    if ((rc = after_launch(ctx, "k_nfourier"))) return rc;
  }
  k_symmetrize<<<cdiv((long long)d.Nc * d.Nf, 128), 128, 0, ctx->stream>>>(ctx->s.SigmaV, ctx->s.order2, ctx->t.ibz, ctx->t.symlist,
                                                       ctx->t.symq, ctx->s.Sigma, d.Nx, d.Ny, d.Nf, d.Nx_IBZ,
                                                       ctx->p.use_U2);
  return after_launch(ctx, "k_symmetrize");
}

}  // namespace tups
