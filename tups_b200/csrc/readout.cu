// Readout of the output block (SRC/loop.f90:181-213) without HDF5:
//   exact chi0 bubble, cal_chi branch of calc_Gkw_Grt (SRC/parquet_chi.f90:216-430)
//   susceptibilities calc_sus (SRC/parquet_sus.f90:18-643)
//   symmetrize_sus (SRC/parquet_plot.f90:14-58)
#include <cmath>
#include <vector>

#include "tups_device.cuh"

namespace tups {

// pre-FFT G(k, tau) times FF_sd(k, ff)^2 for the four s/d-wave projections
// (SRC/parquet_chi.f90:355-390); in/out (n1, n2, Nf), out has 4 such blocks
__global__ void k_scale_sd(const cplx* __restrict__ pre, const double* __restrict__ sd2, cplx* __restrict__ out,
                           int Nx, int Ny, int Ng, int Nf) {
  const int n1 = Nx * Ng, n2 = Ny * Ng;
  const size_t n = (size_t)n1 * n2 * Nf;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < 4 * n; e += (size_t)gridDim.x * blockDim.x) {
    const int ff = (int)(e / n);
    const size_t r = e % n;
    const int x = (int)(r % n1), y = (int)((r / n1) % n2);
    // coarse k of the fine point: inverse of idx = k*Ng + (kc + 1 - (Ng+1)/2) mod n
    const int kx = ((x + (Ng + 1) / 2 - 1) % n1) / Ng, ky = ((y + (Ng + 1) / 2 - 1) % n2) / Ng;
    out[e] = cscale(pre[r], sd2[(kx * Ny + ky) + (size_t)Nx * Ny * ff]);
  }
}

// the ten tau-space products whose backward FFT and spline transform give
// chi0: [0] -G(r,t)G(-r,b-t), [1] -G^2/2, [2+ff] -G(r,t)FFG_ff(-r,b-t),
// [6+ff] -G FFG_ff / 2
__global__ void k_chi0_products(const cplx* __restrict__ Grt, const cplx* __restrict__ FFG,
                                cplx* __restrict__ out, int n1, int n2, int Nf) {
  const size_t n = (size_t)n1 * n2 * Nf;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(e % n1), y = (int)((e / n1) % n2), t = (int)(e / ((size_t)n1 * n2));
    const int xm = x == 0 ? 0 : n1 - x, ym = y == 0 ? 0 : n2 - y;
    const size_t em = xm + (size_t)n1 * (ym + (size_t)n2 * (Nf - 1 - t));
    const cplx g = Grt[e];
    out[e] = cscale(cmul(g, Grt[em]), -1.0);
    out[e + n] = cscale(cmul(g, g), -0.5);
    for (int ff = 0; ff < 4; ff++) {
      out[e + (2 + ff) * n] = cscale(cmul(g, FFG[em + ff * n]), -1.0);
      out[e + (6 + ff) * n] = cscale(cmul(g, FFG[e + ff * n]), -0.5);
    }
  }
}

// FDfit + nfourier('Bosonic') at every IBZ point of `narr` fine-grid arrays
// (SRC/parquet_chi.f90:242-257, SRC/MATH_mod.f90:95-212); one CTA per
// (IBZ point, array); out[arr][ip * Nf/2 + k]
__global__ void k_spline_bosonic(const cplx* __restrict__ data, const int* __restrict__ ibz, cplx* __restrict__ out,
                                 int Nx, int Ny, int Ng, int Nf, int NIBZ, double beta) {
  extern __shared__ double sp[];
  double* r = sp;
  double* qv = sp + Nf;
  double* u = sp + 2 * Nf;
  double* xm = sp + 3 * Nf;
  const int ip = blockIdx.x, arr = blockIdx.y;
  const int nh = Nf / 2;
  const int n1 = Nx * Ng, n2 = Ny * Ng;
  const int i = ibz[3 * ip * nh], j = ibz[3 * ip * nh + 1];
  const int x = (i - 1) * Ng, y = (j - 1) * Ng;
  const cplx* d = data + (size_t)arr * n1 * n2 * Nf;
  for (int t = threadIdx.x; t < Nf; t += blockDim.x) r[t] = d[x + (size_t)n1 * (y + (size_t)n2 * t)].x;
  __syncthreads();
  const int L = Nf - 1;
  const double delta = beta / L;
  if (threadIdx.x == 0) {
    const double dt = beta / (double)(Nf - 1);
    const double fd1 = (-25.0 * r[0] + 48.0 * r[1] - 36.0 * r[2] + 16.0 * r[3] - 3.0 * r[4]) / 12.0 / dt;
    const double fd2 =
        (25.0 * r[L] - 48.0 * r[L - 1] + 36.0 * r[L - 2] - 16.0 * r[L - 3] + 3.0 * r[L - 4]) / 12.0 / dt;
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
  cplx* o = out + (size_t)arr * NIBZ * nh + (size_t)ip * nh;
  for (int w = threadIdx.x + 1; w <= nh; w += blockDim.x) {
    const double om = 2.0 * (w - 1) * M_PI / beta;
    double cr = 0.0, ci = 0.0;
    for (int jj = 1; jj <= L; jj++) {
      const double a = r[jj - 1], c = xm[jj - 1] / 2.0;
      const double b = (r[jj] - r[jj - 1]) / delta - (2.0 * xm[jj - 1] + xm[jj]) * delta / 6.0;
      const double dd = (xm[jj] - xm[jj - 1]) / (6.0 * delta);
      if (fabs(om) < 1e-6) {
        cr += a * delta + 0.5 * b * delta * delta + c * delta * delta * delta / 3.0 +
              dd * delta * delta * delta * delta / 4.0;
        continue;
      }
      const double om2 = om * om, om3 = om2 * om, om4 = om3 * om;
      double sp1, cp1, sm1, cm1;
      sincos(om * delta * jj, &sp1, &cp1);
      sincos(om * delta * (jj - 1), &sm1, &cm1);
      const double p1r = (-6.0 * dd) / om4 + (b + 2.0 * delta * c + 3.0 * delta * delta * dd) / om2;
      const double p1i =
          (2.0 * c + 6.0 * delta * dd) / om3 + (-a - delta * b - delta * delta * c - delta * delta * delta * dd) / om;
      const double p2r = 6.0 * dd / om4 - b / om2;
      const double p2i = -2.0 * c / om3 + a / om;
      cr += cp1 * p1r - sp1 * p1i + cm1 * p2r - sm1 * p2i;
      ci += cp1 * p1i + sp1 * p1r + cm1 * p2i + sm1 * p2r;
    }
    o[w - 1] = cmk(cr, ci);
  }
}

// GG_ph / GG_pp (SRC/parquet_sus.f90:528-643): one CTA per (slot, extended
// frequency j); out[(l*nbox + j) + Nl*nbox*(q + Nb*ff)]
__global__ void k_GG(const cplx* __restrict__ Sigma, const cplx* __restrict__ SigmaH, const double* __restrict__ Ekg,
                     const double* __restrict__ FF, const double* __restrict__ sd, const int* __restrict__ ibz,
                     const double* __restrict__ scal, cplx* __restrict__ gph, cplx* __restrict__ gpp, int Nx, int Ny,
                     int Nf, int Ng, int Nl, int f_range, int Nb, double beta) {
  extern __shared__ cplx sm[];
  const int Nc = Nx * Ny;
  const int nbox = (2 * f_range + 1) * Nf;
  cplx* sph = sm;
  cplx* spp = sm + Nc;
  const int q = blockIdx.x, j = blockIdx.y;
  const int nu = j - f_range * Nf + 1;
  const int qx = ibz[3 * q], qy = ibz[3 * q + 1], w = ibz[3 * q + 2];
  const double mu = scal[S_MU];
  const double inv = 1.0 / Ng / Ng;
  for (int k = threadIdx.x; k < Nc; k += blockDim.x) {
    const int kx = k % Nx, ky = k / Nx;
    const int kpqx = (kx + qx - 1) % Nx, kpqy = (ky + qy - 1) % Ny;
    const int qmkx = ((Nx - kx) % Nx + qx - 1) % Nx, qmky = ((Ny - ky) % Ny + qy - 1) % Ny;
    cplx aph = cmk(0.0, 0.0), app = cmk(0.0, 0.0);
    for (int gx = 0; gx < Ng; gx++)
      for (int gy = 0; gy < Ng; gy++) {
        auto gc = [&](int ax, int ay, int bx, int by, int iw) {
          double e = Ekg[ax + Ng * (ay + Ng * (bx + Nx * by))];
          cplx s = (iw >= 1 && iw <= Nf) ? Sigma[((size_t)bx * Ny + by) * Nf + iw - 1] : SigmaH[bx + Nx * by];
          return crecip(cmk(0.0 - e + mu - s.x, matsubara(iw, Nf, beta) - s.y));
        };
        const cplx gk = gc(gx, gy, kx, ky, nu);
        aph = cadd(aph, cscale(cmul(gk, gc(gx, gy, kpqx, kpqy, nu + w - 1)), inv));
        app = cadd(app, cscale(cmul(gk, gc(Ng - 1 - gx, Ng - 1 - gy, qmkx, qmky, (-nu + Nf + 1) + w - 1)), inv));
      }
    sph[k] = aph;
    spp[k] = app;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < Nl * 4; t += blockDim.x) {
    const int l = t % Nl, ff = t / Nl;
    cplx a = cmk(0.0, 0.0), b = cmk(0.0, 0.0);
    for (int k = 0; k < Nc; k++) {
      const int kx = k % Nx, ky = k / Nx;
      const double f = sd[(kx * Ny + ky) + (size_t)Nc * ff] * FF[k + (size_t)Nc * l];
      a = cadd(a, cscale(sph[k], f));
      b = cadd(b, cscale(spp[k], f));
    }
    const size_t o = (size_t)l * nbox + j + (size_t)Nl * nbox * (q + (size_t)Nb * ff);
    gph[o] = a;
    gpp[o] = b;
  }
}

// sus_r(q, ff) = norm sum_{ij in box} F_r[i,j,q] v_ff[i] v_ff[j]
//              + (f_range > 0) terms with an extended frequency outside the box;
// one CTA per (slot, channel)
__global__ void __launch_bounds__(256) k_sus(const cplx* __restrict__ F0, const cplx* __restrict__ F1,
                                             const cplx* __restrict__ F2, const cplx* __restrict__ F3,
                                             const cplx* __restrict__ P0, const cplx* __restrict__ P1,
                                             const cplx* __restrict__ P2, const cplx* __restrict__ P3,
                                             const cplx* __restrict__ gph, const cplx* __restrict__ gpp,
                                             cplx* __restrict__ sus, int Nz, int Nf, int Nl, int f_range, int Nb,
                                             double norm, double U, double ff2) {
  __shared__ double sh[32];
  extern __shared__ cplx v[];  // [4][Nl*nbox]
  const int q = blockIdx.x, r = blockIdx.y;
  const int nbox = (2 * f_range + 1) * Nf;
  const int ne = Nl * nbox;
  const cplx* F = r == 0 ? F0 : (r == 1 ? F1 : (r == 2 ? F2 : F3));
  const cplx* Ph = r == 0 ? P0 : (r == 1 ? P1 : (r == 2 ? P2 : P3));
  const cplx* g = r < 2 ? gph : gpp;
  for (int t = threadIdx.x; t < 4 * ne; t += blockDim.x) {
    const int ff = t / ne, e = t % ne;
    v[t] = g[e + (size_t)ne * (q + (size_t)Nb * ff)];
  }
  __syncthreads();
  const size_t n2 = (size_t)Nz * Nz;
  // in-box: i = l*Nf + nu  <->  extended index l*nbox + nu + f_range*Nf
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < Nz; i += blockDim.x) {
    const int ei = (i / Nf) * nbox + i % Nf + f_range * Nf;
    cplx rs[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int jc = 0; jc < Nz; jc++) {
      const int ej = (jc / Nf) * nbox + jc % Nf + f_range * Nf;
      const cplx f = F[i + (size_t)Nz * jc + n2 * q];
#pragma unroll
      for (int ff = 0; ff < 4; ff++) rs[ff] = cfma(f, v[ff * ne + ej], rs[ff]);
    }
#pragma unroll
    for (int ff = 0; ff < 4; ff++) {
      const cplx t = cmul(rs[ff], v[ff * ne + ei]);
      acc[2 * ff] += t.x;
      acc[2 * ff + 1] += t.y;
    }
  }
  if (f_range > 0) {
    const double lam = r == 0 ? U : (r == 1 ? -U : (r == 2 ? 2.0 * U : 0.0));
    for (int ei = threadIdx.x; ei < ne; ei += blockDim.x) {
      const int l1 = ei / nbox, j1 = ei % nbox;
      const int n1 = j1 - f_range * Nf + 1;
      const bool in1 = n1 > 0 && n1 < Nf + 1;
      const int p1 = n1 < 1 ? 1 : (n1 > Nf ? Nf : n1);
      cplx rs[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
      for (int ej = 0; ej < ne; ej++) {
        const int l2 = ej / nbox, j2 = ej % nbox;
        const int n2i = j2 - f_range * Nf + 1;
        const bool in2 = n2i > 0 && n2i < Nf + 1;
        if (in1 && in2) continue;
        const int p2 = n2i < 1 ? 1 : (n2i > Nf ? Nf : n2i);
        cplx c = Ph[(size_t)(l1 * Nf + p1 - 1) + (size_t)Nz * (l2 * Nf + p2 - 1) + n2 * q];
        if (l1 == 0 && l2 == 0) c = cadd(c, cmk(lam * ff2, 0.0));
#pragma unroll
        for (int ff = 0; ff < 4; ff++) rs[ff] = cfma(c, v[ff * ne + ej], rs[ff]);
      }
#pragma unroll
      for (int ff = 0; ff < 4; ff++) {
        const cplx t = cmul(rs[ff], v[ff * ne + ei]);
        acc[2 * ff] += t.x;
        acc[2 * ff + 1] += t.y;
      }
    }
  }
  for (int x = 0; x < 8; x++) acc[x] = block_sum(acc[x], sh);
  if (threadIdx.x == 0)
    for (int ff = 0; ff < 4; ff++)
      sus[q + (size_t)Nb * (ff + 4 * (size_t)r)] = cmk(acc[2 * ff] * norm, acc[2 * ff + 1] * norm);
}

// symmetrize_array (SRC/parquet_util.f90:1215-1272) for `narr` IBZ arrays of
// nfreq frequencies: one thread per (array, frequency), reference loop order
__global__ void k_symmetrize_batch(const cplx* __restrict__ in, cplx* __restrict__ out, const int* __restrict__ symlist,
                                   const int* __restrict__ symq, int narr, int nfreq, int Nx, int Ny, int nxibz,
                                   int NIBZ) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= narr * nfreq) return;
  const int a = t / nfreq, nu = t % nfreq;
  const cplx* src = in + (size_t)a * NIBZ * nfreq;
  cplx* dst = out + (size_t)a * Nx * Ny * nfreq;
  for (int k = 0; k < Nx * Ny; k++) dst[(size_t)k * nfreq + nu] = cmk(0.0, 0.0);
  int ip = 0;
  for (int qx = 1; qx <= nxibz; qx++)
    for (int qy = 1; qy <= qx; qy++, ip++) {
      const cplx v = src[(size_t)ip * nfreq + nu];
      for (int s = 0; s < NS; s++) {
        if (!symlist[NS * ip + s]) continue;
        const int sx = symq[2 * (NS * ip + s)], sy = symq[2 * (NS * ip + s) + 1];
        const size_t o = ((size_t)(sx - 1) * Ny + sy - 1) * nfreq + nu;
        dst[o] = cadd(dst[o], v);
      }
    }
}

int launch_readout(tups_ctx* ctx) {
  const auto& d = ctx->d;
  auto& rd = ctx->rd;
  const int n1 = d.Nx * d.Ngrain, n2 = d.Ny * d.Ngrain;
  const size_t ng = (size_t)n1 * n2 * d.Nf;
  int rc;
  // pre-FFT G(k, tau) for the current mu and Sigma
  if ((rc = launch_grt_pre(ctx, rd.pre))) return rc;
  k_scale_sd<<<cdiv(4 * ng, 256), 256, 0, ctx->stream>>>(rd.pre, rd.sd2, rd.ffg_in, d.Nx, d.Ny, d.Ngrain, d.Nf);
  if ((rc = after_launch(ctx, "k_scale_sd"))) return rc;
  if ((rc = launch_fft2d_batch(ctx, rd.ffg_in, rd.ffg, 4 * d.Nf, 1))) return rc;
  k_chi0_products<<<cdiv(ng, 256), 256, 0, ctx->stream>>>(ctx->s.Grt, rd.ffg, rd.prod, n1, n2, d.Nf);
  if ((rc = after_launch(ctx, "k_chi0_products"))) return rc;
  if ((rc = launch_fft2d_batch(ctx, rd.prod, rd.prod_ft, 10 * d.Nf, 0))) return rc;
  k_spline_bosonic<<<dim3(d.NIBZ, 10), 64, 4 * (size_t)d.Nf * sizeof(double), ctx->stream>>>(
      rd.prod_ft, ctx->t.ibz, rd.chi0, d.Nx, d.Ny, d.Ngrain, d.Nf, d.NIBZ, ctx->p.beta);
  if ((rc = after_launch(ctx, "k_spline_bosonic"))) return rc;
  // susceptibilities
  k_GG<<<dim3(d.Nb, d.nbox), 128, 2 * (size_t)d.Nc * sizeof(cplx), ctx->stream>>>(
      ctx->s.Sigma, ctx->s.SigmaH, ctx->t.Ekg, ctx->t.FF, rd.sd, ctx->t.ibz, ctx->s.scal, rd.gph, rd.gpp, d.Nx, d.Ny,
      d.Nf, d.Ngrain, d.Nl, ctx->p.f_range, d.Nb, ctx->p.beta);
  if ((rc = after_launch(ctx, "k_GG"))) return rc;
  const double norm = 1.0 / ((double)d.Nx * d.Nx * d.Ny * d.Ny * ctx->p.beta * ctx->p.beta);
  const size_t vsm = 4 * (size_t)d.Nl * d.nbox * sizeof(cplx);
  if (vsm > 48 * 1024) cudaFuncSetAttribute(k_sus, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm);
  k_sus<<<dim3(d.Nb, 4), 256, vsm, ctx->stream>>>(ctx->s.F[0], ctx->s.F[1], ctx->s.F[2], ctx->s.F[3], ctx->s.G[0],
                                                   ctx->s.G[1], ctx->s.G[2], ctx->s.G[3], rd.gph, rd.gpp, rd.sus, d.Nz,
                                                   d.Nf, d.Nl, ctx->p.f_range, d.Nb, norm, ctx->p.U,
                                                   1.0 / (ctx->FF[0] * ctx->FF[0]));
  if ((rc = after_launch(ctx, "k_sus"))) return rc;
  // whole-BZ arrays: 16 sus (channel, ff) + 10 chi0 arrays
  const int nh = d.Nf / 2;
  k_symmetrize_batch<<<cdiv(16 * nh, 64), 64, 0, ctx->stream>>>(rd.sus, rd.sus_bz, ctx->t.symlist, ctx->t.symq, 16,
                                                                  nh, d.Nx, d.Ny, d.Nx_IBZ, d.NIBZ);
  if ((rc = after_launch(ctx, "k_symmetrize_batch"))) return rc;
  k_symmetrize_batch<<<cdiv(10 * nh, 64), 64, 0, ctx->stream>>>(rd.chi0, rd.chi0_bz, ctx->t.symlist, ctx->t.symq, 10,
                                                                  nh, d.Nx, d.Ny, d.Nx_IBZ, d.NIBZ);
  return after_launch(ctx, "k_symmetrize_batch");
}

}  // namespace tups
