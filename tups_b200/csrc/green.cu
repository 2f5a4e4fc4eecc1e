// Green's function, chemical-potential bisection and G(r, tau):
// calc_Gkw_Grt (SRC/parquet_chi.f90:18-210), fftf2d/fftb2d (SRC/MATH_mod.f90:215-259).
#include "tups_device.cuh"

namespace tups {

// parquet_chi.f90:120 compares against the single-precision literal 1e-6
__device__ __constant__ double kMuTol = 9.999999974752427e-07;

// Sigma_H(kx, ky) = Sigma(k, nu = Nf) (SRC/parquet_chi.f90:105-111)
__global__ void k_sigma_hartree(const cplx* __restrict__ Sigma, cplx* __restrict__ SigmaH, int Nx, int Ny,
                                int Nf) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Nx * Ny) return;
  int kx = k / Ny, ky = k % Ny;
  SigmaH[kx + Nx * ky] = Sigma[(size_t)k * Nf + Nf - 1];
}

// G(k, tau) before the spatial FFT for one fine-grid point and one tau:
// sum_nu Re(tw(tau,nu) (G - G0)(nu))/beta - exp((beta-tau)(e-mu))/(1+exp(beta(e-mu)))
// (SRC/parquet_chi.f90:144-165).  `gd` holds (G - G0)(nu) for this point.
__device__ __forceinline__ double grt_point(const cplx* __restrict__ tw_tau, const cplx* gd, int it, int Nf,
                                            double beta, double e, double mu) {
  double tau = beta / (Nf - 1) * (it - 1);
  double dummy = 0.0;
  for (int nu = 0; nu < Nf; nu++) {
    cplx t = tw_tau[(it - 1) + (size_t)Nf * nu];
    cplx v = cmul(t, gd[nu]);
    dummy = dummy + v.x / beta;
  }
  return dummy - exp((beta - tau) * (e - mu)) / (1.0 + exp(beta * (e - mu)));
}

// The whole bisection in one CTA: each step needs only the particle number
// n = -2 Re G(r=0, tau=beta) = -2 * mean over fine k of G(k, tau=beta), the
// r = 0 term of fftf2d.  The loop is capped; on overrun S_STATUS is set.
__global__ void __launch_bounds__(512) k_bisection(const cplx* __restrict__ Sigma, const double* __restrict__ Ekg,
                                                   const cplx* __restrict__ tw_tau, double* scal, int Nx, int Ny,
                                                   int Nf, int Ng, double beta, double U, double nParticle,
                                                   int cal_chi, int max_steps) {
  __shared__ double sh[32];
  __shared__ double s_t1;
  const int npts = Nx * Ny * Ng * Ng;
  double mu = scal[S_MU];
  double up = mu + U, lo = mu - U;
  double t1 = 3.0;
  int steps = 0;
  int status = 0;
  while (fabs(t1 - nParticle) > kMuTol) {
    if (steps >= max_steps) {
      status = TUPS_ERR_MU_NOCONV;
      break;
    }
    mu = 0.5 * (up + lo);
    double part = 0.0;
    for (int pt = threadIdx.x; pt < npts; pt += blockDim.x) {
      // pt -> (kxc, kyc, kx, ky) with kxc fastest, as Ek_grain is laid out
      const int r = pt / (Ng * Ng);
      const int kx = r % Nx, ky = r / Nx;
      double e = Ekg[pt];
      const cplx* sg = Sigma + ((size_t)kx * Ny + ky) * Nf;
      // only tau = beta (it = Nf) is needed
      double tau = beta / (Nf - 1) * (Nf - 1);
      double dummy = 0.0;
      for (int nu = 1; nu <= Nf; nu++) {
        cplx fr = cmk(0.0, matsubara(nu, Nf, beta));
        cplx gc = crecip(cmk(fr.x + mu - e - sg[nu - 1].x, fr.y - sg[nu - 1].y));
        cplx g0 = crecip(cmk(fr.x + mu - e, fr.y));
        cplx d = csub(gc, g0);
        cplx v = cmul(tw_tau[(Nf - 1) + (size_t)Nf * (nu - 1)], d);
        dummy = dummy + v.x / beta;
      }
      part += dummy - exp((beta - tau) * (e - mu)) / (1.0 + exp(beta * (e - mu)));
    }
    double tot = block_sum(part, sh);
    if (threadIdx.x == 0) s_t1 = -2.0 * (tot / (double)(Nx * Ng) / (double)(Ny * Ng));
    __syncthreads();
    t1 = s_t1;
    __syncthreads();
    steps++;
    if (cal_chi) break;
    if (t1 > nParticle) up = mu;
    else lo = mu;
  }
  if (threadIdx.x == 0) {
    if (steps > 0) scal[S_MU] = mu;
    scal[S_T1] = t1;
    scal[S_STEPS] = (double)steps;
    if (status) scal[S_STATUS] = (double)status;
  }
}

// G(k, tau) on the fine grid for the final mu, one CTA per fine-grid point,
// one thread per tau (SRC/parquet_chi.f90:124-174).  Output indexed by the
// fine-grid position (idx1, idx2) of parquet_chi.f90:135-139.
__global__ void k_grt_points(const cplx* __restrict__ Sigma, const double* __restrict__ Ekg,
                             const cplx* __restrict__ tw_tau, const double* __restrict__ scal, cplx* __restrict__ out,
                             int Nx, int Ny, int Nf, int Ng, double beta) {
  extern __shared__ cplx gd[];
  const int pt = blockIdx.x;
  int kxc = pt % Ng, r = pt / Ng;
  int kyc = r % Ng;
  r /= Ng;
  int kx = r % Nx, ky = r / Nx;
  const double mu = scal[S_MU];
  const double e = Ekg[pt];
  const cplx* sg = Sigma + ((size_t)kx * Ny + ky) * Nf;
  for (int nu = threadIdx.x; nu < Nf; nu += blockDim.x) {
    cplx fr = cmk(0.0, matsubara(nu + 1, Nf, beta));
    cplx gc = crecip(cmk(fr.x + mu - e - sg[nu].x, fr.y - sg[nu].y));
    cplx g0 = crecip(cmk(fr.x + mu - e, fr.y));
    gd[nu] = csub(gc, g0);
  }
  __syncthreads();
  int idx1 = kx * Ng + (kxc + 1 - (Ng + 1) / 2);
  if (idx1 < 0) idx1 += Ng * Nx;
  int idx2 = ky * Ng + (kyc + 1 - (Ng + 1) / 2);
  if (idx2 < 0) idx2 += Ng * Ny;
  const int n1 = Nx * Ng, n2 = Ny * Ng;
  for (int it = threadIdx.x + 1; it <= Nf; it += blockDim.x) {
    double v = grt_point(tw_tau, gd, it, Nf, beta, e, mu);
    out[idx1 + (size_t)n1 * (idx2 + (size_t)n2 * (it - 1))] = cmk(v, 0.0);
  }
}

// 2D DFT of every (n1, n2) slice: forward (e^{-i}, divided by n1 and n2) as
// fftf2d, or backward (e^{+i}, unnormalised) as fftb2d.  One CTA per slice;
// first along dim 1 then dim 2, like the reference.
__global__ void k_fft2d(const cplx* __restrict__ in, cplx* __restrict__ out, const cplx* __restrict__ tw1,
                        const cplx* __restrict__ tw2, int n1, int n2, int forward) {
  extern __shared__ cplx buf[];
  cplx* a = buf;            // n1*n2
  cplx* b = buf + n1 * n2;  // n1*n2
  const size_t off = (size_t)blockIdx.x * n1 * n2;
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) a[i] = in[off + i];
  __syncthreads();
  const double s1 = forward ? 1.0 / n1 : 1.0, s2 = forward ? 1.0 / n2 : 1.0;
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) {
    int x = i % n1, col = i / n1;
    cplx acc = cmk(0.0, 0.0);
    for (int aa = 0; aa < n1; aa++) {
      cplx t = tw1[(aa * x) % n1];
      if (!forward) t = cconj(t);
      acc = cfma(a[aa + n1 * col], t, acc);
    }
    b[i] = cscale(acc, s1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) {
    int x = i % n1, y = i / n1;
    cplx acc = cmk(0.0, 0.0);
    for (int bb = 0; bb < n2; bb++) {
      cplx t = tw2[(bb * y) % n2];
      if (!forward) t = cconj(t);
      acc = cfma(b[x + n1 * bb], t, acc);
    }
    out[off + i] = cscale(acc, s2);
  }
}

// G(k, nu) = 1/(i nu - e_k + mu - Sigma) (SRC/parquet_chi.f90:203-210)
__global__ void k_gkw(const cplx* __restrict__ Sigma, const double* __restrict__ Ek, const double* __restrict__ scal,
                      cplx* __restrict__ Gkw, int Nx, int Ny, int Nf, double beta) {
  int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= Nx * Ny * Nf) return;
  int nu = idx % Nf, k = idx / Nf;
  int kx = k / Ny, ky = k % Ny;
  double mu = scal[S_MU];
  double e = Ek[kx + Nx * ky];
  cplx s = Sigma[idx];
  double fi = matsubara(nu + 1, Nf, beta);
  Gkw[idx] = crecip(cmk(0.0 - e + mu - s.x, fi - s.y));
}

// mu <- 0.5*((mu+U)+(mu-U)): the first bisection midpoint of the readout's
// calc_Gkw_Grt(.true.) call (SRC/parquet_chi.f90:114-122)
__global__ void k_output_mu(double* scal, double U) {
  double mu = scal[S_MU];
  scal[S_MU] = 0.5 * ((mu + U) + (mu - U));
}

int launch_sigma_hartree(tups_ctx* ctx) {
  const auto& d = ctx->d;
  k_sigma_hartree<<<cdiv(d.Nc, 128), 128, 0, ctx->stream>>>(ctx->s.Sigma, ctx->s.SigmaH, d.Nx, d.Ny, d.Nf);
  return after_launch(ctx, "k_sigma_hartree");
}

int launch_bisection(tups_ctx* ctx, int cal_chi, int max_steps) {
  const auto& d = ctx->d;
  k_bisection<<<1, 512, 0, ctx->stream>>>(ctx->s.Sigma, ctx->t.Ekg, ctx->t.tw_tau, ctx->s.scal, d.Nx, d.Ny, d.Nf,
                                          d.Ngrain, ctx->p.beta, ctx->p.U, ctx->p.nParticle, cal_chi, max_steps);
  return after_launch(ctx, "k_bisection");
}

int launch_grt_pre(tups_ctx* ctx, cplx* out) {
  const auto& d = ctx->d;
  const int npts = d.Nc * d.Ngrain * d.Ngrain;
  k_grt_points<<<npts, 64, d.Nf * sizeof(cplx), ctx->stream>>>(ctx->s.Sigma, ctx->t.Ekg, ctx->t.tw_tau, ctx->s.scal,
                                                               out, d.Nx, d.Ny, d.Nf, d.Ngrain, ctx->p.beta);
  return after_launch(ctx, "k_grt_points");
}

int launch_grt(tups_ctx* ctx) {
  int rc = launch_grt_pre(ctx, ctx->s.Grt_work);
  if (rc) return rc;
  return launch_fft2d(ctx, ctx->s.Grt_work, ctx->s.Grt, 1);
}

int launch_fft2d_batch(tups_ctx* ctx, const cplx* in, cplx* out, int nslices, int forward) {
  const auto& d = ctx->d;
  const int n1 = d.Nx * d.Ngrain, n2 = d.Ny * d.Ngrain;
  size_t sm = 2 * (size_t)n1 * n2 * sizeof(cplx);
  if (sm > 200 * 1024) return set_error(ctx, TUPS_ERR_BADDIM, "fine k grid too large for the in-CTA DFT");
  if (sm > 48 * 1024) cudaFuncSetAttribute(k_fft2d, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_fft2d<<<nslices, 256, sm, ctx->stream>>>(in, out, ctx->t.tw_x, ctx->t.tw_y, n1, n2, forward);
  return after_launch(ctx, "k_fft2d");
}

int launch_fft2d(tups_ctx* ctx, const cplx* in, cplx* out, int forward) {
  return launch_fft2d_batch(ctx, in, out, ctx->d.Nf, forward);
}

int launch_gkw(tups_ctx* ctx) {
  const auto& d = ctx->d;
  k_gkw<<<cdiv(d.Nt, 256), 256, 0, ctx->stream>>>(ctx->s.Sigma, ctx->t.Ek, ctx->s.scal, ctx->s.Gkw, d.Nx, d.Ny,
                                                  d.Nf, ctx->p.beta);
  return after_launch(ctx, "k_gkw");
}

int launch_output_mu(tups_ctx* ctx) {
  k_output_mu<<<1, 1, 0, ctx->stream>>>(ctx->s.scal, ctx->p.U);
  return after_launch(ctx, "k_output_mu");
}

}  // namespace tups
