// Bubbles: calc_chi (SRC/parquet_chi.f90:438-523) for the BSE and
// calc_chi_aux (SRC/parquet_SDE.f90:344-435) for the Schwinger-Dyson equation.
#include <algorithm>

#include "tups_device.cuh"

namespace tups {

// get_green_coarse (SRC/parquet_util.f90:1303-1327), 0-based grain/momentum
// indices, 1-based frequency; out of the box Sigma -> Sigma_H
__device__ __forceinline__ cplx green_coarse(const cplx* __restrict__ Sigma, const cplx* __restrict__ SigmaH,
                                             const double* __restrict__ Ekg, int gx, int gy, int kx, int ky, int iw,
                                             int Nx, int Ny, int Nf, int Ng, double beta, double mu) {
  double e = Ekg[gx + Ng * (gy + Ng * (kx + Nx * ky))];
  cplx s = (iw >= 1 && iw <= Nf) ? Sigma[((size_t)kx * Ny + ky) * Nf + iw - 1] : SigmaH[kx + Nx * ky];
  return crecip(cmk(0.0 - e + mu - s.x, matsubara(iw, Nf, beta) - s.y));
}

// chi_ph(k, nu; q) and chi_pp(k, nu; q) for one momentum point, averaged over
// the grain (SRC/parquet_chi.f90:470-494, SRC/parquet_SDE.f90:388-424)
__device__ __forceinline__ void bubble_k(const cplx* Sigma, const cplx* SigmaH, const double* Ekg, int kx, int ky,
                                         int nu, int qx, int qy, int w, int Nx, int Ny, int Nf, int Ng, double beta,
                                         double mu, cplx* ph, cplx* pp) {
  int kpqx = (kx + qx - 1) % Nx, kpqy = (ky + qy - 1) % Ny;
  int mkx = (Nx - kx) % Nx, mky = (Ny - ky) % Ny;
  int qmkx = (mkx + qx - 1) % Nx, qmky = (mky + qy - 1) % Ny;
  int w_kpq = nu + w - 1;
  int w_qmk = (-nu + Nf + 1) + w - 1;
  cplx aph = cmk(0.0, 0.0), app = cmk(0.0, 0.0);
  const double inv = 1.0 / Ng / Ng;
  for (int gx = 0; gx < Ng; gx++)
    for (int gy = 0; gy < Ng; gy++) {
      cplx gk = green_coarse(Sigma, SigmaH, Ekg, gx, gy, kx, ky, nu, Nx, Ny, Nf, Ng, beta, mu);
      cplx gkpq = green_coarse(Sigma, SigmaH, Ekg, gx, gy, kpqx, kpqy, w_kpq, Nx, Ny, Nf, Ng, beta, mu);
      aph = cadd(aph, cscale(cmul(gk, gkpq), inv));
      cplx gqmk =
          green_coarse(Sigma, SigmaH, Ekg, Ng - 1 - gx, Ng - 1 - gy, qmkx, qmky, w_qmk, Nx, Ny, Nf, Ng, beta, mu);
      app = cadd(app, cscale(cmul(gk, gqmk), inv));
    }
  *ph = aph;
  *pp = app;
}

// one CTA per (q slot, chunk of nc frequencies): the nu-diagonal blocks
// chi_LL[(l1,nu),(l2,nu)] = sum_k chi(k,nu) FF(k,l1) FF(k,l2) (k ascending);
// output layout (Nl, Nl, Nf, Nb).  Dynamic shared memory: 2 nc Nc complex.
__global__ void __launch_bounds__(256) k_chi_blocks(const cplx* __restrict__ Sigma, const cplx* __restrict__ SigmaH,
                                                    const double* __restrict__ Ekg, const double* __restrict__ FF,
                                                    const int* __restrict__ ibz, const double* __restrict__ scal,
                                                    cplx* __restrict__ chi_ph, cplx* __restrict__ chi_pp,
                                                    int q_begin, int Nx, int Ny, int Nf, int Ng, int Nl, double beta,
                                                    int nc) {
  extern __shared__ cplx sm[];
  const int Nc = Nx * Ny;
  cplx* sph = sm;             // [nc][Nc]
  cplx* spp = sm + nc * Nc;
  const int q = q_begin + blockIdx.x;
  const int nu0 = blockIdx.y * nc + 1;
  const int nn = min(nc, Nf + 1 - nu0);
  const int qx = ibz[3 * q], qy = ibz[3 * q + 1], w = ibz[3 * q + 2];
  const double mu = scal[S_MU];
  for (int x = threadIdx.x; x < Nc * nn; x += blockDim.x) {
    const int k = x % Nc, j = x / Nc;
    const int kx = k % Nx, ky = k / Nx;
    bubble_k(Sigma, SigmaH, Ekg, kx, ky, nu0 + j, qx, qy, w, Nx, Ny, Nf, Ng, beta, mu, &sph[j * Nc + k],
             &spp[j * Nc + k]);
  }
  __syncthreads();
  const int nl2 = Nl * Nl;
  for (int x = threadIdx.x; x < nl2 * nn; x += blockDim.x) {
    const int ll = x % nl2, j = x / nl2;
    const int l1 = ll % Nl, l2 = ll / Nl;
    const cplx* ph = sph + j * Nc;
    const cplx* pp = spp + j * Nc;
    cplx a = cmk(0.0, 0.0), b = cmk(0.0, 0.0);
    for (int k = 0; k < Nc; k++) {
      double f = FF[k + (size_t)Nc * l1] * FF[k + (size_t)Nc * l2];
      a = cadd(a, cscale(ph[k], f));
      b = cadd(b, cscale(pp[k], f));
    }
    size_t o = (size_t)l1 + Nl * (l2 + (size_t)Nl * ((nu0 + j - 1) + (size_t)Nf * q));
    chi_ph[o] = a;
    chi_pp[o] = b;
  }
}

// chi_aux_ph/pp (SRC/parquet_SDE.f90:344-435): one CTA per (q slot, chunk
// of nc extended frequencies j), output ((l4-1)*nbox + j, q)
__global__ void __launch_bounds__(256) k_chi_aux(const cplx* __restrict__ Sigma, const cplx* __restrict__ SigmaH,
                                                 const double* __restrict__ Ekg, const double* __restrict__ FF,
                                                 const int* __restrict__ ibz, const double* __restrict__ scal,
                                                 cplx* __restrict__ cph, cplx* __restrict__ cpp, int Nx, int Ny,
                                                 int Nf, int Ng, int Nl, int f_range, double beta, int nc) {
  extern __shared__ cplx sm[];
  const int Nc = Nx * Ny;
  const int nbox = (2 * f_range + 1) * Nf;
  cplx* sph = sm;             // [nc][Nc]
  cplx* spp = sm + nc * Nc;
  const int q = blockIdx.x;
  const int j0 = blockIdx.y * nc;
  const int nn = min(nc, nbox - j0);
  const int qx = ibz[3 * q], qy = ibz[3 * q + 1], w = ibz[3 * q + 2];
  const double mu = scal[S_MU];
  for (int x = threadIdx.x; x < Nc * nn; x += blockDim.x) {
    const int k = x % Nc, jj = x / Nc;
    const int kx = k % Nx, ky = k / Nx;
    const int nu = j0 + jj - f_range * Nf + 1;  // l4_0, 1-based, may lie outside the box
    bubble_k(Sigma, SigmaH, Ekg, kx, ky, nu, qx, qy, w, Nx, Ny, Nf, Ng, beta, mu, &sph[jj * Nc + k],
             &spp[jj * Nc + k]);
  }
  __syncthreads();
  for (int x = threadIdx.x; x < Nl * nn; x += blockDim.x) {
    const int l = x % Nl, jj = x / Nl;
    const cplx* ph = sph + jj * Nc;
    const cplx* pp = spp + jj * Nc;
    cplx a = cmk(0.0, 0.0), b = cmk(0.0, 0.0);
    for (int k = 0; k < Nc; k++) {
      double f = FF[k + (size_t)Nc * l];
      a = cadd(a, cscale(ph[k], f));
      b = cadd(b, cscale(pp[k], f));
    }
    size_t o = (size_t)l * nbox + (j0 + jj) + (size_t)Nl * nbox * q;
    cph[o] = a;
    cpp[o] = b;
  }
}

// frequencies per CTA of the bubble kernels: up to 8 on lattices of at
// most 128 momenta (8x8: 0.059 -> 0.054 ms per call), one on larger ones,
// where a CTA already has Nc bubbles to sum (16x16: 6.45 ms with one, 6.62
// with two, 7.27 with eight per CTA); 128 threads for one, 256 for a chunk
static int chi_chunk(int Nc, int nfreq) {
  if (Nc > 128) return 1;
  const int nc = std::max(1, (16 * 1024) / (2 * Nc * (int)sizeof(cplx)));
  return std::min(std::min(nc, 8), nfreq);
}
static int chi_threads(int nc) { return nc == 1 ? 128 : 256; }

int launch_chi(tups_ctx* ctx, int q_begin, int q_count) {
  const auto& d = ctx->d;
  const int nc = chi_chunk(d.Nc, d.Nf);
  dim3 grid(q_count, (d.Nf + nc - 1) / nc);
  const size_t sm = 2 * (size_t)nc * d.Nc * sizeof(cplx);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_chi_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_chi_blocks smem attribute");
  }
  k_chi_blocks<<<grid, chi_threads(nc), sm, ctx->stream>>>(ctx->s.Sigma, ctx->s.SigmaH, ctx->t.Ekg, ctx->t.FF, ibz_local(ctx),
                                               ctx->s.scal, ctx->s.chi_ph, ctx->s.chi_pp, q_begin, d.Nx, d.Ny, d.Nf,
                                               d.Ngrain, d.Nl, ctx->p.beta, nc);
  return after_launch(ctx, "k_chi_blocks");
}

int launch_chi_aux(tups_ctx* ctx) {
  const auto& d = ctx->d;
  const int nc = chi_chunk(d.Nc, d.nbox);
  dim3 grid(d.Nb, (d.nbox + nc - 1) / nc);
  const size_t sm = 2 * (size_t)nc * d.Nc * sizeof(cplx);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_chi_aux, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_chi_aux smem attribute");
  }
  k_chi_aux<<<grid, chi_threads(nc), sm, ctx->stream>>>(ctx->s.Sigma, ctx->s.SigmaH, ctx->t.Ekg, ctx->t.FF, ibz_local(ctx),
                                            ctx->s.scal, ctx->s.chi_aux_ph, ctx->s.chi_aux_pp, d.Nx, d.Ny, d.Nf,
                                            d.Ngrain, d.Nl, ctx->p.f_range, ctx->p.beta, nc);
  return after_launch(ctx, "k_chi_aux");
}

}  // namespace tups
