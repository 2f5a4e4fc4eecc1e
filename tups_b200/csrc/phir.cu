// Phi(q) -> Phi(R) transform and crossing tensors.
//   calc_PhiR / FTPhis / symop_arr (SRC/parquet_PhiR.f90:35-356)
//   calculate_expSqR / calculate_expqSR (SRC/parquet_PhiR.f90:360-435)
//   calc_M_* (SRC/parquet_EQMatrix.f90:21-360), evaluated per IBZ momentum
#include <cmath>
#include <vector>

#include "tups_device.cuh"

namespace tups {

struct PhirPtrs {
  const cplx* G[4];
  cplx* PhiR[4];
};

// PhiR_r[(i,j), w, R] = (1/Nx) sum_Q sum_{sym in star(Q)} fac_sym(l_i) fac_sym(l_j)
//     Phi_r[(lsym(l_i), nu_i), (lsym(l_j), nu_j), (Q, w)] expSqR(Q, R, sym)
// One thread per (i, j) entry, all R at once.  The (sym, Q) pairs with
// sym in the star of Q (expSqR = 0 elsewhere; Nc pairs in all) are listed
// once per CTA with Q outermost, so at any moment the CTAs in flight read
// the few Nz^2 slices of one or two momenta: every symmetric image of an
// entry is then an L2 hit and Phi(Q) streams from DRAM once (the slab of all
// momenta of one (w, r), 239 MB at 16x16 / Nl = 9 / Nf = 64, exceeds L2).
// Loads are issued four pairs ahead of their FMAs.
__global__ void __launch_bounds__(256) k_phir(PhirPtrs P, const cplx* __restrict__ expSqR,
                                              const int* __restrict__ symlist, const int* __restrict__ lsym,
                                              const double* __restrict__ lfac, int Nz, int Nf, int Nl, int NIBZ,
                                              int NR, int slot0, int Nb, double inv_nx) {
  // the phase tables (expSqR, pair list, l-space maps) in shared memory: the
  // inner loop reads only Phi from global memory
  extern __shared__ __align__(16) unsigned char phir_sm[];
  cplx* sE = reinterpret_cast<cplx*>(phir_sm);                    // (NIBZ, NR, NS)
  int* sPair = reinterpret_cast<int*>(sE + (size_t)NIBZ * NR * NS);  // sym + NS Q, Q ascending
  __shared__ int sL[NS * 16];
  __shared__ double sF[NS * 16];
  __shared__ int sNp;
  for (int t = threadIdx.x; t < NIBZ * NR * NS; t += blockDim.x) sE[t] = expSqR[t];
  for (int t = threadIdx.x; t < NS * Nl; t += blockDim.x) {
    sL[t] = lsym[t];
    sF[t] = lfac[t];
  }
  const int w = blockIdx.y;  // 0..Nf/2-1
  const int nh = Nf / 2;
  if (threadIdx.x == 0) {
    int np = 0;
    for (int Q = 0; Q < NIBZ; Q++) {
      // slot (Q, w) is global slot Q nh + w; a sharded context sums its own
      const int lq = Q * nh + w - slot0;
      if (lq < 0 || lq >= Nb) continue;
      for (int sy = 0; sy < NS; sy++)
        if (symlist[NS * Q + sy]) sPair[np++] = sy + NS * Q;
    }
    sNp = np;
  }
  __syncthreads();
  const int r = blockIdx.z;
  const size_t n2 = (size_t)Nz * Nz;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n2) return;
  const int i = (int)(e % Nz), j = (int)(e / Nz);
  const int li = i / Nf, ni = i % Nf, lj = j / Nf, nj = j % Nf;
  // per symmetry: offset of the permuted entry and its sign
  long long off[NS];
  double fac[NS];
#pragma unroll
  for (int sy = 0; sy < NS; sy++) {
    off[sy] = (long long)(sL[sy + NS * li] * Nf + ni) + (long long)Nz * (sL[sy + NS * lj] * Nf + nj);
    fac[sy] = sF[sy + NS * li] * sF[sy + NS * lj];
  }
  cplx acc[8];
#pragma unroll
  for (int R = 0; R < 8; R++) acc[R] = cmk(0.0, 0.0);
  const cplx* G = P.G[r];
  const int np = sNp;
  constexpr int U = 4;
  for (int p0 = 0; p0 < np; p0 += U) {
    cplx v[U];
    int pr[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      pr[u] = p0 + u < np ? sPair[p0 + u] : -1;
      v[u] = cmk(0.0, 0.0);
      if (pr[u] >= 0) {
        const int sy = pr[u] % NS, Q = pr[u] / NS;
        long long o = off[0];
#pragma unroll
        for (int t = 1; t < NS; t++)
          if (t == sy) o = off[t];
        v[u] = __ldg(G + o + (long long)n2 * (Q * nh + w - slot0));
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (pr[u] < 0) continue;
      const int sy = pr[u] % NS, Q = pr[u] / NS;
      double f = fac[0];
#pragma unroll
      for (int t = 1; t < NS; t++)
        if (t == sy) f = fac[t];
      const cplx vv = cscale(v[u], f);
      const cplx* eq = sE + Q + (size_t)NIBZ * NR * sy;
#pragma unroll
      for (int R = 0; R < 8; R++)
        if (R < NR) acc[R] = cfma(vv, eq[(size_t)NIBZ * R], acc[R]);
    }
  }
  cplx* out = P.PhiR[r];
  for (int R = 0; R < NR; R++) out[e + n2 * ((size_t)w + (size_t)nh * R)] = cscale(acc[R], inv_nx);
}

// Crossing tensors per IBZ momentum Q; layout (Nl^4, NIBZ, NR) with l1 fastest.
// which: 0 phbar_to_ph, 1 pp_to_ph, 2 ph_to_pp, 3 phbar_to_pp.
__global__ void k_M(cplx* __restrict__ M, int which, const double* __restrict__ FF, const double* __restrict__ FFinv,
                    const cplx* __restrict__ E, const int* __restrict__ qibz_xy, const int* __restrict__ symlistR,
                    int Nx, int Ny, int Nl, int NIBZ, int NR) {
  const int nl4 = Nl * Nl * Nl * Nl;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nl4 * NIBZ * NR) return;
  int t = (int)(e % nl4);
  const int Q = (int)((e / nl4) % NIBZ), R = (int)(e / ((size_t)nl4 * NIBZ));
  const int l1 = t % Nl, l2 = (t / Nl) % Nl, l3 = (t / (Nl * Nl)) % Nl, l4 = t / (Nl * Nl * Nl);
  const int qx = qibz_xy[2 * Q] - 1, qy = qibz_xy[2 * Q + 1] - 1;  // 0-based
  const int Nc = Nx * Ny;
  auto ff = [&](int kx, int ky, int l) { return FF[kx + Nx * (ky + Ny * l)]; };
  auto ffi = [&](int s, int kx, int ky, int l) { return FFinv[s + NS * (kx + Nx * (ky + Ny * l))]; };
  auto ex = [&](int kx, int ky, int s) { return E[(ky * Nx + kx) + (size_t)Nc * (R + (size_t)NR * s)]; };
  cplx out = cmk(0.0, 0.0);
  for (int s = 0; s < NS; s++) {
    if (!symlistR[NS * R + s]) continue;  // expqSR(:, R, s) = 0 there
    if (which == 0) {
      // M1(l1,l3,l4) = sum_k conj(E) FF_l1 FFinv_l3(k) FFinv_l4(k+Q); M2(l2) = sum_k E FF_l2
      cplx m1 = cmk(0.0, 0.0), m2 = cmk(0.0, 0.0);
      for (int ky = 0; ky < Ny; ky++)
        for (int kx = 0; kx < Nx; kx++) {
          cplx ev = ex(kx, ky, s);
          double a = ff(kx, ky, l1) * ffi(s, kx, ky, l3) * ffi(s, (kx + qx) % Nx, (ky + qy) % Ny, l4);
          m1 = cadd(m1, cscale(cconj(ev), a));
          m2 = cadd(m2, cscale(ev, ff(kx, ky, l2)));
        }
      out = cfma(m1, m2, out);
    } else if (which == 1 || which == 2) {
      // M1(a,c) = sum_k FF_a FFinv_c E (or conj E); M = sum_s E(Q) M1(l1,l3) M1(l2,l4)
      cplx a13 = cmk(0.0, 0.0), a24 = cmk(0.0, 0.0);
      for (int ky = 0; ky < Ny; ky++)
        for (int kx = 0; kx < Nx; kx++) {
          cplx ev = ex(kx, ky, s);
          if (which == 2) ev = cconj(ev);
          a13 = cadd(a13, cscale(ev, ff(kx, ky, l1) * ffi(s, kx, ky, l3)));
          a24 = cadd(a24, cscale(ev, ff(kx, ky, l2) * ffi(s, kx, ky, l4)));
        }
      out = cadd(out, cmul(ex(qx, qy, s), cmul(a13, a24)));
    } else {
      // M1(l1,l3) = sum_k FF FFinv conj(E); M2(l2,l4) = sum_k FFinv_l4(Q-k) FF_l2 E
      cplx m1 = cmk(0.0, 0.0), m2 = cmk(0.0, 0.0);
      for (int ky = 0; ky < Ny; ky++)
        for (int kx = 0; kx < Nx; kx++) {
          cplx ev = ex(kx, ky, s);
          m1 = cadd(m1, cscale(cconj(ev), ff(kx, ky, l1) * ffi(s, kx, ky, l3)));
          m2 = cadd(m2, cscale(ev, ffi(s, (qx - kx + Nx) % Nx, (qy - ky + Ny) % Ny, l4) * ff(kx, ky, l2)));
        }
      out = cfma(m1, m2, out);
    }
  }
  M[e] = out;
}

int launch_phir(tups_ctx* ctx) {
  const auto& d = ctx->d;
  PhirPtrs P;
  for (int r = 0; r < 4; r++) {
    P.G[r] = ctx->s.G[r];
    P.PhiR[r] = ctx->s.PhiR[r];
  }
  if (d.NR > 8) return set_error(ctx, TUPS_ERR_BADDIM, "NR > 8 not supported");
  if (d.Nl > 16) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 16 not supported by k_phir");
  const size_t n2 = (size_t)d.Nz * d.Nz;
  const size_t sm = (size_t)d.NIBZ * d.NR * NS * sizeof(cplx) + (size_t)d.NIBZ * NS * sizeof(int);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_phir, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_phir smem attribute");
  }
  dim3 grid(cdiv(n2, 256), d.Nf / 2, 4);
  k_phir<<<grid, 256, sm, ctx->stream>>>(P, ctx->t.expSqR, ctx->t.symlist, ctx->t.lsym, ctx->t.lfac, d.Nz, d.Nf,
                                         d.Nl, d.NIBZ, d.NR, ctx->slot0, d.Nb, 1.0 / d.Nx);
  int rc = after_launch(ctx, "k_phir");
  if (rc) return rc;
  // a sharded context summed over its own momenta: Phi(R) over all ranks
  for (int r = 0; r < 4 && !rc; r++)
    rc = exchange(ctx, TUPS_XCH_PHIR + r, reinterpret_cast<double*>(ctx->s.PhiR[r]),
                  2 * n2 * (size_t)(d.Nf / 2) * d.NR, TUPS_XCH_SUM);
  return rc;
}

int launch_M(tups_ctx* ctx, int which) {
  const auto& d = ctx->d;
  // IBZ momenta (1-based) and the star lists of the lattice vectors R
  std::vector<int> qxy(2 * d.NIBZ), slR(NS * d.NR);
  for (int Q = 0; Q < d.NIBZ; Q++) {
    qxy[2 * Q] = ctx->ibz[3 * Q * (d.Nf / 2)];
    qxy[2 * Q + 1] = ctx->ibz[3 * Q * (d.Nf / 2) + 1];
  }
  for (int R = 0; R < d.NR; R++)
    for (int s = 0; s < NS; s++) slR[NS * R + s] = ctx->symlist[NS * R + s];
  int* dq = nullptr;
  int* ds = nullptr;
  int rc = cuda_check(ctx, cudaMalloc(&dq, qxy.size() * sizeof(int)), "M tables");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaMalloc(&ds, slR.size() * sizeof(int)), "M tables");
  if (rc) {
    cudaFree(dq);
    return rc;
  }
  cudaMemcpyAsync(dq, qxy.data(), qxy.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
  cudaMemcpyAsync(ds, slR.data(), slR.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream);
  const size_t n = (size_t)d.Nl * d.Nl * d.Nl * d.Nl * d.NIBZ * d.NR;
  k_M<<<cdiv(n, 128), 128, 0, ctx->stream>>>(ctx->s.M[which], which, ctx->t.FF, ctx->t.FF_inv, ctx->t.expqSR, dq, ds,
                                             d.Nx, d.Ny, d.Nl, d.NIBZ, d.NR);
  rc = after_launch(ctx, "k_M");
  cudaStreamSynchronize(ctx->stream);
  cudaFree(dq);
  cudaFree(ds);
  return rc;
}

}  // namespace tups

using tups::cplx;

namespace {
inline int wrap_neg(int i, int N) { return ((-(i - 1) + N) % N) + 1; }
void sym_op(int s, int ix, int iy, int N, int* ox, int* oy) {
  switch (s) {
    case 1: *ox = ix; *oy = iy; break;
    case 2: *ox = ix; *oy = wrap_neg(iy, N); break;
    case 3: *ox = wrap_neg(ix, N); *oy = iy; break;
    case 4: *ox = wrap_neg(ix, N); *oy = wrap_neg(iy, N); break;
    case 5: *ox = iy; *oy = ix; break;
    case 6: *ox = iy; *oy = wrap_neg(ix, N); break;
    case 7: *ox = wrap_neg(iy, N); *oy = wrap_neg(ix, N); break;
    default: *ox = wrap_neg(iy, N); *oy = ix; break;
  }
}
}  // namespace

// expSqR(Q, R, sym) = e^{i S(Q).R} for sym in the star of Q, else 0
extern "C" int tups_calculate_expSqR(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  const int nh = d.Nf / 2;
  std::vector<cplx> v((size_t)d.NIBZ * d.NR * tups::NS, make_double2(0.0, 0.0));
  for (int iq = 0; iq < d.NIBZ; iq++) {
    int qx = ctx->ibz[3 * iq * nh], qy = ctx->ibz[3 * iq * nh + 1];
    for (int s = 1; s <= tups::NS; s++) {
      if (!ctx->symlist[tups::NS * iq + s - 1]) continue;
      int sx, sy;
      sym_op(s, qx, qy, d.Nx, &sx, &sy);
      for (int ir = 0; ir < d.NR; ir++) {
        int rx = ctx->ibz[3 * ir * nh], ry = ctx->ibz[3 * ir * nh + 1];
        double qdr = (2.0 * M_PI / d.Nx) * (sx - 1) * (rx - 1) + (2.0 * M_PI / d.Ny) * (sy - 1) * (ry - 1);
        v[iq + (size_t)d.NIBZ * (ir + (size_t)d.NR * (s - 1))] = make_double2(std::cos(qdr), std::sin(qdr));
      }
    }
  }
  int rc = tups::cuda_check(ctx, cudaMemcpy(ctx->t.expSqR, v.data(), v.size() * sizeof(cplx), cudaMemcpyHostToDevice),
                            "expSqR");
  if (rc == TUPS_OK) ctx->have_exp = true;
  return rc;
}

// expqSR(k, R, sym) = e^{-i k.S(R)} for sym in the star of R, k index (ky-1)*Nx+kx
extern "C" int tups_calculate_expqSR(tups_ctx* ctx) {
  if (!ctx) return TUPS_ERR_BADARG;
  const auto& d = ctx->d;
  const int nh = d.Nf / 2;
  std::vector<cplx> v((size_t)d.Nc * d.NR * tups::NS, make_double2(0.0, 0.0));
  for (int ir = 0; ir < d.NR; ir++) {
    int rx = ctx->ibz[3 * ir * nh], ry = ctx->ibz[3 * ir * nh + 1];
    for (int s = 1; s <= tups::NS; s++) {
      if (!ctx->symlist[tups::NS * ir + s - 1]) continue;
      int sx, sy;
      sym_op(s, rx, ry, d.Nx, &sx, &sy);
      for (int ky = 1; ky <= d.Ny; ky++)
        for (int kx = 1; kx <= d.Nx; kx++) {
          int ik = (ky - 1) * d.Nx + kx;
          double kd = (2.0 * M_PI / d.Nx) * (kx - 1) * (sx - 1) + (2.0 * M_PI / d.Ny) * (ky - 1) * (sy - 1);
          v[(ik - 1) + (size_t)d.Nc * (ir + (size_t)d.NR * (s - 1))] = make_double2(std::cos(kd), -std::sin(kd));
        }
    }
  }
  return tups::cuda_check(ctx, cudaMemcpy(ctx->t.expqSR, v.data(), v.size() * sizeof(cplx), cudaMemcpyHostToDevice),
                          "expqSR");
}
