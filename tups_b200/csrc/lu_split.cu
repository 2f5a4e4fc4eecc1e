// LU form of the Bethe-Salpeter equation in split precision with FP64
// iterative refinement, batched over instances of uneven size (no
// counterpart in the reference, whose BSE is the damped update of
// SRC/parquet_BSE.f90:72-128; this mode agrees with it at the fixed point):
//   F = (1 - c Gamma chi)^{-1} Gamma,   Phi = F - Gamma.
//
// Instances are grouped by size n and each group is solved in group-
// contiguous buffers:
//  * A = I - c Gamma chi (chi block-diagonal in nu, n^2 Nl per instance).
//  * Blocked right-looking LU with partial pivoting, blocks of 128 columns.
//    The panel (all rows, 128 columns) is factored in FP64 by one CTA per
//    instance, in sub-panels of 32 with the sub-panel updates on the FP64
//    tensor cores; the trailing update A22 -= L21 U12 (K = 128) runs on the
//    int8 tensor cores as an Ozaki split GEMM with s slices (ozaki.cu), so
//    the factors are those of a matrix within about 10^(1.1-2s) of A.
//  * X = U^{-1} L^{-1} P Gamma: 128-row diagonal blocks in FP64 (sub-blocks
//    of 32 plus FP64 tensor-core updates), the off-diagonal updates on the
//    int8 path.
//  * Refinement: R = Gamma - A X = Gamma - X + c Gamma (chi X) in FP64 (the
//    GEMM on the FP64 tensor cores, three real products per complex one);
//    stop when max|R| <= tol max|Gamma| for every instance of the group (or
//    after max_refine corrections), else D = U^{-1} L^{-1} P R as above and
//    X += D.  Each correction multiplies the error by about
//    kappa(A) 10^(1.1-2s).
//
// Caller-owned workspace only (tups_bse_lu_split_workspace bytes).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "lu_device.cuh"
#include "tups_device.cuh"

namespace tups {
namespace {

using lud::cabs1;
using lud::rank_update;

constexpr int LS_NB = 128;      // block of the split-precision updates
constexpr int LS_SUB = 32;      // inner block of the FP64 work
constexpr int LS_THREADS = 256;
constexpr int LS_EPI_SUB = 2;   // OzRun::epi: C -= A B

struct LsDesc {
  long long g_off;  // complex offset of Gamma_i / out_i in the caller's packed arrays
  long long c_off;  // complex offset of chi_i
  int nl;
  double scale;     // c
};

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

__device__ double block_max(double v) {
  __shared__ double red[LS_THREADS / 32];
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

// Gg = Xg = Gamma_i, Ag = I - c Gamma_i chi_i (sums over l1 ascending, as the
// FP64 LU form in lu.cu)
__global__ void __launch_bounds__(LS_THREADS) k_ls_form(const LsDesc* __restrict__ desc, const cplx* __restrict__ gamma,
                                                        const cplx* __restrict__ chi_all, cplx* __restrict__ Gg,
                                                        cplx* __restrict__ Xg, cplx* __restrict__ Ag,
                                                        unsigned long long* gmax, int n) {
  const int i = blockIdx.y;
  const LsDesc d = desc[i];
  const int nl = d.nl, nf = n / nl;
  const size_t n2 = (size_t)n * n;
  const cplx* G = gamma + d.g_off;
  const cplx* chi = chi_all + d.c_off;
  double mx = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(e % n), col = (int)(e / n);
    const int l2 = col / nf, nu = col % nf;
    cplx acc = cmk(0.0, 0.0);
    for (int l1 = 0; l1 < nl; l1++) acc = cfma(G[row + (size_t)n * (l1 * nf + nu)], chi[l1 + nl * (l2 + (size_t)nl * nu)], acc);
    const cplx g = G[e];
    Gg[n2 * i + e] = g;
    Xg[n2 * i + e] = g;
    Ag[n2 * i + e] = cmk((row == col ? 1.0 : 0.0) - d.scale * acc.x, -d.scale * acc.y);
    mx = fmax(mx, fmax(fabs(g.x), fabs(g.y)));
  }
  mx = block_max(mx);
  if (threadIdx.x == 0) atomic_max_nonneg(&gmax[i], mx);
}

// one column b[0:kb] = L^{-1} b (L unit lower, kb <= 32) with the column in
// registers: b[r] -= L[r, k] b[k] for k < r in ascending order
__device__ __forceinline__ void col_lower(const cplx* __restrict__ L, int ldl, cplx* b, int kb) {
  cplx v[LS_SUB];
#pragma unroll
  for (int r = 0; r < LS_SUB; r++) v[r] = r < kb ? b[r] : cmk(0.0, 0.0);
#pragma unroll
  for (int r = 1; r < LS_SUB; r++) {
    if (r < kb) {
      cplx acc = v[r];
#pragma unroll
      for (int k = 0; k < r; k++) acc = csub(acc, cmul(L[r + (size_t)ldl * k], v[k]));
      v[r] = acc;
    }
  }
#pragma unroll
  for (int r = 0; r < LS_SUB; r++)
    if (r < kb) b[r] = v[r];
}

// one column b[0:kb] = U^{-1} b (U upper with its diagonal, kb <= 32)
__device__ __forceinline__ void col_upper(const cplx* __restrict__ U, int ldu, cplx* b, int kb) {
  cplx v[LS_SUB];
#pragma unroll
  for (int r = 0; r < LS_SUB; r++) v[r] = r < kb ? b[r] : cmk(0.0, 0.0);
#pragma unroll
  for (int r = LS_SUB - 1; r >= 0; r--) {
    if (r < kb) {
      cplx acc = v[r];
#pragma unroll
      for (int k = r + 1; k < LS_SUB; k++)
        if (k < kb) acc = csub(acc, cmul(U[r + (size_t)ldu * k], v[k]));
      const cplx u = U[r + (size_t)ldu * r];
      v[r] = (u.x == 0.0 && u.y == 0.0) ? acc : cmul(acc, crecip(u));
    }
  }
#pragma unroll
  for (int r = 0; r < LS_SUB; r++)
    if (r < kb) b[r] = v[r];
}

// Panel [j0, j0 + jb) of every instance of the group (one CTA each): partial
// pivoting LU of rows j0..n-1 in sub-panels of 32, within the panel's columns
// (k_ls_rows applies its interchanges to the other columns and forms U12).
__global__ void __launch_bounds__(LS_THREADS) k_ls_panel(cplx* __restrict__ Ag, int* __restrict__ ipiv_all,
                                                         int* __restrict__ status, int n, int j0, int jb) {
  __shared__ double s_val[LS_THREADS / 32];
  __shared__ int s_idx[LS_THREADS / 32];
  __shared__ int s_piv;
  __shared__ cplx s_inv;
  const int i = blockIdx.x;
  cplx* A = Ag + (size_t)n * n * i;
  int* ipiv = ipiv_all + (size_t)n * i;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int je = j0 + jb;
  for (int jj = j0; jj < je; jj += LS_SUB) {
    const int kb = min(LS_SUB, je - jj);
    for (int c = jj; c < jj + kb; c++) {
      double best = -1.0;
      int bi = c;
      for (int r = c + tid; r < n; r += nt) {
        const double v = cabs1(A[r + (size_t)n * c]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if ((tid & 31) == 0) {
        s_val[tid >> 5] = best;
        s_idx[tid >> 5] = bi;
      }
      __syncthreads();
      if (tid == 0) {
        double bv = s_val[0];
        int bx = s_idx[0];
        for (int w = 1; w < nt / 32; w++)
          if (s_val[w] > bv || (s_val[w] == bv && s_idx[w] < bx)) {
            bv = s_val[w];
            bx = s_idx[w];
          }
        s_piv = bx;
        ipiv[c] = bx;
        if (bv == 0.0) {
          s_inv = cmk(0.0, 0.0);
          if (status[i] == 0) status[i] = c + 1;
        } else {
          s_inv = crecip(A[bx + (size_t)n * c]);
        }
      }
      __syncthreads();
      const int p = s_piv;
      if (p != c)
        for (int col = jj + tid; col < jj + kb; col += nt) {
          const cplx t = A[c + (size_t)n * col];
          A[c + (size_t)n * col] = A[p + (size_t)n * col];
          A[p + (size_t)n * col] = t;
        }
      __syncthreads();
      const cplx inv = s_inv;
      for (int r = c + 1 + tid; r < n; r += nt) A[r + (size_t)n * c] = cmul(A[r + (size_t)n * c], inv);
      __syncthreads();
      const int ncols = jj + kb - (c + 1), nrows = n - (c + 1);
      for (int e = tid; e < ncols * nrows; e += nt) {
        const int r = c + 1 + e % nrows, col = c + 1 + e / nrows;
        A[r + (size_t)n * col] = csub(A[r + (size_t)n * col], cmul(A[r + (size_t)n * c], A[c + (size_t)n * col]));
      }
      __syncthreads();
    }
    // this sub-panel's interchanges on the other columns of the panel
    for (int c = jj; c < jj + kb; c++) {
      const int p = ipiv[c];
      if (p != c)
        for (int col = j0 + tid; col < je; col += nt) {
          if (col >= jj && col < jj + kb) continue;
          const cplx t = A[c + (size_t)n * col];
          A[c + (size_t)n * col] = A[p + (size_t)n * col];
          A[p + (size_t)n * col] = t;
        }
      __syncthreads();
    }
    const int rc = je - jj - kb;
    if (rc > 0) {
      for (int col = tid; col < rc; col += nt)
        col_lower(A + jj + (size_t)n * jj, n, A + jj + (size_t)n * (jj + kb + col), kb);
      __syncthreads();
      rank_update(A + (jj + kb) + (size_t)n * (jj + kb), A + (jj + kb) + (size_t)n * jj, A + jj + (size_t)n * (jj + kb),
                  n - jj - kb, rc, kb, n, n, n);
      __syncthreads();
    }
  }
}

// Columns outside the panel [j0, j0 + jb), LS_COLS per CTA (grid (column
// chunks, instances)): the panel's row interchanges, thread per column, then
// for the columns right of the panel U12 = L11^{-1} A12 in sub-blocks of 32
// (column in registers) with the FP64 tensor-core update between them.
constexpr int LS_COLS = 128;

__global__ void __launch_bounds__(LS_COLS) k_ls_rows(cplx* __restrict__ Ag, const int* __restrict__ ipiv_all, int n,
                                                     int j0, int jb) {
  const int i = blockIdx.y;
  cplx* A = Ag + (size_t)n * n * i;
  const int* ipiv = ipiv_all + (size_t)n * i;
  const int je = j0 + jb;
  const int c0 = blockIdx.x * LS_COLS;
  const int col = c0 + threadIdx.x;
  if (col < n && (col < j0 || col >= je)) {
    cplx* x = A + (size_t)n * col;
    for (int c = j0; c < je; c++) {
      const int p = ipiv[c];
      if (p != c) {
        const cplx t = x[c];
        x[c] = x[p];
        x[p] = t;
      }
    }
  }
  const int ca = max(c0, je), cb = min(c0 + LS_COLS, n);  // this CTA's columns of A12
  if (ca >= cb) return;
  __syncthreads();
  for (int jj = j0; jj < je; jj += LS_SUB) {
    const int kb = min(LS_SUB, je - jj);
    if (col >= ca && col < cb) col_lower(A + jj + (size_t)n * jj, n, A + jj + (size_t)n * col, kb);
    __syncthreads();
    if (jj + kb < je)
      rank_update(A + (jj + kb) + (size_t)n * ca, A + (jj + kb) + (size_t)n * jj, A + jj + (size_t)n * ca,
                  je - jj - kb, cb - ca, kb, n, n, n);
    __syncthreads();
  }
}

// X <- P X: every thread applies the whole interchange sequence to its columns
__global__ void __launch_bounds__(LS_THREADS) k_ls_perm(cplx* __restrict__ Xg, const int* __restrict__ ipiv_all, int n) {
  const int i = blockIdx.y;
  cplx* X = Xg + (size_t)n * n * i;
  const int* ipiv = ipiv_all + (size_t)n * i;
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    cplx* x = X + (size_t)n * col;
    for (int c = 0; c < n; c++) {
      const int p = ipiv[c];
      if (p != c) {
        const cplx t = x[c];
        x[c] = x[p];
        x[p] = t;
      }
    }
  }
}

// forward substitution on the diagonal block [j0, j0 + jb) (unit lower),
// LS_COLS columns of the right-hand sides per CTA
__global__ void __launch_bounds__(LS_COLS) k_ls_fwd_diag(const cplx* __restrict__ Ag, cplx* __restrict__ Xg, int n,
                                                         int j0, int jb) {
  const int i = blockIdx.y;
  const cplx* A = Ag + (size_t)n * n * i;
  cplx* X = Xg + (size_t)n * n * i;
  const int je = j0 + jb;
  const int ca = blockIdx.x * LS_COLS, cb = min(ca + LS_COLS, n);
  const int col = ca + threadIdx.x;
  for (int jj = j0; jj < je; jj += LS_SUB) {
    const int kb = min(LS_SUB, je - jj);
    if (col < cb) col_lower(A + jj + (size_t)n * jj, n, X + jj + (size_t)n * col, kb);
    __syncthreads();
    if (jj + kb < je)
      rank_update(X + (jj + kb) + (size_t)n * ca, A + (jj + kb) + (size_t)n * jj, X + jj + (size_t)n * ca,
                  je - jj - kb, cb - ca, kb, n, n, n);
    __syncthreads();
  }
}

// back substitution on the diagonal block [j0, j0 + jb) (upper), LS_COLS
// columns per CTA
__global__ void __launch_bounds__(LS_COLS) k_ls_bwd_diag(const cplx* __restrict__ Ag, cplx* __restrict__ Xg, int n,
                                                         int j0, int jb) {
  const int i = blockIdx.y;
  const cplx* A = Ag + (size_t)n * n * i;
  cplx* X = Xg + (size_t)n * n * i;
  const int ca = blockIdx.x * LS_COLS, cb = min(ca + LS_COLS, n);
  const int col = ca + threadIdx.x;
  const int nsub = (jb + LS_SUB - 1) / LS_SUB;
  for (int t = nsub - 1; t >= 0; t--) {
    const int jj = j0 + t * LS_SUB, kb = min(LS_SUB, j0 + jb - jj);
    if (col < cb) col_upper(A + jj + (size_t)n * jj, n, X + jj + (size_t)n * col, kb);
    __syncthreads();
    if (jj > j0)
      rank_update(X + j0 + (size_t)n * ca, A + j0 + (size_t)n * jj, X + jj + (size_t)n * ca, jj - j0, cb - ca, kb, n,
                  n, n);
    __syncthreads();
  }
}

// Y = chi X (chi block-diagonal in nu, sums over l2 ascending)
__global__ void __launch_bounds__(LS_THREADS) k_ls_chimul(const LsDesc* __restrict__ desc, const cplx* __restrict__ chi_all,
                                                          const cplx* __restrict__ Xg, cplx* __restrict__ Yg, int n) {
  const int i = blockIdx.y;
  const LsDesc d = desc[i];
  const int nl = d.nl, nf = n / nl;
  const size_t n2 = (size_t)n * n;
  const cplx* chi = chi_all + d.c_off;
  const cplx* X = Xg + n2 * i;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(e % n), col = (int)(e / n);
    const int l1 = row / nf, nu = row % nf;
    cplx acc = cmk(0.0, 0.0);
    for (int l2 = 0; l2 < nl; l2++) acc = cfma(chi[l1 + nl * (l2 + (size_t)nl * nu)], X[(l2 * nf + nu) + (size_t)n * col], acc);
    Yg[n2 * i + e] = acc;
  }
}

__device__ __forceinline__ void ls_cp_async16(void* sdst, const void* gsrc, bool valid) {
  unsigned sz = valid ? 16u : 0u;
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz));
}

// R = Gamma - X + c Gamma Y on the FP64 tensor cores: 32 x 32 complex tiles,
// 4 warps of 16 x 16, two cp.async stages, three real products per complex
// one (P1 = Ar Br, P2 = Ai Bi, P3 = (Ar + Ai)(Br + Bi))
constexpr int RS_BM = 32, RS_BN = 32, RS_BK = 16, RS_LDL = RS_BM + 2, RS_LDR = RS_BK + 4;

__global__ void __launch_bounds__(128) k_ls_resid(const LsDesc* __restrict__ desc, const cplx* __restrict__ Gg,
                                                  const cplx* __restrict__ Yg, const cplx* __restrict__ Xg,
                                                  cplx* __restrict__ Rg, unsigned long long* rmax, int n) {
  __shared__ __align__(16) cplx sL[2][RS_BK][RS_LDL];
  __shared__ __align__(16) cplx sR[2][RS_BN][RS_LDR];
  const int i = blockIdx.y;
  const size_t n2 = (size_t)n * n;
  const cplx* Gi = Gg + n2 * i;
  const cplx* Yi = Yg + n2 * i;
  const int tiles_m = (n + RS_BM - 1) / RS_BM;
  const int m0 = (blockIdx.x % tiles_m) * RS_BM, n0 = (blockIdx.x / tiles_m) * RS_BN;
  const int ktiles = (n + RS_BK - 1) / RS_BK;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % 2) * 16, wn0 = (warp / 2) * 16;
  const int gid = lane >> 2, tig = lane & 3;
  auto load = [&](int st, int kt) {
    const int k0 = kt * RS_BK;
    for (int e = tid; e < RS_BK * RS_BM; e += 128) {
      const int m = e % RS_BM, kk = e / RS_BM, gm = m0 + m, gk = k0 + kk;
      const bool ok = gm < n && gk < n;
      ls_cp_async16(&sL[st][kk][m], ok ? Gi + gm + (size_t)n * gk : Gi, ok);
    }
    for (int e = tid; e < RS_BK * RS_BN; e += 128) {
      const int kk = e % RS_BK, c = e / RS_BK, gc = n0 + c, gk = k0 + kk;
      const bool ok = gc < n && gk < n;
      ls_cp_async16(&sR[st][c][kk], ok ? Yi + gk + (size_t)n * gc : Yi, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  double p1[2][4] = {}, p2[2][4] = {}, p3[2][4] = {};
  load(0, 0);
  for (int kt = 0; kt < ktiles; kt++) {
    const int cur = kt & 1;
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    if (kt + 1 < ktiles) load(cur ^ 1, kt + 1);
#pragma unroll
    for (int k8 = 0; k8 < RS_BK; k8 += 8) {
      const int mb = wm0 + gid;
      const cplx v0 = sL[cur][k8 + tig][mb], v1 = sL[cur][k8 + tig][mb + 8];
      const cplx v2 = sL[cur][k8 + tig + 4][mb], v3 = sL[cur][k8 + tig + 4][mb + 8];
      const double are[4] = {v0.x, v1.x, v2.x, v3.x}, aim[4] = {v0.y, v1.y, v2.y, v3.y};
      const double asum[4] = {v0.x + v0.y, v1.x + v1.y, v2.x + v2.y, v3.x + v3.y};
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int nb = wn0 + j * 8 + gid;
        const cplx w0 = sR[cur][nb][k8 + tig], w1 = sR[cur][nb][k8 + tig + 4];
        const double bre[2] = {w0.x, w1.x}, bim[2] = {w0.y, w1.y}, bsum[2] = {w0.x + w0.y, w1.x + w1.y};
        lud::dmma8(p1[j], are, bre);
        lud::dmma8(p2[j], aim, bim);
        lud::dmma8(p3[j], asum, bsum);
      }
    }
  }
  const double s = desc[i].scale;
  const cplx* Xi = Xg + n2 * i;
  cplx* Ri = Rg + n2 * i;
  double mx = 0.0;
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int row = m0 + wm0 + gid + (x >= 2 ? 8 : 0), col = n0 + wn0 + j * 8 + 2 * tig + (x & 1);
      if (row < n && col < n) {
        const size_t idx = row + (size_t)n * col;
        const double cre = p1[j][x] - p2[j][x], cim = p3[j][x] - p1[j][x] - p2[j][x];
        const cplx g = Gi[idx], xv = Xi[idx];
        const cplx rv = cmk((g.x - xv.x) + s * cre, (g.y - xv.y) + s * cim);
        Ri[idx] = rv;
        mx = fmax(mx, fmax(fabs(rv.x), fabs(rv.y)));
      }
    }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) atomic_max_nonneg(&rmax[i], mx);
}

// X += D
__global__ void __launch_bounds__(LS_THREADS) k_ls_update(cplx* __restrict__ Xg, const cplx* __restrict__ Dg, int n) {
  const int i = blockIdx.y;
  const size_t n2 = (size_t)n * n;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (size_t)gridDim.x * blockDim.x)
    Xg[n2 * i + e] = cadd(Xg[n2 * i + e], Dg[n2 * i + e]);
}

// out_i = X_i (want_phi: X_i - Gamma_i) at the instance's place in the caller's layout
__global__ void __launch_bounds__(LS_THREADS) k_ls_scatter(const LsDesc* __restrict__ desc, const cplx* __restrict__ Xg,
                                                           const cplx* __restrict__ Gg, cplx* __restrict__ out, int n,
                                                           int want_phi) {
  const int i = blockIdx.y;
  const size_t n2 = (size_t)n * n;
  cplx* o = out + desc[i].g_off;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (size_t)gridDim.x * blockDim.x) {
    cplx v = Xg[n2 * i + e];
    if (want_phi) v = csub(v, Gg[n2 * i + e]);
    o[e] = v;
  }
}

// ---- host side ------------------------------------------------------------------------
size_t up256(size_t x) { return (x + 255) / 256 * 256; }

struct LsLayout {
  size_t mat, ipiv, desc, norms, status, oz, total;
};

LsLayout ls_layout(int b, int n, int slices) {
  LsLayout L;
  L.mat = up256((size_t)b * n * n * sizeof(cplx));
  L.ipiv = up256((size_t)b * n * sizeof(int));
  L.desc = up256((size_t)b * sizeof(LsDesc));
  L.norms = up256((size_t)2 * b * sizeof(unsigned long long));  // max|R_i|, max|Gamma_i|
  L.status = up256((size_t)b * sizeof(int) + sizeof(double));
  L.oz = up256(oz_work_layout(b, n, n, std::min(LS_NB, n), slices).total + 256);
  L.total = 5 * L.mat + L.ipiv + L.desc + L.norms + L.status + L.oz + 256;
  return L;
}

// instances by size, largest first
std::map<int, std::vector<int>, std::greater<int>> ls_groups(int n_inst, const int* n) {
  std::map<int, std::vector<int>, std::greater<int>> g;
  for (int i = 0; i < n_inst; i++) g[n[i]].push_back(i);
  return g;
}

int ls_gemm_sub(cudaStream_t st, void* ozw, int b, int M, int N, int K, const cplx* A, int lda, const cplx* B,
                int ldb, cplx* C, int ldc, long long stride, int s, double* ozstat, long long* launches) {
  OzRun R;
  R.batch = b;
  R.M = M;
  R.N = N;
  R.s = s;
  R.A.p1 = A;
  R.A.s1 = stride;
  R.A.ld1 = lda;
  R.A.K1 = K;
  R.B.p1 = B;
  R.B.s1 = stride;
  R.B.ld1 = ldb;
  R.B.K1 = K;
  oz_bind_work(R, oz_work_layout(b, M, N, K, s), ozw);
  R.status = ozstat;
  R.status_code = 1.0;
  R.epi = LS_EPI_SUB;
  R.C = C;
  R.ldc = ldc;
  R.c_stride = stride;
  return oz_run(R, st, launches);
}

// X <- U^{-1} L^{-1} P X for every instance of the group
int ls_solve(cudaStream_t st, cplx* Ag, cplx* Xg, const int* ipiv, void* ozw, int b, int n, int s, double* ozstat,
             long long* launches) {
  const long long n2 = (long long)n * n;
  k_ls_perm<<<dim3((n + LS_THREADS - 1) / LS_THREADS, b), LS_THREADS, 0, st>>>(Xg, ipiv, n);
  (*launches)++;
  for (int j0 = 0; j0 < n; j0 += LS_NB) {
    const int jb = std::min(LS_NB, n - j0), je = j0 + jb;
    k_ls_fwd_diag<<<dim3((n + LS_COLS - 1) / LS_COLS, b), LS_COLS, 0, st>>>(Ag, Xg, n, j0, jb);
    (*launches)++;
    if (je < n) {
      int rc = ls_gemm_sub(st, ozw, b, n - je, n, jb, Ag + je + (size_t)n * j0, n, Xg + j0, n, Xg + je, n, n2, s,
                           ozstat, launches);
      if (rc) return rc;
    }
  }
  const int nblk = (n + LS_NB - 1) / LS_NB;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int j0 = bk * LS_NB, jb = std::min(LS_NB, n - j0);
    k_ls_bwd_diag<<<dim3((n + LS_COLS - 1) / LS_COLS, b), LS_COLS, 0, st>>>(Ag, Xg, n, j0, jb);
    (*launches)++;
    if (j0 > 0) {
      int rc = ls_gemm_sub(st, ozw, b, j0, n, jb, Ag + (size_t)n * j0, n, Xg + j0, n, Xg, n, n2, s, ozstat, launches);
      if (rc) return rc;
    }
  }
  return cudaGetLastError() == cudaSuccess ? TUPS_OK : TUPS_ERR_CUDA;
}

}  // namespace
}  // namespace tups

extern "C" size_t tups_bse_lu_split_workspace(int n_inst, const int* n, int slices) {
  using namespace tups;
  if (n_inst < 1 || !n || slices < 2 || slices > 8) return 0;
  size_t best = 0;
  for (const auto& kv : ls_groups(n_inst, n)) {
    if (kv.first < 1) return 0;
    best = std::max(best, ls_layout((int)kv.second.size(), kv.first, slices).total);
  }
  return best;
}

extern "C" int tups_bse_lu_split_batched(int n_inst, const int* n, const int* nl, const double* scale,
                                         const double* gamma, const double* chi, double* out, int want_phi,
                                         int slices, double tol, int max_refine, void* work, size_t work_bytes,
                                         int* refinements, double* residual, int* status, void* stream) {
  using namespace tups;
  if (n_inst < 1 || !n || !nl || !scale || !gamma || !chi || !out || !work) return TUPS_ERR_BADARG;
  if (slices < 2 || slices > 8 || max_refine < 0 || !(tol > 0.0)) return TUPS_ERR_BADARG;
  if (work_bytes < tups_bse_lu_split_workspace(n_inst, n, slices)) return TUPS_ERR_BADARG;
  std::vector<long long> goff(n_inst), coff(n_inst);
  long long go = 0, co = 0;
  for (int i = 0; i < n_inst; i++) {
    if (n[i] < 1 || nl[i] < 1 || n[i] % nl[i]) return TUPS_ERR_BADDIM;
    goff[i] = go;
    coff[i] = co;
    go += (long long)n[i] * n[i];
    co += (long long)nl[i] * nl[i] * (n[i] / nl[i]);
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  (void)cudaGetLastError();
  long long launches = 0;
  const cplx* G = reinterpret_cast<const cplx*>(gamma);
  const cplx* CH = reinterpret_cast<const cplx*>(chi);
  cplx* OUT = reinterpret_cast<cplx*>(out);
  for (const auto& kv : ls_groups(n_inst, n)) {
    const int nn = kv.first;
    const std::vector<int>& idx = kv.second;
    const int b = (int)idx.size();
    const LsLayout L = ls_layout(b, nn, slices);
    uint8_t* p = (uint8_t*)(((uintptr_t)work + 255) & ~(uintptr_t)255);
    cplx* Gg = (cplx*)p;
    cplx* Ag = (cplx*)(p + L.mat);
    cplx* Xg = (cplx*)(p + 2 * L.mat);
    cplx* Rg = (cplx*)(p + 3 * L.mat);
    cplx* Yg = (cplx*)(p + 4 * L.mat);
    p += 5 * L.mat;
    int* ipiv = (int*)p;
    p += L.ipiv;
    LsDesc* desc = (LsDesc*)p;
    p += L.desc;
    unsigned long long* norms = (unsigned long long*)p;  // max|R_i| [b], max|Gamma_i| [b]
    p += L.norms;
    int* stat = (int*)p;
    double* ozstat = (double*)(((uintptr_t)(stat + b) + 7) & ~(uintptr_t)7);
    p += L.status;
    void* ozw = p;
    std::vector<LsDesc> hd(b);
    for (int k = 0; k < b; k++) hd[k] = {goff[idx[k]], coff[idx[k]], nl[idx[k]], scale[idx[k]]};
    if (cudaMemcpyAsync(desc, hd.data(), b * sizeof(LsDesc), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(stat, 0, L.status, st) != cudaSuccess) {
      cudaGetLastError();
      return TUPS_ERR_CUDA;
    }
    const size_t n2 = (size_t)nn * nn;
    const dim3 eg((unsigned)std::min<size_t>((n2 + LS_THREADS - 1) / LS_THREADS, 512), b);
    if (cudaMemsetAsync(norms, 0, 2 * b * sizeof(unsigned long long), st) != cudaSuccess) return TUPS_ERR_CUDA;
    k_ls_form<<<eg, LS_THREADS, 0, st>>>(desc, G, CH, Gg, Xg, Ag, norms + b, nn);
    // P A = L U
    for (int j0 = 0; j0 < nn; j0 += LS_NB) {
      const int jb = std::min(LS_NB, nn - j0), je = j0 + jb;
      k_ls_panel<<<b, LS_THREADS, 0, st>>>(Ag, ipiv, stat, nn, j0, jb);
      if (jb < nn) k_ls_rows<<<dim3((nn + LS_COLS - 1) / LS_COLS, b), LS_COLS, 0, st>>>(Ag, ipiv, nn, j0, jb);
      if (je < nn) {
        int rc = ls_gemm_sub(st, ozw, b, nn - je, nn - je, jb, Ag + je + (size_t)nn * j0, nn, Ag + j0 + (size_t)nn * je,
                             nn, Ag + je + (size_t)nn * je, nn, (long long)n2, slices, ozstat, &launches);
        if (rc) return rc;
      }
    }
    if (cudaGetLastError() != cudaSuccess) return TUPS_ERR_CUDA;
    int rc = ls_solve(st, Ag, Xg, ipiv, ozw, b, nn, slices, ozstat, &launches);
    if (rc) return rc;
    // refinement: residual in FP64; stop once max|R_i| <= tol max|Gamma_i| for
    // every instance of the group, else correct with the split-precision factors
    int steps = 0;
    const int tiles = ((nn + RS_BM - 1) / RS_BM) * ((nn + RS_BN - 1) / RS_BN);
    std::vector<unsigned long long> hn(2 * b);
    std::vector<double> rel(b, 0.0);
    for (;;) {
      if (cudaMemsetAsync(norms, 0, b * sizeof(unsigned long long), st) != cudaSuccess) return TUPS_ERR_CUDA;
      k_ls_chimul<<<eg, LS_THREADS, 0, st>>>(desc, CH, Xg, Yg, nn);
      k_ls_resid<<<dim3(tiles, b), 128, 0, st>>>(desc, Gg, Yg, Xg, Rg, norms, nn);
      if (cudaGetLastError() != cudaSuccess) return TUPS_ERR_CUDA;
      if (cudaMemcpyAsync(hn.data(), norms, 2 * b * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st) !=
              cudaSuccess ||
          cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return TUPS_ERR_CUDA;
      }
      double worst = 0.0;
      for (int k = 0; k < b; k++) {
        double rm, gm;
        std::memcpy(&rm, &hn[k], sizeof(double));
        std::memcpy(&gm, &hn[b + k], sizeof(double));
        rel[k] = gm > 0.0 ? rm / gm : rm;
        worst = std::max(worst, rel[k]);
      }
      if (worst <= tol || steps >= max_refine) break;
      rc = ls_solve(st, Ag, Rg, ipiv, ozw, b, nn, slices, ozstat, &launches);
      if (rc) return rc;
      k_ls_update<<<eg, LS_THREADS, 0, st>>>(Xg, Rg, nn);
      steps++;
    }
    k_ls_scatter<<<eg, LS_THREADS, 0, st>>>(desc, Xg, Gg, OUT, nn, want_phi);
    std::vector<int> hs(b);
    double ozflag = 0.0;
    if (cudaMemcpyAsync(hs.data(), stat, b * sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(&ozflag, ozstat, sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      return TUPS_ERR_CUDA;
    }
    for (int k = 0; k < b; k++) {
      if (status) status[idx[k]] = hs[k];
      if (refinements) refinements[idx[k]] = steps;
      if (residual) residual[idx[k]] = rel[k];
    }
    if (ozflag != 0.0) return TUPS_ERR_TIMEOUT;
  }
  return TUPS_OK;
}
