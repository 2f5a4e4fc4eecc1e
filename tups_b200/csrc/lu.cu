// LU form of the Bethe-Salpeter equation, batched over instances of uneven
// size (no counterpart in the reference, whose BSE is the damped update of
// SRC/parquet_BSE.f90:72-128; this mode agrees with it at the fixed point):
//   F = (1 - c Gamma chi)^{-1} Gamma,   Phi = F - Gamma,
// per (q, channel) instance with n = Nl*Nnu and chi block-diagonal in nu.
//
// One persistent launch: each CTA takes the next instance from an atomic
// counter (instances queued largest first), forms A = I - c Gamma chi (cost
// n^2 Nl), factors P A = L U with partial pivoting (blocked, panel width 32,
// trailing rank-32 updates on the FP64 tensor cores), and solves L U F = P
// Gamma in place for all n right-hand sides.  Caller-owned buffers only; the
// instance table lives in a static device array.
#include <algorithm>
#include <cstdio>
#include <numeric>
#include <vector>

#include "tups_device.cuh"
#include "lu_device.cuh"

namespace {

using tups::cplx;
using tups::cmk;
using tups::lud::cabs1;
using tups::lud::rank_update;

constexpr int kLuMaxInst = 16384;
constexpr int NB = 32;
constexpr int LU_THREADS = 256;

struct LuDesc {
  long long g_off;  // complex offset of Gamma_i / F_i / A_i (n^2 each)
  long long c_off;  // complex offset of chi_i (Nl*Nl*Nnu)
  long long p_off;  // int offset of the pivots (n)
  int n, nl;
  double scale;     // c
};

__device__ LuDesc g_lu_desc[kLuMaxInst];
__device__ int g_lu_next;
__device__ int g_lu_status[kLuMaxInst];

// one instance: A = I - s Gamma chi; P A = L U; F = Gamma -> A^{-1} Gamma
__device__ void lu_instance(const LuDesc& d, const cplx* __restrict__ Gam, const cplx* __restrict__ chi_all,
                            cplx* __restrict__ Fout, cplx* __restrict__ Aw, int* __restrict__ piv_all, int inst) {
  __shared__ double s_val[LU_THREADS / 32];
  __shared__ int s_idx[LU_THREADS / 32];
  __shared__ int s_piv;
  __shared__ cplx s_inv;
  const int n = d.n, nl = d.nl, nf = n / nl;
  const size_t n2 = (size_t)n * n;
  const cplx* G = Gam + d.g_off;
  const cplx* chi = chi_all + d.c_off;
  cplx* A = Aw + d.g_off;
  cplx* F = Fout + d.g_off;
  int* ipiv = piv_all + d.p_off;
  const int tid = threadIdx.x, nt = blockDim.x;
  // A = I - s Gamma chi, F = Gamma
  for (size_t e = tid; e < n2; e += nt) {
    const int row = (int)(e % n), col = (int)(e / n);
    const int l2 = col / nf, nu = col % nf;
    cplx acc = cmk(0.0, 0.0);
    for (int l1 = 0; l1 < nl; l1++)
      acc = tups::cfma(G[row + (size_t)n * (l1 * nf + nu)], chi[l1 + nl * (l2 + (size_t)nl * nu)], acc);
    A[e] = cmk((row == col ? 1.0 : 0.0) - d.scale * acc.x, -d.scale * acc.y);
    F[e] = G[e];
  }
  __syncthreads();
  int singular = 0;
  for (int j0 = 0; j0 < n; j0 += NB) {
    const int jb = min(NB, n - j0);
    // ---- panel factorization, columns j0 .. j0+jb-1 ----
    for (int c = j0; c < j0 + jb; c++) {
      double best = -1.0;
      int bi = c;
      for (int r = c + tid; r < n; r += nt) {
        const double v = cabs1(A[r + (size_t)n * c]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
      // warp then block argmax (lowest row index on ties, as izamax)
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
        const cplx pv = A[bx + (size_t)n * c];
        if (bv == 0.0) {
          s_inv = cmk(0.0, 0.0);
          if (!singular) g_lu_status[inst] = c + 1;
          singular = 1;
        } else {
          s_inv = tups::crecip(pv);
        }
      }
      __syncthreads();
      const int p = s_piv;
      if (p != c)
        for (int col = j0 + tid; col < j0 + jb; col += nt) {
          const cplx t = A[c + (size_t)n * col];
          A[c + (size_t)n * col] = A[p + (size_t)n * col];
          A[p + (size_t)n * col] = t;
        }
      __syncthreads();
      const cplx inv = s_inv;
      for (int r = c + 1 + tid; r < n; r += nt) A[r + (size_t)n * c] = tups::cmul(A[r + (size_t)n * c], inv);
      __syncthreads();
      const int ncols = j0 + jb - (c + 1), nrows = n - (c + 1);
      for (int e = tid; e < ncols * nrows; e += nt) {
        const int r = c + 1 + e % nrows, col = c + 1 + e / nrows;
        A[r + (size_t)n * col] =
            tups::csub(A[r + (size_t)n * col], tups::cmul(A[r + (size_t)n * c], A[c + (size_t)n * col]));
      }
      __syncthreads();
    }
    // ---- the panel's interchanges on the columns outside it ----
    for (int c = j0; c < j0 + jb; c++) {
      const int p = ipiv[c];
      if (p != c)
        for (int col = tid; col < n; col += nt) {
          if (col >= j0 && col < j0 + jb) continue;
          const cplx t = A[c + (size_t)n * col];
          A[c + (size_t)n * col] = A[p + (size_t)n * col];
          A[p + (size_t)n * col] = t;
        }
      __syncthreads();
    }
    const int rest = n - j0 - jb;
    if (rest <= 0) continue;
    // ---- U12 = L11^{-1} A12 ----
    for (int col = j0 + jb + tid; col < n; col += nt)
      for (int rr = 1; rr < jb; rr++) {
        cplx acc = A[j0 + rr + (size_t)n * col];
        for (int kk = 0; kk < rr; kk++)
          acc = tups::csub(acc, tups::cmul(A[j0 + rr + (size_t)n * (j0 + kk)], A[j0 + kk + (size_t)n * col]));
        A[j0 + rr + (size_t)n * col] = acc;
      }
    __syncthreads();
    // ---- A22 -= L21 U12 ----
    rank_update(A + (j0 + jb) + (size_t)n * (j0 + jb), A + (j0 + jb) + (size_t)n * j0, A + j0 + (size_t)n * (j0 + jb),
                 rest, rest, jb, n, n, n);
    __syncthreads();
  }
  // ---- solve: F <- P F, L Y = F, U X = Y ----
  for (int c = 0; c < n; c++) {
    const int p = ipiv[c];
    if (p != c)
      for (int col = tid; col < n; col += nt) {
        const cplx t = F[c + (size_t)n * col];
        F[c + (size_t)n * col] = F[p + (size_t)n * col];
        F[p + (size_t)n * col] = t;
      }
    __syncthreads();
  }
  for (int j0 = 0; j0 < n; j0 += NB) {
    const int jb = min(NB, n - j0);
    for (int col = tid; col < n; col += nt)
      for (int rr = 1; rr < jb; rr++) {
        cplx acc = F[j0 + rr + (size_t)n * col];
        for (int kk = 0; kk < rr; kk++)
          acc = tups::csub(acc, tups::cmul(A[j0 + rr + (size_t)n * (j0 + kk)], F[j0 + kk + (size_t)n * col]));
        F[j0 + rr + (size_t)n * col] = acc;
      }
    __syncthreads();
    const int rest = n - j0 - jb;
    if (rest > 0) rank_update(F + (j0 + jb), A + (j0 + jb) + (size_t)n * j0, F + j0, rest, n, jb, n, n, n);
    __syncthreads();
  }
  const int nblk = (n + NB - 1) / NB;
  for (int bk = nblk - 1; bk >= 0; bk--) {
    const int j0 = bk * NB, jb = min(NB, n - j0);
    for (int col = tid; col < n; col += nt)
      for (int rr = jb - 1; rr >= 0; rr--) {
        cplx acc = F[j0 + rr + (size_t)n * col];
        for (int kk = rr + 1; kk < jb; kk++)
          acc = tups::csub(acc, tups::cmul(A[j0 + rr + (size_t)n * (j0 + kk)], F[j0 + kk + (size_t)n * col]));
        const cplx u = A[j0 + rr + (size_t)n * (j0 + rr)];
        F[j0 + rr + (size_t)n * col] = (u.x == 0.0 && u.y == 0.0) ? acc : tups::cmul(acc, tups::crecip(u));
      }
    __syncthreads();
    if (j0 > 0) rank_update(F, A + (size_t)n * j0, F + j0, j0, n, jb, n, n, n);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(LU_THREADS, 2) k_lu_batched(const cplx* __restrict__ Gam, const cplx* __restrict__ chi,
                                                           cplx* __restrict__ F, cplx* __restrict__ Aw,
                                                           int* __restrict__ ipiv, int n_inst, int want_phi) {
  __shared__ int s_inst;
  while (true) {
    if (threadIdx.x == 0) s_inst = atomicAdd(&g_lu_next, 1);
    __syncthreads();
    const int i = s_inst;
    __syncthreads();
    if (i >= n_inst) break;
    const LuDesc d = g_lu_desc[i];
    lu_instance(d, Gam, chi, F, Aw, ipiv, i);
    if (want_phi) {
      const size_t n2 = (size_t)d.n * d.n;
      for (size_t e = threadIdx.x; e < n2; e += blockDim.x)
        F[d.g_off + e] = tups::csub(F[d.g_off + e], Gam[d.g_off + e]);
    }
    __syncthreads();
  }
}

}  // namespace

extern "C" int tups_bse_lu_batched(int n_inst, const int* n, const int* nl, const double* scale, const double* gamma,
                                   const double* chi, double* out, double* work, int* ipiv, int want_phi,
                                   int* status, void* stream) {
  if (n_inst < 1 || n_inst > kLuMaxInst || !n || !nl || !scale || !gamma || !chi || !out || !work || !ipiv)
    return TUPS_ERR_BADARG;
  std::vector<LuDesc> desc(n_inst);
  long long go = 0, co = 0, po = 0;
  for (int i = 0; i < n_inst; i++) {
    if (n[i] < 1 || nl[i] < 1 || n[i] % nl[i]) return TUPS_ERR_BADDIM;
    desc[i] = {go, co, po, n[i], nl[i], scale[i]};
    go += (long long)n[i] * n[i];
    co += (long long)nl[i] * nl[i] * (n[i] / nl[i]);
    po += n[i];
  }
  // largest first: the queue order is a permutation of the packed layout
  std::vector<int> order(n_inst);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
  std::vector<LuDesc> queued(n_inst);
  for (int i = 0; i < n_inst; i++) queued[i] = desc[order[i]];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int zero = 0;
  std::vector<int> zeros(n_inst, 0);
  if (cudaMemcpyToSymbolAsync(g_lu_desc, queued.data(), n_inst * sizeof(LuDesc), 0, cudaMemcpyHostToDevice, st) !=
          cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_lu_next, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(g_lu_status, zeros.data(), n_inst * sizeof(int), 0, cudaMemcpyHostToDevice, st) !=
          cudaSuccess) {
    cudaGetLastError();
    return TUPS_ERR_CUDA;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = std::min(n_inst, 2 * sms);
  k_lu_batched<<<grid, LU_THREADS, 0, st>>>(reinterpret_cast<const cplx*>(gamma), reinterpret_cast<const cplx*>(chi),
                                            reinterpret_cast<cplx*>(out), reinterpret_cast<cplx*>(work), ipiv, n_inst,
                                            want_phi);
  if (cudaGetLastError() != cudaSuccess) return TUPS_ERR_CUDA;
  if (status) {
    std::vector<int> st_q(n_inst);
    if (cudaMemcpyFromSymbolAsync(st_q.data(), g_lu_status, n_inst * sizeof(int), 0, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      cudaGetLastError();
      return TUPS_ERR_CUDA;
    }
    for (int i = 0; i < n_inst; i++) status[order[i]] = st_q[i];
  }
  return TUPS_OK;
}
