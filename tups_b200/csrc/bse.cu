// Bethe-Salpeter step, BSE(ite) (SRC/parquet_BSE.f90:19-135).
//
// Per bosonic slot q and channel r the reference computes, with four ZGEMMs,
//   Phi_r = c_r f [ (a Gamma chi) F + F (a chi Gamma) ] + (1-f)(F - Gamma),
// a = 1/(beta Nx Ny), c_d = c_m = 1/2 (chi_ph), c_s = -1/4, c_t = +1/4 (chi_pp).
// chi is block-diagonal in nu (one Nl x Nl block per nu), so Gamma chi and
// chi Gamma cost Nz^2 Nl each (k_bse_prep + k_bse_prep_b, or the two in one
// launch, k_bse_prep_ab: a tuner choice).  The remaining work is ONE complex
// GEMM with K = 2 Nz,  [Gamma chi | F] x [F ; chi Gamma],  run on the FP64
// tensor cores (mma.sync m16n8k8 f64, k_bse_gemm) with the scale and the
// damping term fused into the epilogue; Phi_r overwrites Gamma_r in place.
#include <algorithm>
#include <string>

#include "tups_device.cuh"

namespace tups {

struct BsePtrs {
  cplx* F[4];
  cplx* G[4];
  double scale[4];  // c_r * f * a
};

// A = Gamma chi and B = chi Gamma for the instances (q, r) of one chunk;
// instance = (q - q_begin) * 4 + r.  Column-major (Nz, Nz), row = l*Nf + nu.
// Each thread owns one (row, nu) line of Gamma chi or one (nu, col) line of
// chi Gamma: it loads the Nl entries of Gamma that the line needs once and
// forms all Nl outputs from registers (sums in l ascending order).  LMAX >= Nl
// sizes the register array (instantiated for the shell counts 1, 5, 9, 13).
// One row of CTAs per instance (blockIdx.y); every thread takes one line
// (a grid-stride loop over all instances at a few CTAs per SM was slower at
// 9 form factors: one line's loads in flight per thread).
//
// Gamma chi: the lanes of a warp run over rows at one nu, so every chi
// entry they read is one address.
template <int LMAX>
__device__ __forceinline__ void prep_gamma_chi(const BsePtrs& P, const cplx* __restrict__ chi_ph,
                                               const cplx* __restrict__ chi_pp, cplx* __restrict__ A, int q_begin,
                                               int Nz, int Nf, int Nl, int cta, int ncta) {
  const size_t lines = (size_t)Nz * Nf;
  const int inst = blockIdx.y;
  const int q = q_begin + inst / 4, r = inst % 4;
  const cplx* chi = (r < 2 ? chi_ph : chi_pp) + (size_t)Nl * Nl * Nf * q;
  // constant indices keep the parameter struct out of local memory
  const cplx* Gr = r == 0 ? P.G[0] : r == 1 ? P.G[1] : r == 2 ? P.G[2] : P.G[3];
  const cplx* Gm = Gr + (size_t)Nz * Nz * q;
  cplx* Ai = A + (size_t)Nz * Nz * inst;
  for (size_t t = (size_t)cta * blockDim.x + threadIdx.x; t < lines; t += (size_t)ncta * blockDim.x) {
    cplx g[LMAX];
    // A[row, (l2, nu)] = sum_l1 Gamma[row, (l1, nu)] chi[l1, l2, nu]
    const int row = (int)(t % Nz), nu = (int)(t / Nz);
#pragma unroll
    for (int l = 0; l < LMAX; l++)
      if (l < Nl) g[l] = Gm[row + (size_t)Nz * (l * Nf + nu)];
    for (int l2 = 0; l2 < Nl; l2++) {
      cplx acc = cmk(0.0, 0.0);
#pragma unroll
      for (int l1 = 0; l1 < LMAX; l1++)
        if (l1 < Nl) acc = cfma(g[l1], chi[l1 + Nl * (l2 + (size_t)Nl * nu)], acc);
      Ai[row + (size_t)Nz * (l2 * Nf + nu)] = acc;
    }
  }
}

// chi Gamma: B[(l1, nu), col] = sum_l2 chi[l1, l2, nu] Gamma[(l2, nu), col]
// (sum in l2 ascending).  CTA = 32 frequencies (lanes) x 8 columns (warps)
// of one instance; the lanes' chi entries differ in nu, so the CTA first
// stages chi[:, :, nu0 .. nu0 + 31] in shared memory, [l1 + Nl l2][lane]
// with a row pitch of 33 (conflict-free stores of consecutive l1 + Nl l2)
// (read straight from global memory they were 32 cache lines per load).
// Shared memory chs: Nl^2 x 33 complex.
template <int LMAX>
__device__ __forceinline__ void prep_chi_gamma(const BsePtrs& P, const cplx* __restrict__ chi_ph,
                                               const cplx* __restrict__ chi_pp, cplx* __restrict__ B, int q_begin,
                                               int Nz, int Nf, int Nl, int cta, cplx* chs) {
  const int inst = blockIdx.y;
  const int q = q_begin + inst / 4, r = inst % 4;
  const int nchunk = (Nf + 31) / 32;
  const int nu0 = (cta % nchunk) * 32, col = (cta / nchunk) * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31, nu = nu0 + lane;
  const int nl2 = Nl * Nl;
  const cplx* chi = (r < 2 ? chi_ph : chi_pp) + (size_t)nl2 * Nf * q;
  const int nn = min(32, Nf - nu0);
  // chi[:, :, nu0 .. nu0 + nn) is contiguous in global memory
  for (int e = threadIdx.x; e < nl2 * nn; e += blockDim.x) {
    const int ll = e % nl2, j = e / nl2;
    chs[ll * 33 + j] = chi[(size_t)ll + (size_t)nl2 * (nu0 + j)];
  }
  __syncthreads();
  if (nu >= Nf || col >= Nz) return;
  const cplx* Gr = r == 0 ? P.G[0] : r == 1 ? P.G[1] : r == 2 ? P.G[2] : P.G[3];
  const cplx* Gm = Gr + (size_t)Nz * Nz * q + (size_t)Nz * col;
  cplx* Bi = B + (size_t)Nz * Nz * inst + (size_t)Nz * col;
  cplx g[LMAX];
#pragma unroll
  for (int l = 0; l < LMAX; l++)
    if (l < Nl) g[l] = Gm[l * Nf + nu];
  for (int l1 = 0; l1 < Nl; l1++) {
    cplx acc = cmk(0.0, 0.0);
#pragma unroll
    for (int l2 = 0; l2 < LMAX; l2++)
      if (l2 < Nl) acc = cfma(chs[(l1 + Nl * l2) * 33 + lane], g[l2], acc);
    Bi[l1 * Nf + nu] = acc;
  }
}

// the two halves as separate launches (Gamma chi, then chi Gamma) ...
template <int LMAX>
__global__ void __launch_bounds__(256) k_bse_prep(BsePtrs P, const cplx* __restrict__ chi_ph,
                                                  const cplx* __restrict__ chi_pp, cplx* __restrict__ A, int q_begin,
                                                  int Nz, int Nf, int Nl) {
  prep_gamma_chi<LMAX>(P, chi_ph, chi_pp, A, q_begin, Nz, Nf, Nl, blockIdx.x, gridDim.x);
}
template <int LMAX>
__global__ void __launch_bounds__(256) k_bse_prep_b(BsePtrs P, const cplx* __restrict__ chi_ph,
                                                    const cplx* __restrict__ chi_pp, cplx* __restrict__ B, int q_begin,
                                                    int Nz, int Nf, int Nl) {
  extern __shared__ cplx chs[];
  prep_chi_gamma<LMAX>(P, chi_ph, chi_pp, B, q_begin, Nz, Nf, Nl, blockIdx.x, chs);
}
// ... or as one: the first nA CTAs of an instance's row form Gamma chi, the
// rest chi Gamma, so the instance's Gamma, read by the first, is still in L2
// for the second
template <int LMAX>
__global__ void __launch_bounds__(256) k_bse_prep_ab(BsePtrs P, const cplx* __restrict__ chi_ph,
                                                     const cplx* __restrict__ chi_pp, cplx* __restrict__ A,
                                                     cplx* __restrict__ B, int q_begin, int Nz, int Nf, int Nl,
                                                     int nA) {
  extern __shared__ cplx chs[];
  if ((int)blockIdx.x < nA) prep_gamma_chi<LMAX>(P, chi_ph, chi_pp, A, q_begin, Nz, Nf, Nl, blockIdx.x, nA);
  else prep_chi_gamma<LMAX>(P, chi_ph, chi_pp, B, q_begin, Nz, Nf, Nl, blockIdx.x - nA, chs);
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc, bool valid) {
  unsigned sz = valid ? 16u : 0u;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(sdst)), "l"(gsrc), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D += A*B on 16x8x8 f64 tiles (row.col): a[4], b[2], c[4] per thread
__device__ __forceinline__ void dmma16x8x8(double* c, const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Batched complex GEMM on the FP64 tensor cores with the BSE epilogue.
// CTA tile BM x BN (complex), K step BK; WM x WN warps, warp tile
// (16 TM) x (8 TN).  Left operand L = [A | F] (Nz x 2Nz), right R = [F ; B].
template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool M3>
__global__ void __launch_bounds__(WM* WN * 32) k_bse_gemm(BsePtrs P, const cplx* __restrict__ A,
                                                          const cplx* __restrict__ B, int q_begin, int Nz,
                                                          double one_minus_f) {
  constexpr int TM = BM / WM / 16, TN = BN / WN / 8;
  constexpr int LDL = BM + 2;  // conflict-free 16-byte fragment loads
  constexpr int LDR = BK + 4;
  constexpr int NT = WM * WN * 32;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* sL = reinterpret_cast<cplx*>(smraw);           // [STAGES][BK][LDL]
  cplx* sR = sL + (size_t)STAGES * BK * LDL;           // [STAGES][BN][LDR]

  const int inst = blockIdx.y;
  const int q = q_begin + inst / 4, r = inst % 4;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* Ai = A + n2 * inst;
  const cplx* Bi = B + n2 * inst;
  const cplx* Fq = P.F[r] + n2 * q;
  cplx* Gq = P.G[r] + n2 * q;
  const int tiles_m = (Nz + BM - 1) / BM;
  const int m0 = (blockIdx.x % tiles_m) * BM, n0 = (blockIdx.x / tiles_m) * BN;
  const int K = 2 * Nz;
  const int ktiles = (K + BK - 1) / BK;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % WM) * (16 * TM), wn0 = (warp / WM) * (8 * TN);
  const int gid = lane >> 2, tig = lane & 3;

  auto load_stage = [&](int stage, int kt) {
    const int k0 = kt * BK;
    cplx* dL = sL + (size_t)stage * BK * LDL;
    cplx* dR = sR + (size_t)stage * BN * LDR;
    for (int e = tid; e < BK * BM; e += NT) {
      int m = e % BM, kk = e / BM;
      int gm = m0 + m, gk = k0 + kk;
      bool ok = gm < Nz && gk < K;
      const cplx* src = Ai;
      if (ok) src = gk < Nz ? Ai + gm + (size_t)Nz * gk : Fq + gm + (size_t)Nz * (gk - Nz);
      cp_async16(dL + kk * LDL + m, src, ok);
    }
    for (int e = tid; e < BK * BN; e += NT) {
      int kk = e % BK, n = e / BK;
      int gn = n0 + n, gk = k0 + kk;
      bool ok = gn < Nz && gk < K;
      const cplx* src = Fq;
      if (ok) src = gk < Nz ? Fq + gk + (size_t)Nz * gn : Bi + (gk - Nz) + (size_t)Nz * gn;
      cp_async16(dR + n * LDR + kk, src, ok);
    }
  };

  // M3: three real products per complex one (Gauss): P1 = Ar Br, P2 = Ai Bi,
  // P3 = (Ar + Ai)(Br + Bi); Re = P1 - P2, Im = P3 - P1 - P2.  Otherwise four:
  // Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br (accumulated in p1 = Re, p2 = Im).
  double p1[TM][TN][4], p2[TM][TN][4], p3[M3 ? TM : 1][M3 ? TN : 1][4];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        p1[i][j][e] = p2[i][j][e] = 0.0;
        if (M3) p3[M3 ? i : 0][M3 ? j : 0][e] = 0.0;
      }

#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < ktiles) load_stage(s, s);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; kt++) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      int nk = kt + STAGES - 1;
      if (nk < ktiles) load_stage(nk % STAGES, nk);
      cp_async_commit();
    }
    const cplx* cL = sL + (size_t)(kt % STAGES) * BK * LDL;
    const cplx* cR = sR + (size_t)(kt % STAGES) * BN * LDR;
#pragma unroll
    for (int k8 = 0; k8 < BK; k8 += 8) {
      double are[TM][4], aim[TM][4], anim[TM][4], bre[TN][2], bim[TN][2];
#pragma unroll
      for (int i = 0; i < TM; i++) {
        const int mb = wm0 + i * 16 + gid;
        cplx v0 = cL[(k8 + tig) * LDL + mb];
        cplx v1 = cL[(k8 + tig) * LDL + mb + 8];
        cplx v2 = cL[(k8 + tig + 4) * LDL + mb];
        cplx v3 = cL[(k8 + tig + 4) * LDL + mb + 8];
        are[i][0] = v0.x; aim[i][0] = v0.y;
        are[i][1] = v1.x; aim[i][1] = v1.y;
        are[i][2] = v2.x; aim[i][2] = v2.y;
        are[i][3] = v3.x; aim[i][3] = v3.y;
#pragma unroll
        for (int e = 0; e < 4; e++) anim[i][e] = -aim[i][e];
      }
#pragma unroll
      for (int j = 0; j < TN; j++) {
        const int nb = wn0 + j * 8 + gid;
        cplx w0 = cR[nb * LDR + k8 + tig];
        cplx w1 = cR[nb * LDR + k8 + tig + 4];
        bre[j][0] = w0.x; bim[j][0] = w0.y;
        bre[j][1] = w1.x; bim[j][1] = w1.y;
      }
      if (M3) {
        double asum[TM][4], bsum[TN][2];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int e = 0; e < 4; e++) asum[i][e] = are[i][e] + aim[i][e];
#pragma unroll
        for (int j = 0; j < TN; j++)
#pragma unroll
          for (int e = 0; e < 2; e++) bsum[j][e] = bre[j][e] + bim[j][e];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) {
            dmma16x8x8(p1[i][j], are[i], bre[j]);
            dmma16x8x8(p2[i][j], aim[i], bim[j]);
            dmma16x8x8(p3[M3 ? i : 0][M3 ? j : 0], asum[i], bsum[j]);
          }
      } else {
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
          for (int j = 0; j < TN; j++) {
            dmma16x8x8(p1[i][j], are[i], bre[j]);
            dmma16x8x8(p1[i][j], anim[i], bim[j]);
            dmma16x8x8(p2[i][j], are[i], bim[j]);
            dmma16x8x8(p2[i][j], aim[i], bre[j]);
          }
      }
    }
  }
  cp_async_wait<0>();
  double cre[TM][TN][4], cim[TM][TN][4];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        if (M3) {
          cre[i][j][e] = p1[i][j][e] - p2[i][j][e];
          cim[i][j][e] = p3[M3 ? i : 0][M3 ? j : 0][e] - p1[i][j][e] - p2[i][j][e];
        } else {
          cre[i][j][e] = p1[i][j][e];
          cim[i][j][e] = p2[i][j][e];
        }
      }

  // epilogue: Phi = s * C + (1-f) (F - Gamma), written over Gamma
  const double s = P.scale[r];
#pragma unroll
  for (int i = 0; i < TM; i++)
#pragma unroll
    for (int j = 0; j < TN; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        int row = m0 + wm0 + i * 16 + gid + (e >= 2 ? 8 : 0);
        int col = n0 + wn0 + j * 8 + 2 * tig + (e & 1);
        if (row < Nz && col < Nz) {
          size_t idx = row + (size_t)Nz * col;
          cplx f = Fq[idx], g = Gq[idx];
          Gq[idx] = cmk(s * cre[i][j][e] + one_minus_f * (f.x - g.x), s * cim[i][j][e] + one_minus_f * (f.y - g.y));
        }
      }
}

template <int BM, int BN, int BK, int WM, int WN, int STAGES, bool M3>
static int run_gemm(tups_ctx* ctx, const BsePtrs& P, int q_begin, int q_count) {
  const int Nz = ctx->d.Nz;
  constexpr int LDL = BM + 2, LDR = BK + 4;
  size_t sm = (size_t)STAGES * (BK * LDL + BN * LDR) * sizeof(cplx);
  auto kern = k_bse_gemm<BM, BN, BK, WM, WN, STAGES, M3>;
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_bse_gemm smem attribute");
  }
  int tiles = ((Nz + BM - 1) / BM) * ((Nz + BN - 1) / BN);
  dim3 grid(tiles, 4 * q_count);
  kern<<<grid, WM * WN * 32, sm, ctx->stream>>>(P, ctx->s.bse_A, ctx->s.bse_B, q_begin, Nz,
                                                1.0 - ctx->p.f_damping);
  return after_launch(ctx, "k_bse_gemm");
}

// Tile candidates of the FP64 BSE GEMM for Nz >= 32, all with three real
// products per complex one: they differ in CTA tile, warps and pipeline
// depth, never in the order of any element's K sum, so every candidate
// writes the same bits.  Index 0 is the choice measured best on a B200 before
// the tuner existed: 32 x 32 tiles of 4 warps (16 x 16 each), two cp.async
// stages (38 KB of shared memory, 5 CTAs per SM): 8x8 / Nl = 5 (Nz = 160)
// 1.79 ms, against 1.93 ms with three stages, 2.01 ms with BK = 32 and
// 2.13 ms with four products; 16x16 / Nl = 9 (Nz = 576) 480 ms, against
// 541 ms for 64 x 64 tiles of 8 warps with four products, 656 ms with three.
struct BseCand {
  const char* name;
  int (*run)(tups_ctx*, const BsePtrs&, int, int);
};
static const BseCand kBseCands[] = {
    {"32x32x16_w2x2_s2", run_gemm<32, 32, 16, 2, 2, 2, true>},
    {"32x32x16_w2x2_s3", run_gemm<32, 32, 16, 2, 2, 3, true>},
    {"64x32x16_w4x2_s2", run_gemm<64, 32, 16, 4, 2, 2, true>},
    {"32x64x16_w2x4_s2", run_gemm<32, 64, 16, 2, 4, 2, true>},
    {"32x32x32_w2x2_s2", run_gemm<32, 32, 32, 2, 2, 2, true>},
};
constexpr int kNumBseCands = sizeof(kBseCands) / sizeof(kBseCands[0]);

// The candidate for this Nz: cached, or timed now on the first chunk's
// operands (q_begin = 0) with the GEMM writing into scratch copies of the
// chunk's Gamma, so the call's own result is untouched.
static int bse_choice(tups_ctx* ctx, const BsePtrs& P, int q_begin, int q_count, int* choice) {
  const int Nz = ctx->d.Nz;
  const std::string key = "k_bse_gemm Nz=" + std::to_string(Nz);
  *choice = 0;
  std::vector<std::string> names;
  for (int c = 0; c < kNumBseCands; c++) names.push_back(kBseCands[c].name);
  const int forced = tune_forced(key, names);
  if (forced >= 0) {
    *choice = forced;
    return TUPS_OK;
  }
  if (!ctx->autotune || tune_get(key, choice)) return TUPS_OK;
  if (q_begin != 0 || !tune_allowed(ctx)) return TUPS_OK;
  // enough instances for several waves of the smallest tiles
  const long long tiles32 = (long long)((Nz + 31) / 32) * ((Nz + 31) / 32);
  const int qt = (int)std::min<long long>(q_count, std::max<long long>(1, (3000 + 4 * tiles32 - 1) / (4 * tiles32)));
  const size_t n2 = (size_t)Nz * Nz;
  cplx* scratch = nullptr;
  int rc = cuda_check(ctx, cudaMalloc(&scratch, 4 * (size_t)qt * n2 * sizeof(cplx)), "tuner scratch");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaMemsetAsync(scratch, 0, 4 * (size_t)qt * n2 * sizeof(cplx), ctx->stream), "tuner scratch");
  BsePtrs T = P;
  for (int r = 0; r < 4; r++) T.G[r] = scratch + (size_t)r * qt * n2;
  if (!rc)
    rc = tune_pick(ctx, key, kNumBseCands, names, [&](int c) { return kBseCands[c].run(ctx, T, 0, qt); }, 2,
                   choice);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  cudaFree(scratch);
  if (!rc && e != cudaSuccess) rc = cuda_check(ctx, e, "tuner");
  return rc;
}

// Slices of the split GEMM for the next BSE call; 0 = FP64 tensor cores.
// Fixed mode: bse_slices.  Ladder: the accuracy needed is chosen from the last
// relative Sigma change r so that the GEMM error (about 10^(1.1 - 2 s) of
// max|A| max|B| K) stays two decades below it, s_req = ceil((3.1 - log10 r)/2)
// (3 before the first conv); the online tuner then takes the faster of FP64
// and s_req slices, from device times of earlier BSE calls.  FP64 is timed on
// the first call; a slice count is tried once unless a smaller one already
// proved no faster than FP64 (the cost grows with s).
int current_bse_slices(const tups_ctx* ctx) {
  if (!ctx->precision_ladder) return ctx->bse_slices;
  const double* tms = ctx->use_graph ? ctx->tune_graph_ms : ctx->tune_ms;
  const double r = ctx->last_dsigma_rel;
  int s_req = 3;
  if (r == 0.0) s_req = 9;
  else if (r > 0.0) s_req = std::max(2, (int)std::ceil((3.1 - std::log10(r)) / 2.0));
  if (s_req > 8) return 0;
  if (tms[0] < 0.0) return 0;
  if (tms[s_req] >= 0.0) return tms[s_req] < tms[0] ? s_req : 0;
  // not measured yet: the cost grows with s, so a measured s' <= s_req that
  // was no faster than FP64 rules s_req out; otherwise try it once
  for (int s = 2; s < s_req; s++)
    if (tms[s] >= 0.0 && tms[s] >= tms[0]) return 0;
  return s_req;
}

void bse_tune_collect(tups_ctx* ctx) {
  if (ctx->tune_pending < 0) return;
  float ms = 0.0f;
  if (cudaEventElapsedTime(&ms, ctx->tune_ev[0], ctx->tune_ev[1]) == cudaSuccess) {
    double& slot = (ctx->use_graph ? ctx->tune_graph_ms : ctx->tune_ms)[ctx->tune_pending];
    slot = slot < 0.0 ? ms : 0.5 * (slot + ms);
  } else {
    cudaGetLastError();
  }
  ctx->tune_pending = -1;
}

// Split-precision GEMM [Gamma chi | F] [F ; chi Gamma] for the chunk, in
// sub-chunks that fit the int8 workspace; same epilogue as k_bse_gemm.
static int run_split(tups_ctx* ctx, const BsePtrs& P, int q_begin, int q_count, int slices) {
  const int Nz = ctx->d.Nz;
  if (!ctx->oz_work) {
    // workspace for up to 8 slices, bounded to 8 GiB
    const size_t per = oz_work_layout(4, Nz, Nz, 2 * Nz, 8).total / 4 + 1;
    size_t cap = ((size_t)8 << 30) / per;
    cap = std::max<size_t>(4, std::min<size_t>(cap, ctx->s.bse_chunk)) / 4 * 4;
    const size_t bytes = oz_work_layout((int)cap, Nz, Nz, 2 * Nz, 8).total;
    cudaError_t e = cudaMalloc(&ctx->oz_work, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      ctx->oz_work = nullptr;
      return set_error(ctx, TUPS_ERR_OOM, "split-precision BSE workspace");
    }
    ctx->allocations.push_back(ctx->oz_work);
    ctx->oz_cap = cap;
  }
  const int n_inst = 4 * q_count;
  for (int i0 = 0; i0 < n_inst; i0 += (int)ctx->oz_cap) {
    const int nb = std::min<int>((int)ctx->oz_cap, n_inst - i0);
    OzRun R;
    R.batch = nb;
    R.M = Nz;
    R.N = Nz;
    R.s = slices;
    const int qb = q_begin + i0 / 4;
    // [Gamma chi | F] and [F ; chi Gamma] from k_bse_prep's products and F_r
    OzOperand A{}, B{};
    A.p1 = ctx->s.bse_A + (size_t)Nz * Nz * i0;
    A.s1 = (long long)Nz * Nz;
    A.ld1 = Nz;
    A.K1 = Nz;
    A.bse2 = 1;
    A.ld2 = Nz;
    A.K2 = Nz;
    B.bse1 = 1;
    B.ld1 = Nz;
    B.K1 = Nz;
    B.p2 = ctx->s.bse_B + (size_t)Nz * Nz * i0;
    B.s2 = (long long)Nz * Nz;
    B.ld2 = Nz;
    B.K2 = Nz;
    for (int r = 0; r < 4; r++) A.F[r] = B.F[r] = P.F[r];
    A.q_begin = B.q_begin = qb;
    A.Nz = B.Nz = Nz;
    R.A = A;
    R.B = B;
    oz_bind_work(R, oz_work_layout(nb, Nz, Nz, 2 * Nz, slices), ctx->oz_work);
    R.status = ctx->s.scal + S_STATUS;
    R.status_code = (double)TUPS_ERR_TIMEOUT;
    R.epi = 1;
    for (int r = 0; r < 4; r++) {
      R.F[r] = P.F[r];
      R.G[r] = P.G[r];
      R.scale[r] = P.scale[r];
    }
    R.omf = 1.0 - ctx->p.f_damping;
    R.q_begin = qb;
    int rc = oz_run(R, ctx->stream, &ctx->launches);
    if (rc) return set_error(ctx, rc, "split-precision BSE launch failed");
  }
  return TUPS_OK;
}

// BSE prep launch forms (same bits): 0 = two launches, 1 = one launch
static int prep_run(tups_ctx* ctx, const BsePtrs& P, int q_begin, int q_count, int form) {
  const auto& d = ctx->d;
  const int nA = (int)std::min<size_t>(cdiv((size_t)d.Nz * d.Nf, 256), 4096);
  const int nB = (int)(cdiv(d.Nf, 32) * cdiv(d.Nz, 8));
  const size_t smb = (size_t)d.Nl * d.Nl * 33 * sizeof(cplx);
  const int L = d.Nl <= 1 ? 1 : d.Nl <= 5 ? 5 : d.Nl <= 9 ? 9 : d.Nl <= 13 ? 13 : 16;
  auto attr = [&](const void* fn) {
    if (smb <= 48 * 1024) return TUPS_OK;
    return cuda_check(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb),
                      "k_bse_prep smem attribute");
  };
  if (form == 1) {
    auto ab = L == 1 ? k_bse_prep_ab<1> : L == 5 ? k_bse_prep_ab<5> : L == 9 ? k_bse_prep_ab<9>
            : L == 13 ? k_bse_prep_ab<13> : k_bse_prep_ab<16>;
    int rc = attr((const void*)ab);
    if (rc) return rc;
    ab<<<dim3(nA + nB, 4 * q_count), 256, smb, ctx->stream>>>(P, ctx->s.chi_ph, ctx->s.chi_pp, ctx->s.bse_A,
                                                               ctx->s.bse_B, q_begin, d.Nz, d.Nf, d.Nl, nA);
    return after_launch(ctx, "k_bse_prep_ab");
  }
  auto pa = L == 1 ? k_bse_prep<1> : L == 5 ? k_bse_prep<5> : L == 9 ? k_bse_prep<9>
          : L == 13 ? k_bse_prep<13> : k_bse_prep<16>;
  pa<<<dim3(nA, 4 * q_count), 256, 0, ctx->stream>>>(P, ctx->s.chi_ph, ctx->s.chi_pp, ctx->s.bse_A, q_begin, d.Nz,
                                                      d.Nf, d.Nl);
  int rc = after_launch(ctx, "k_bse_prep");
  if (rc) return rc;
  auto pb = L == 1 ? k_bse_prep_b<1> : L == 5 ? k_bse_prep_b<5> : L == 9 ? k_bse_prep_b<9>
          : L == 13 ? k_bse_prep_b<13> : k_bse_prep_b<16>;
  rc = attr((const void*)pb);
  if (rc) return rc;
  pb<<<dim3(nB, 4 * q_count), 256, smb, ctx->stream>>>(P, ctx->s.chi_ph, ctx->s.chi_pp, ctx->s.bse_B, q_begin, d.Nz,
                                                        d.Nf, d.Nl);
  return after_launch(ctx, "k_bse_prep_b");
}

// Gamma chi and chi Gamma for one chunk; the launch form is a tuner choice
// per shape, timed on the first chunk's own operands (the prep writes only
// the scratch A and B, so running it more than once is harmless)
static int prep_chunk(tups_ctx* ctx, const BsePtrs& P, int q_begin, int q_count) {
  const auto& d = ctx->d;
  if (d.Nl > 16) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 16 not supported by k_bse_prep");
  if (4 * q_count > 65535) return set_error(ctx, TUPS_ERR_BADDIM, "k_bse_prep: more than 16383 slots in a chunk");
  const std::string key = "k_bse_prep Nz=" + std::to_string(d.Nz) + " Nl=" + std::to_string(d.Nl);
  const std::vector<std::string> names = {"two_launches", "one_launch"};
  int choice = 0;
  const int forced = tune_forced(key, names);
  if (forced >= 0) {
    choice = forced;
  } else if (ctx->autotune && !tune_get(key, &choice) && q_begin == 0 && tune_allowed(ctx)) {
    int rc = tune_pick(ctx, key, (int)names.size(), names,
                       [&](int c) { return prep_run(ctx, P, q_begin, q_count, c); }, 2, &choice);
    if (rc) return rc;
  }
  return prep_run(ctx, P, q_begin, q_count, choice);
}

int launch_bse_chunk(tups_ctx* ctx, int q_begin, int q_count) {
  const auto& d = ctx->d;
  BsePtrs P;
  const double a = 1.0 / (ctx->p.beta * d.Nx * d.Ny);
  const double c[4] = {0.5, 0.5, -0.25, 0.25};
  for (int r = 0; r < 4; r++) {
    P.F[r] = ctx->s.F[r];
    P.G[r] = ctx->s.G[r];
    P.scale[r] = c[r] * ctx->p.f_damping * a;
  }
  const int slices = ctx->cur_slices;
  if (d.Nl > 16) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 16 not supported by k_bse_prep");
  if (4 * q_count > 65535) return set_error(ctx, TUPS_ERR_BADDIM, "k_bse_prep: more than 16383 slots in a chunk");
  phase_begin(ctx, TUPS_PHASE_BSE_PREP);
  int rc = prep_chunk(ctx, P, q_begin, q_count);
  phase_end(ctx, TUPS_PHASE_BSE_PREP);
  if (rc) return rc;
  if (slices > 0) {
    phase_begin(ctx, TUPS_PHASE_BSE_GEMM);
    rc = run_split(ctx, P, q_begin, q_count, slices);
    phase_end(ctx, TUPS_PHASE_BSE_GEMM);
    return rc;
  }
  phase_begin(ctx, TUPS_PHASE_BSE_GEMM);
  if (d.Nz >= 32) {
    int choice = 0;
    rc = bse_choice(ctx, P, q_begin, q_count, &choice);
    if (!rc) rc = kBseCands[choice].run(ctx, P, q_begin, q_count);
  } else {
    rc = run_gemm<16, 16, 16, 1, 2, 3, true>(ctx, P, q_begin, q_count);
  }
  phase_end(ctx, TUPS_PHASE_BSE_GEMM);
  return rc;
}

}  // namespace tups
