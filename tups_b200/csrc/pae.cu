// Parquet equation: calculate_PAE (SRC/parquet_EQOuter.f90:16-118) with the
// eight crossing contributions of SRC/parquet_EQContribs.f90:44-524.
//
// The reference loops over source channel and w2 and scatter-adds every
// contribution into F.  Here the loop is turned around (output-stationary).
// For a target element F_a/F_b[(l1,nu1),(l2,nu2), q] (W = bosonic index of q,
// 1-based frequencies, d = nu2 - nu1, s = nu1 + nu2, nh = Nf/2) the eight
// calls group into two families per target pair, and inside a family at
// most ONE (call, w2) reaches the element:
//
//  pair (F_d, F_m):
//   D  phbar_to_ph     w2 = d + 1 >= 1,        Phi_R[(l3,nu1),(l4,pick(nu1+W-1))]
//      phbar_to_ph_TR  w2 = 1 - d >= 2,        conj Phi_R[(l3,mF(nu1)),(l4,pick(Nf+2-nu1-W))]
//   A  pp_to_ph        w2 = s + W - Nf - 1 >= 1, Phi_R[(l3,nu1),(l4,nu2)]
//      pp_to_ph_TR     w2 = Nf + 3 - s - W >= 2, conj Phi_R[(l3,mF(nu1)),(l4,mF(nu2))]
//  pair (F_s, F_t):
//   A  ph_to_pp        w2 = W + Nf + 1 - s >= 1, Phi_R[(l3,nu1),(l4,nu2)]
//      ph_to_pp_TR     w2 = s - W - Nf + 1 >= 2, conj Phi_R[(l3,mF(nu1)),(l4,mF(nu2))]
//   D  phbar_to_pp     w2 = d + 1 >= 1,        Phi_R[(l3,nu1),(l4,pick(W+Nf-nu2))]
//      phbar_to_pp_TR  w2 = 1 - d >= 2,        conj Phi_R[(l3,mF(nu1)),(l4,pick(nu2-W+1))]
//
// (w2 <= nh always; mF(x) = Nf+1-x; pick = clamp to [1, Nf]; TR terms carry
// signs(l3) signs(l4)).  Both calls of a family use the same crossing tensor
// M and the same two source channels, combined with the dispatch factors of
// SRC/parquet_EQOuter.f90:84-113 as they are gathered.  So per (q, pair) the
// whole parquet equation is ONE complex GEMM
//     C^T[(target, element), (l1,l2)] = X^T[(target, element), (family,l3,l4,R)] M^T
// run on the FP64 tensor cores (mma.sync m16n8k8), with X gathered from
// Phi(R) on load and F = Phi + Lambda*Nc + C/Nx: a base pass writes
// Phi + Lambda*Nc, and each family pass adds C/Nx to the elements it reaches
// by reductions in L2, each element at most once per pass, so the result
// does not depend on the order of the CTAs (deterministic).
#include <string>

#include "tups_device.cuh"

namespace tups {

struct PaePtrs {
  const cplx* Phi[4];   // Phi_r (G arrays after the BSE), (Nz, Nz, Nb)
  const cplx* PhiR[4];  // (Nz*Nz, Nf/2, NR)
  const cplx* M[4];     // (Nl^4, NIBZ, NR): 0 phbar_to_ph 1 pp_to_ph 2 ph_to_pp 3 phbar_to_pp
  const cplx* L[4];     // (Nf, Nf, Nf/2)
  cplx* F[4];
};

__host__ __device__ __forceinline__ int clampnu(int x, int Nf) { return x < 1 ? 1 : (x > Nf ? Nf : x); }

// dispatch factors [pair][family][source][target] of SRC/parquet_EQOuter.f90:84-113:
// pair 0: D = phbar_to_ph from (d, m), A = pp_to_ph from (s, t);
// pair 1: D = phbar_to_pp from (d, m), A = ph_to_pp from (d, m)
__constant__ double c_pae_fac[2][2][2][2] = {{{{-0.5, -0.5}, {-1.5, 0.5}}, {{0.5, -0.5}, {1.5, 0.5}}},
                                             {{{0.5, -0.5}, {-1.5, -0.5}}, {{0.5, 0.5}, {-1.5, 0.5}}}};

// Frequency map of family fam (0 = D, 1 = A) of target pair `pair` at the
// element (nu1, nu2).  Returns false when the family does not reach it.
__host__ __device__ __forceinline__ bool pae_family(int pair, int fam, int nu1, int nu2, int W, int Nf, int* w2,
                                                    int* a, int* b, int* tr) {
  const int nh = Nf / 2;
  const int d = nu2 - nu1, s = nu1 + nu2;
  int ww;
  if (fam == 0) {  // diagonal families: phbar_to_ph (pair 0) / phbar_to_pp (pair 1)
    if (d >= 0) {
      ww = d + 1;
      if (ww > nh) return false;
      *tr = 0;
      *a = nu1;
      *b = pair == 0 ? clampnu(nu1 + W - 1, Nf) : clampnu((W - 1) - (nu1 + ww - 1) + Nf + 1, Nf);
    } else {
      ww = 1 - d;
      if (ww > nh) return false;
      *tr = 1;
      *a = Nf + 1 - nu1;
      *b = pair == 0 ? clampnu(Nf + 2 - nu1 - W, Nf) : clampnu(nu1 - (W + ww - 1) + 1, Nf);
    }
  } else if (pair == 0) {  // pp_to_ph
    ww = s + W - Nf - 1;
    if (ww >= 1) {
      if (ww > nh) return false;
      *tr = 0;
      *a = nu1;
      *b = nu2;
    } else {
      ww = Nf + 3 - s - W;
      if (ww < 2 || ww > nh) return false;
      *tr = 1;
      *a = Nf + 1 - nu1;
      *b = Nf + 1 - nu2;
    }
  } else {  // ph_to_pp
    ww = W + Nf + 1 - s;
    if (ww >= 1) {
      if (ww > nh) return false;
      *tr = 0;
      *a = nu1;
      *b = nu2;
    } else {
      ww = s - W - Nf + 1;
      if (ww < 2 || ww > nh) return false;
      *tr = 1;
      *a = Nf + 1 - nu1;
      *b = nu1 - (W + ww - 1) + 1;
    }
  }
  *w2 = ww;
  return true;
}

__device__ __forceinline__ unsigned smem_u32p(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16p(void* sdst, const void* gsrc, bool valid) {
  unsigned sz = valid ? 16u : 0u;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32p(sdst)), "l"(gsrc), "r"(sz));
}
__device__ __forceinline__ void dmma_16x8x8(double* c, const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

#ifndef PAE_MIN_BLOCKS
#define PAE_MIN_BLOCKS 3  // CTAs per SM asked of ptxas for the 8-warp, <= 2 n-tile configs (2 beyond)
#endif
constexpr int PAE_BK = 16;
// M^T stage row pitch [k][n] in complex entries: BN + 2, so that a warp's
// fragment reads (k = k8 + tig, n = .. + gid) fall in distinct banks and a
// K row is copied by consecutive threads from consecutive columns of M
__host__ __device__ constexpr int pae_ldn(int bn) { return bn + 2; }

// Element lists: for target pair p, family f and bosonic index W the
// elements (nu1, nu2) the family reaches, packed as int4
// {nu1 + 256 nu2, w2, a, b + 65536 tr}; capacity Nf^2 per list.
__host__ __device__ __forceinline__ int pae_list(int pair, int fam, int W, int nh) {
  return (pair * 2 + fam) * nh + (W - 1);
}

// F_r = Phi_r + Lambda_r * aux on the (l=1, l=1) block, all r and slots
__global__ void k_pae_base(PaePtrs P, const int* __restrict__ ibz, int Nz, int Nf, int Nb, double aux) {
  const size_t n2 = (size_t)Nz * Nz;
  const size_t n = n2 * Nb;
  const int r = blockIdx.y;
  // constant indices keep the parameter struct out of local memory
  const cplx* Phi = r == 0 ? P.Phi[0] : r == 1 ? P.Phi[1] : r == 2 ? P.Phi[2] : P.Phi[3];
  const cplx* L = r == 0 ? P.L[0] : r == 1 ? P.L[1] : r == 2 ? P.L[2] : P.L[3];
  cplx* F = r == 0 ? P.F[0] : r == 1 ? P.F[1] : r == 2 ? P.F[2] : P.F[3];
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    cplx f = __ldcs(Phi + e);
    const int i = (int)(e % Nz), j = (int)((e / Nz) % Nz);
    if (i < Nf && j < Nf) {
      const int q = (int)(e / n2);
      const int W = ibz[3 * q + 2];
      const cplx lam = L[(size_t)i + (size_t)Nf * (j + (size_t)Nf * (W - 1))];
      f = cadd(f, cscale(lam, aux));
    }
    F[e] = f;
  }
}

// One CTA per (tile of E = 8 RW listed elements, target pair x column chunk, q)
// for one family: C^T[(target, element), (l1,l2)] = X^T[(target, element), (l3,l4,R)] M^T
// and F_target += C / Nx.  Warps: RW along rows (16 rows each) x WN along
// the (l1,l2) columns, TN n8 tiles each; BN = 8 TN WN >= Nl^2 (or a chunk).
// Columns: QN > 0 puts QN IBZ momenta side by side, (momentum, (l1, l2)),
// one group per blockIdx.x; QN = 0 numbers the columns (momentum, (l1, l2))
// of all the context's momenta flat and tiles them by BN regardless of
// momentum boundaries, so only the last tile pads (Nl^2 = 81 at 45 momenta:
// 3645 columns in 38 tiles of 96, against 45 tiles of 96 with 81 used).
// The X operand is copied raw: cp.async brings the Phi(R) entries of the two
// source channels for the K step STG-1 ahead into shared memory, and the
// dispatch factors, the time-reversal conjugation and its form-factor sign
// are applied when the MMA fragments are read, so no warp waits on a gather
// between K steps.  The per-k offsets into Phi(R) and the signs s(l3) s(l4)
// are tabulated once per CTA.
// G3: three real DMMA products per complex one (P1 = Xr Mr, P2 = Xi Mi,
// P3 = (Xr + Xi)(Mr + Mi); Re = P1 - P2, Im = P3 - P1 - P2), else four.
// PRE: once a stage has landed, the CTA rewrites its raw (source, k, element)
// X entries in place as (target, k, element) operands, dispatch factors,
// conjugation and sign applied (the same operations in the same order as
// the per-fragment form, so the same bits), behind a second barrier; the
// MMA warps then load finished fragments.
template <int TN, int WN, int RW, int STG, int QN, bool G3 = false, bool PRE = false>
__global__ void __launch_bounds__(32 * RW * WN, RW * WN == 8 ? (TN <= 2 ? PAE_MIN_BLOCKS : 2) : 1)
    k_pae_mma(PaePtrs P, const int4* __restrict__ elems, const int* __restrict__ counts,
              const int* __restrict__ ibz, const int* __restrict__ signs, int Nz, int Nf, int Nl, int NIBZ, int NR,
              int nchunks, int fam, int Kpad, int slot0, int Nb, double inv_nx) {
  constexpr int BN = 8 * TN * WN;
  constexpr int NT = 32 * RW * WN;
  constexpr int E = 8 * RW;      // listed elements per CTA
  constexpr int LDX = E + 2;     // elements + pad
  constexpr int LDN = pae_ldn(BN);
  static_assert(E % 16 == 0, "a warp's 16 rows must share one target");
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* sX = reinterpret_cast<cplx*>(smraw);                                  // [STG][2][BK][LDX]
  cplx* sB = sX + (size_t)STG * 2 * PAE_BK * LDX;                             // [STG][BK][LDN]
  long long* koff = reinterpret_cast<long long*>(sB + (size_t)STG * PAE_BK * LDN);  // [Kpad]
  double* ksg = reinterpret_cast<double*>(koff + Kpad);                       // [Kpad]
  // M^T offsets, split as (k part) + (column part); -1 marks a zero fill
  // (M holds Nl^4 NIBZ NR < 2^31 entries: checked at launch)
  int* bko = reinterpret_cast<int*>(ksg + Kpad);                              // [Kpad]
  int* bco = bko + Kpad;                                                      // [BN]
  __shared__ long long e_off[E];
  __shared__ int e_ok[E], e_tr[E];
  __shared__ int erow[E];        // output offset (nu1-1) + Nz (nu2-1), -1 past the list
  __shared__ long long ecol[BN];  // output offset of column n (l1, l2, slot), -1 if not written

  // grid (Q, tile x pair x chunk, w): the CTAs in flight are the IBZ momenta of
  // one element tile, so they gather the same Phi(R) entries (Phi(R) does not
  // depend on Q) and L2 serves all but the first
  const int pc = blockIdx.y % (2 * nchunks), tile = blockIdx.y / (2 * nchunks);
  const int pair = pc / nchunks, chunk = pc % nchunks;
  // blockIdx.x runs over groups of QN IBZ momenta among those that hold this
  // context's slots (QN > 0), or over flat column tiles (QN = 0); the
  // momenta sit side by side in the columns (momentum, (l1, l2)), so X
  // serves all of them
  const int nh = Nf / 2;
  const int w = blockIdx.z;
  const int nl2 = Nl * Nl;
  const int Qhi = (slot0 + Nb - 1) / nh;
  const int Q0 = slot0 / nh + (QN > 0 ? blockIdx.x * QN : 0);
  const int col0 = QN > 0 ? chunk * BN : blockIdx.x * BN;  // first column of the CTA, relative to Q0
  auto local_slot = [&](int iq) {  // local index of slot (Q0 + iq, w), or -1
    const int lq = (Q0 + iq) * nh + w - slot0;
    return ((QN == 0 || iq < QN) && Q0 + iq <= Qhi && lq >= 0 && lq < Nb) ? lq : -1;
  };
  bool any = false;
  for (int iq = col0 / nl2; iq <= (col0 + BN - 1) / nl2; iq++) any = any || local_slot(iq) >= 0;
  if (!any) return;
  const int W = ibz[3 * (Q0 * nh + w) + 2];  // the bosonic index of w, the same for every Q
  const int list = pae_list(pair, fam, W, nh);
  const int cnt = counts[list];
  const int e0 = tile * E;
  if (e0 >= cnt) return;
  const int nl4 = nl2 * nl2;
  const int K = nl2 * NR;
  const size_t n2 = (size_t)Nz * Nz;
  const int tid = threadIdx.x;

  if (tid < E) {
    int4 rec = make_int4(0, 0, 1, 1);
    if (e0 + tid < cnt) rec = elems[(size_t)list * Nf * Nf + e0 + tid];
    const int w2 = rec.y, a = rec.z, b = rec.w & 65535;
    erow[tid] = e0 + tid < cnt ? ((rec.x & 255) - 1) + Nz * ((rec.x >> 8) - 1) : -1;
    e_ok[tid] = w2 != 0;
    e_tr[tid] = rec.w >> 16;
    // element part of the Phi(R) index (a-1) + Nz (b-1) + Nz^2 (w2-1)
    e_off[tid] = w2 != 0 ? (long long)(a - 1) + (long long)Nz * (b - 1) + (long long)n2 * (w2 - 1) : 0;
  }
  // k part of the index l3 Nf + Nz l4 Nf + Nz^2 (Nf/2) R, and s(l3) s(l4)
  for (int k = tid; k < Kpad; k += NT) {
    long long off = 0;
    double sg = 1.0;
    if (k < K) {
      const int l34 = k % nl2, R = k / nl2;
      const int l3 = l34 % Nl, l4 = l34 / Nl;
      off = (long long)l3 * Nf + (long long)Nz * l4 * Nf + (long long)n2 * nh * R;
      sg = (double)(signs[l3] * signs[l4]);
    }
    koff[k] = off;
    ksg[k] = sg;
    bko[k] = k < K ? nl2 * (k % nl2) + nl4 * NIBZ * (k / nl2) : -1;
  }
  for (int n = tid; n < BN; n += NT) {
    const int nn = col0 + n;
    const int iq = QN == 1 ? 0 : nn / nl2;
    const int col = nn - iq * nl2;
    const bool ok = col < nl2 && (QN == 0 || iq < QN) && Q0 + iq <= Qhi;
    bco[n] = ok ? col + nl4 * (Q0 + iq) : -1;
    const int lq = col < nl2 ? local_slot(iq) : -1;
    ecol[n] = lq >= 0 ? (long long)((col % Nl) * Nf) + (long long)Nz * ((col / Nl) * Nf) + (long long)n2 * lq : -1;
  }
  // dispatch factors fac[source][target] of this family (SRC/parquet_EQOuter.f90:84-113)
  const double f00 = c_pae_fac[pair][fam][0][0], f01 = c_pae_fac[pair][fam][0][1];
  const double f10 = c_pae_fac[pair][fam][1][0], f11 = c_pae_fac[pair][fam][1][1];
  // constant indices keep the parameter struct out of local memory
  const cplx* Mf = pair == 0 ? (fam == 0 ? P.M[0] : P.M[1]) : (fam == 0 ? P.M[3] : P.M[2]);
  // sources: (d, m), except pp_to_ph from (s, t)
  const bool st_src = fam == 1 && pair == 0;
  const cplx* X0 = st_src ? P.PhiR[2] : P.PhiR[0];
  const cplx* X1 = st_src ? P.PhiR[3] : P.PhiR[1];
  __syncthreads();

  // one K step: raw X (2 sources x BK x E) and M^T (BN x BK), zero-filled
  // outside K, past the list and for columns beyond Nl^2
  auto load_stage = [&](int stage, int kt) {
    cplx* dX = sX + (size_t)stage * 2 * PAE_BK * LDX;
    for (int p = tid; p < 2 * E * PAE_BK; p += NT) {
      const int e = p % E, rest = p / E;
      const int kk = rest % PAE_BK, src = rest / PAE_BK;
      const int k = kt * PAE_BK + kk;
      const bool ok = k < K && e_ok[e];
      const cplx* g = src ? X1 : X0;
      cp_async16p(dX + (src * PAE_BK + kk) * LDX + e, ok ? g + e_off[e] + koff[k] : g, ok);
    }
    cplx* dB = sB + (size_t)stage * PAE_BK * LDN;
    for (int p = tid; p < BN * PAE_BK; p += NT) {
      const int n = p % BN, kk = p / BN;
      const int bk = bko[kt * PAE_BK + kk], bc = bco[n];
      const bool ok = bk >= 0 && bc >= 0;
      cp_async16p(dB + kk * LDN + n, ok ? Mf + bk + bc : Mf, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };

  const int lane = tid & 31, warp = tid >> 5;
  const int wr = warp % RW, wc = warp / RW;
  const int gid = lane >> 2, tig = lane & 3;
  const int tgt = (wr * 16) / E;            // the warp's target channel
  const int er = (wr * 16) % E + gid;       // its elements er and er + 8
  const double fa = tgt == 0 ? f00 : f01, fb = tgt == 0 ? f10 : f11;
  const bool tr0 = e_tr[er] != 0, tr1 = e_tr[er + 8] != 0;
  // four products: cre, cim; three: P1 in cre, P2 in cim, P3 in c3
  double cre[TN][4], cim[TN][4], c3[G3 ? TN : 1][4];
#pragma unroll
  for (int j = 0; j < TN; j++)
#pragma unroll
    for (int x = 0; x < 4; x++) {
      cre[j][x] = cim[j][x] = 0.0;
      if (G3) c3[G3 ? j : 0][x] = 0.0;
    }

  // fragment value of element e at k: fa x0 + fb x1, conjugated with sign
  // s(l3) s(l4) for time-reversed elements
  auto combine = [](cplx x0, cplx x1, double a, double b, bool trv, double sg) {
    double re = __fma_rn(b, x1.x, __dmul_rn(a, x0.x));
    double im = __fma_rn(b, x1.y, __dmul_rn(a, x0.y));
    if (trv) {
      re = sg * re;
      im = -sg * im;
    }
    return cmk(re, im);
  };
  auto xval = [&](const cplx* cX, int kk, int e, bool trv, double sg, double& re, double& im) {
    if (PRE) {  // already combined: target tgt's operand at row tgt
      const cplx t = cX[(tgt * PAE_BK + kk) * LDX + e];
      re = t.x;
      im = t.y;
    } else {
      const cplx t = combine(cX[kk * LDX + e], cX[(PAE_BK + kk) * LDX + e], fa, fb, trv, sg);
      re = t.x;
      im = t.y;
    }
  };

  const int kt_hi = Kpad / PAE_BK;
#pragma unroll
  for (int st = 0; st < STG - 1; st++) {
    if (st < kt_hi) load_stage(st, st);
    else asm volatile("cp.async.commit_group;\n" ::);
  }
  for (int kt = 0; kt < kt_hi; kt++) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(STG - 2));
    __syncthreads();
    {
      const int nk = kt + STG - 1;
      if (nk < kt_hi) load_stage(nk % STG, nk);
      else asm volatile("cp.async.commit_group;\n" ::);
    }
    cplx* cX = sX + (size_t)(kt % STG) * 2 * PAE_BK * LDX;
    const cplx* cB = sB + (size_t)(kt % STG) * PAE_BK * LDN;
    if (PRE) {
      // (source 0, source 1) at (k, e) -> (target 0, target 1) at (k, e):
      // each thread rewrites the entries it read
      for (int p = tid; p < E * PAE_BK; p += NT) {
        const int e = p % E, kk = p / E;
        const cplx x0 = cX[kk * LDX + e], x1 = cX[(PAE_BK + kk) * LDX + e];
        const bool trv = e_tr[e] != 0;
        const double sg = ksg[kt * PAE_BK + kk];
        cX[kk * LDX + e] = combine(x0, x1, f00, f10, trv, sg);
        cX[(PAE_BK + kk) * LDX + e] = combine(x0, x1, f01, f11, trv, sg);
      }
      __syncthreads();
    }
#pragma unroll
    for (int k8 = 0; k8 < PAE_BK; k8 += 8) {
      double are[4], aim[4], anim[4];
      const double sa = PRE ? 1.0 : ksg[kt * PAE_BK + k8 + tig], sb = PRE ? 1.0 : ksg[kt * PAE_BK + k8 + tig + 4];
      xval(cX, k8 + tig, er, tr0, sa, are[0], aim[0]);
      xval(cX, k8 + tig, er + 8, tr1, sa, are[1], aim[1]);
      xval(cX, k8 + tig + 4, er, tr0, sb, are[2], aim[2]);
      xval(cX, k8 + tig + 4, er + 8, tr1, sb, are[3], aim[3]);
#pragma unroll
      for (int x = 0; x < 4; x++) anim[x] = G3 ? are[x] + aim[x] : -aim[x];  // G3: the sum Xr + Xi
#pragma unroll
      for (int j = 0; j < TN; j++) {
        const int nb = (wc * TN + j) * 8 + gid;
        const cplx w0 = cB[(k8 + tig) * LDN + nb], w1 = cB[(k8 + tig + 4) * LDN + nb];
        const double bre[2] = {w0.x, w1.x}, bim[2] = {w0.y, w1.y};
        if (G3) {
          const double bsum[2] = {w0.x + w0.y, w1.x + w1.y};
          dmma_16x8x8(cre[j], are, bre);
          dmma_16x8x8(cim[j], aim, bim);
          dmma_16x8x8(c3[G3 ? j : 0], anim, bsum);
        } else {
          dmma_16x8x8(cre[j], are, bre);
          dmma_16x8x8(cre[j], anim, bim);
          dmma_16x8x8(cim[j], are, bim);
          dmma_16x8x8(cim[j], aim, bre);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  if (G3) {
#pragma unroll
    for (int j = 0; j < TN; j++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const double p1 = cre[j][x], p2 = cim[j][x];
        cre[j][x] = p1 - p2;
        cim[j][x] = c3[G3 ? j : 0][x] - p1 - p2;
      }
  }

  // epilogue: F_target += C / Nx on the listed elements (each element is in
  // a family's list once, so a pass writes it at most once)
  cplx* Ft = pair == 0 ? (tgt == 0 ? P.F[0] : P.F[1]) : (tgt == 0 ? P.F[2] : P.F[3]);
  const int rw0 = erow[er], rw1 = erow[er + 8];
#pragma unroll
  for (int j = 0; j < TN; j++)
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int rw = x >= 2 ? rw1 : rw0;
      const long long c = ecol[(wc * TN + j) * 8 + 2 * tig + (x & 1)];
      if (rw < 0 || c < 0) continue;
      // a reduction in L2 (no value returned, so no wait for the old F);
      // each element is in a family's list once, so no two CTAs of a launch
      // add to the same entry
      cplx* f = Ft + c + rw;
      atomicAdd(&f->x, __dmul_rn(inv_nx, cre[j][x]));
      atomicAdd(&f->y, __dmul_rn(inv_nx, cim[j][x]));
    }
}

template <int TN, int WN, int RW, int STG, int QN = 1, bool G3 = false, bool PRE = false>
static int run_pae(tups_ctx* ctx, const PaePtrs& P, int nchunks, int fam, int max_count) {
  const auto& d = ctx->d;
  constexpr int BN = 8 * TN * WN;
  constexpr int E = 8 * RW;
  constexpr int LDX = E + 2;
  const int K = d.Nl * d.Nl * d.NR;
  const int Kpad = (K + PAE_BK - 1) / PAE_BK * PAE_BK;
  const size_t sm = (size_t)(STG * 2 * PAE_BK * LDX + STG * PAE_BK * pae_ldn(BN)) * sizeof(cplx) +
                    (size_t)Kpad * (sizeof(long long) + sizeof(double) + sizeof(int)) + (size_t)BN * sizeof(int);
  auto kern = k_pae_mma<TN, WN, RW, STG, QN, G3, PRE>;
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_pae_mma smem attribute");
  }
  const int max_tiles = (max_count + E - 1) / E;
  if (max_tiles == 0) return TUPS_OK;
  const int nh = d.Nf / 2;
  const int nQ = (ctx->slot0 + d.Nb - 1) / nh - ctx->slot0 / nh + 1;  // momenta holding this context's slots
  const int gx = QN > 0 ? (nQ + QN - 1) / QN : (nQ * d.Nl * d.Nl + BN - 1) / BN;
  if (QN == 0) nchunks = 1;
  dim3 grid(gx, max_tiles * 2 * nchunks, nh);
  kern<<<grid, 32 * RW * WN, sm, ctx->stream>>>(P, ctx->t.pae_elems, ctx->t.pae_counts, ctx->t.ibz, ctx->t.signs,
                                                d.Nz, d.Nf, d.Nl, d.NIBZ, d.NR, nchunks, fam, Kpad, ctx->slot0,
                                                d.Nb, 1.0 / d.Nx);
  return after_launch(ctx, "k_pae_mma");
}

// Element lists of the two families per target pair and bosonic index W,
// built on the host from the frequency maps (pae_family) at the first call.
static int build_pae_lists(tups_ctx* ctx) {
  const auto& d = ctx->d;
  const int Nf = d.Nf, nh = Nf / 2;
  std::vector<int4> el((size_t)4 * nh * Nf * Nf, make_int4(0, 0, 1, 1));
  std::vector<int> cnt((size_t)4 * nh, 0);
  for (int pair = 0; pair < 2; pair++)
    for (int fam = 0; fam < 2; fam++)
      for (int W = 1; W <= nh; W++) {
        const int L = pae_list(pair, fam, W, nh);
        int c = 0;
        for (int nu2 = 1; nu2 <= Nf; nu2++)
          for (int nu1 = 1; nu1 <= Nf; nu1++) {
            int w2, a, b, tr;
            if (!pae_family(pair, fam, nu1, nu2, W, Nf, &w2, &a, &b, &tr)) continue;
            el[(size_t)L * Nf * Nf + c++] = make_int4(nu1 + 256 * nu2, w2, a, b + 65536 * tr);
          }
        cnt[L] = c;
        ctx->pae_max_tiles[fam] = std::max(ctx->pae_max_tiles[fam], c);  // longest list
      }
  void* pe = nullptr;
  void* pc = nullptr;
  int rc = cuda_check(ctx, cudaMalloc(&pe, el.size() * sizeof(int4)), "PAE element lists");
  if (rc) return rc;
  ctx->allocations.push_back(pe);
  rc = cuda_check(ctx, cudaMalloc(&pc, cnt.size() * sizeof(int)), "PAE element counts");
  if (rc) return rc;
  ctx->allocations.push_back(pc);
  ctx->t.pae_elems = (int4*)pe;
  ctx->t.pae_counts = (int*)pc;
  rc = cuda_check(ctx, cudaMemcpyAsync(pe, el.data(), el.size() * sizeof(int4), cudaMemcpyHostToDevice, ctx->stream),
                  "PAE lists H2D");
  if (rc) return rc;
  rc = cuda_check(ctx, cudaMemcpyAsync(pc, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream),
                  "PAE counts H2D");
  if (rc) return rc;
  return cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "PAE lists");
}

// Tile candidates of the crossing kernel per form-factor count.  They differ
// in how the (target, element) rows and the (momentum, (l1, l2)) columns are
// spread over CTAs and warps; every output element is still summed over K in
// the same order, so all candidates write the same bits.  Index 0 is the
// default when the tuner is off: the tuner's pick on a B200, flat 64-column
// tiles, at 8x8 / Nl = 5 (1.677 ms against 1.760 ms for three momenta side
// by side in 80 columns, 1.754 flat 80, 1.734 flat 48) and at 16x16 / Nl = 9
// (403 ms against 481 ms for one momentum per 96-column CTA, 406 flat 80,
// 411 flat 96, 428 flat 112; two CTAs per SM throughout).
struct PaeCand {
  const char* name;
  int (*run)(tups_ctx*, const PaePtrs&, int, int, int);
  int bn;  // columns per CTA; chunks of BN per momentum when QN = 1
};
static const PaeCand kPaeNl1[] = {
    {"flat_bn8_tn1", run_pae<1, 1, 4, 2, 0>, 8},
    {"flat_bn16_tn2", run_pae<2, 1, 4, 2, 0>, 16},
    {"q1_bn8_tn1", run_pae<1, 1, 4, 2, 1>, 8},
};
static const PaeCand kPaeNl5[] = {
    {"flat_bn64_tn4", run_pae<4, 2, 4, 2, 0>, 64},
    {"q3_bn80_tn5", run_pae<5, 2, 4, 2, 3>, 80},
    {"flat_bn80_tn5", run_pae<5, 2, 4, 2, 0>, 80},
    {"flat_bn48_tn3", run_pae<3, 2, 4, 2, 0>, 48},
};
static const PaeCand kPaeWide[] = {
    {"flat_bn64_tn4", run_pae<4, 2, 4, 2, 0>, 64},
    {"q1_bn96_tn6", run_pae<6, 2, 4, 2, 1>, 96},
    {"flat_bn80_tn5", run_pae<5, 2, 4, 2, 0>, 80},
    {"flat_bn96_tn6", run_pae<6, 2, 4, 2, 0>, 96},
    {"flat_bn112_tn7", run_pae<7, 2, 4, 2, 0>, 112},
};
// three real products per complex one (Gauss): a different rounding of each
// sum, so these form their own candidate set, chosen by the context's
// crossing-products setting.  "g3p" candidates rewrite each landed X stage
// as per-target operands (PRE); "_s3" ones run a three-stage pipeline.
// Index 0 is the tuner's pick on a B200: at 8x8 / Nl = 5 64 flat columns
// (1.24 ms against 1.25 for the PRE form on 64 and 1.31-1.37 for the rest),
// at 16x16 / Nl = 9 the PRE form on 64 columns (316 ms against 318 on 48
// and 338 without PRE).
static const PaeCand kPaeNl5G3[] = {
    {"g3_flat_bn64_tn4", run_pae<4, 2, 4, 2, 0, true>, 64},
    {"g3p_flat_bn32_tn2", run_pae<2, 2, 4, 2, 0, true, true>, 32},
    {"g3_flat_bn48_tn3_s3", run_pae<3, 2, 4, 3, 0, true>, 48},
    {"g3_flat_bn32_tn2", run_pae<2, 2, 4, 2, 0, true>, 32},
    {"g3_flat_bn48_tn3", run_pae<3, 2, 4, 2, 0, true>, 48},
    {"g3p_flat_bn64_tn4", run_pae<4, 2, 4, 2, 0, true, true>, 64},
};
static const PaeCand kPaeWideG3[] = {
    {"g3p_flat_bn64_tn4", run_pae<4, 2, 4, 2, 0, true, true>, 64},
    {"g3p_flat_bn48_tn3", run_pae<3, 2, 4, 2, 0, true, true>, 48},
    {"g3_flat_bn64_tn4", run_pae<4, 2, 4, 2, 0, true>, 64},
    {"g3_flat_bn48_tn3", run_pae<3, 2, 4, 2, 0, true>, 48},
    {"g3_flat_bn48_tn3_s3", run_pae<3, 2, 4, 3, 0, true>, 48},
};

static int pae_all(tups_ctx* ctx, const PaePtrs& P, const PaeCand& c) {
  const auto& d = ctx->d;
  const size_t n = (size_t)d.Nz * d.Nz * d.Nb;
  dim3 bgrid((unsigned)std::min<size_t>(cdiv(n, 256), 148 * 8), 4);
  k_pae_base<<<bgrid, 256, 0, ctx->stream>>>(P, ibz_local(ctx), d.Nz, d.Nf, d.Nb,
                                             std::fabs(1.0 / ctx->FF[0] * 1.0 / ctx->FF[0]));
  int rc = after_launch(ctx, "k_pae_base");
  const int nchunks = (d.Nl * d.Nl + c.bn - 1) / c.bn;
  for (int fam = 0; fam < 2 && !rc; fam++) rc = c.run(ctx, P, nchunks, fam, ctx->pae_max_tiles[fam]);
  return rc;
}

int launch_pae(tups_ctx* ctx) {
  const auto& d = ctx->d;
  if (d.Nl > 13) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 13 not supported by the crossing kernel");
  if (d.Nf > 255) return set_error(ctx, TUPS_ERR_BADDIM, "Nf > 255 not supported by the crossing kernel");
  if ((long long)d.Nl * d.Nl * d.Nl * d.Nl * d.NIBZ * d.NR >= (1LL << 31))
    return set_error(ctx, TUPS_ERR_BADDIM, "crossing tensor too large for 32-bit offsets");
  if (!ctx->t.pae_elems) {
    int rc = build_pae_lists(ctx);
    if (rc) return rc;
  }
  PaePtrs P;
  for (int r = 0; r < 4; r++) {
    P.Phi[r] = ctx->s.G[r];
    P.PhiR[r] = ctx->s.PhiR[r];
    P.M[r] = ctx->s.M[r];
    P.L[r] = ctx->t.L[r];
    P.F[r] = ctx->s.F[r];
  }
  // F = Phi + Lambda Nc, then the diagonal family, then the anti-diagonal one
  const int nl2 = d.Nl * d.Nl;
  const bool g3 = ctx->pae_products == 3 && nl2 > 8;
  const PaeCand* cands = nl2 <= 8 ? kPaeNl1 : nl2 <= 32 ? (g3 ? kPaeNl5G3 : kPaeNl5) : (g3 ? kPaeWideG3 : kPaeWide);
  const int n_cand = nl2 <= 8 ? (int)(sizeof(kPaeNl1) / sizeof(PaeCand))
                     : nl2 <= 32 ? (g3 ? (int)(sizeof(kPaeNl5G3) / sizeof(PaeCand))
                                       : (int)(sizeof(kPaeNl5) / sizeof(PaeCand)))
                                 : (g3 ? (int)(sizeof(kPaeWideG3) / sizeof(PaeCand))
                                       : (int)(sizeof(kPaeWide) / sizeof(PaeCand)));
  const std::string key = std::string(g3 ? "k_pae_mma(3M)" : "k_pae_mma") + " Nl=" + std::to_string(d.Nl) +
                          " Nf=" + std::to_string(d.Nf) +
                          " NIBZ=" + std::to_string(d.NIBZ) + " NR=" + std::to_string(d.NR) +
                          " Nb=" + std::to_string(d.Nb) + " slot0=" + std::to_string(ctx->slot0);
  int choice = 0;
  std::vector<std::string> names;
  for (int c = 0; c < n_cand; c++) names.push_back(cands[c].name);
  const int forced = tune_forced(key, names);
  if (forced >= 0) {
    choice = forced;
  } else if (ctx->autotune && !tune_get(key, &choice) && tune_allowed(ctx)) {
    // every run rebuilds F from Phi, so timing the candidates in place is
    // harmless; the chosen one runs last
    int rc = tune_pick(ctx, key, n_cand, names, [&](int c) { return pae_all(ctx, P, cands[c]); }, 2, &choice);
    if (rc) return rc;
  }
  return pae_all(ctx, P, cands[choice]);
}

}  // namespace tups

// Real DMMA products per complex one in the crossing GEMM: 3 (default;
// Gauss: Xr Mr, Xi Mi, (Xr + Xi)(Mr + Mi)) or 4.  Both agree with the reference
// to rounding; the three-product form rounds differently.
extern "C" int tups_set_crossing_products(tups_ctx* ctx, int products) {
  if (!ctx || (products != 3 && products != 4)) return TUPS_ERR_BADARG;
  if (products != ctx->pae_products) {
    // iterations captured as CUDA graphs hold the other form's kernels
    for (auto& g : ctx->graph_exec)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }
  ctx->pae_products = products;
  return TUPS_OK;
}
