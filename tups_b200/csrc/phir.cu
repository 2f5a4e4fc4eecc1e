// Phi(q) -> Phi(R) transform and crossing tensors.
//   calc_PhiR / FTPhis / symop_arr (SRC/parquet_PhiR.f90:35-356)
//   calculate_expSqR / calculate_expqSR (SRC/parquet_PhiR.f90:360-435)
//   calc_M_* (SRC/parquet_EQMatrix.f90:21-360), evaluated per IBZ momentum
#include <cmath>
#include <string>
#include <vector>

#include "tups_device.cuh"

namespace tups {

struct PhirPtrs {
  const cplx* G[4];
  cplx* PhiR[4];
};

// PhiR_r[(i,j), w, R] = (1/Nx) sum_Q sum_{sym in star(Q)} fac_sym(l_i) fac_sym(l_j)
//     Phi_r[(lsym(l_i), nu_i), (lsym(l_j), nu_j), (Q, w)] expSqR(Q, R, sym)
// (the reference's symop_arr + FTPhis ZGEMM, parquet_PhiR.f90:196-356; the
// symmetries outside the star of Q carry expSqR = 0 and are skipped).
//
// The symmetry operations permute the form-factor index only, never nu, so
// every output of the pair (nu_i, nu_j) reads the same Nl x Nl inputs
// Phi[(a, nu_i), (b, nu_j), Q].  A CTA owns one nu_j, a tile of PH_TI
// consecutive nu_i and one (w, r).  For each momentum Q of the context it
// stages Phi[(a, nu_i), (b, nu_j), (Q, w)] for all a, b and the tile's nu_i
// (Nl^2 runs of PH_TI contiguous complex) in shared memory with cp.async
// (three buffers, copies two momenta ahead, one barrier per momentum), and
// every symmetric image of Q reads its permuted entries
// (lsym(l_i), lsym(l_j)) from there: each Phi(Q) element leaves HBM once and
// the inner loop is FP64 FMAs on shared-memory operands.  Per output the sum
// runs over Q ascending and, within Q, over the star's symmetries ascending.
//
// Thread (pair p = l_i + Nl l_j, lane c < SUB = PH_TI / OPT) owns the OPT
// outputs nu_i = nu_i0 + c + SUB k, all NR lattice vectors; the phases
// expSqR(Q, R, sym) of the star pairs sit in shared memory, packed by pair.
constexpr int PH_TI = 16;
constexpr int PH_STAGES = 3;  // Phi(Q) stages in shared memory (momenta in flight)

__device__ __forceinline__ void ph_cp_async16(void* sdst, const void* gsrc, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  const unsigned sz = valid ? 16u : 0u;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz));
}

// flips the sign of x when bit is set (an integer operation: the FP64 pipe
// stays with the FMAs)
__device__ __forceinline__ double ph_sign(double x, unsigned bit) {
  return __longlong_as_double(__double_as_longlong(x) ^ ((long long)bit << 63));
}

// threads per CTA the register budget allows (acc is 4 OPT NR registers)
__host__ __device__ constexpr int phir_max_threads(int opt, int nr) {
  return nr == 1 ? 1024 : opt == 4 ? 384 : opt == 2 ? 672 : 768;
}

// stage Phi[(a, ni0 + t), (b, nj)] (t < PH_TI, all a, b < Nl) of one slot
// into dst[(a + Nl b) PH_TI + t]; src points at element (0, nj) of the
// slot; entries with ni >= Nf are zero-filled
// (the same entries for every slot: the source offsets are computed once
// per thread, ph_offsets, and reused for every momentum; -1 = zero fill,
// -2 = no entry; a thread owns at most NC entries, NC blockDim >= n)
template <int NC>
__device__ __forceinline__ void ph_offsets(int* off, int n, int Nl, int Nf, int Nz, int ni0) {
#pragma unroll
  for (int u = 0; u < NC; u++) {
    const int x = threadIdx.x + u * blockDim.x;
    off[u] = -2;
    if (x < n) {
      const int t = x % PH_TI, ab = x / PH_TI;
      const int a = ab % Nl, b = ab / Nl, ni = ni0 + t;
      off[u] = ni < Nf ? (a * Nf + ni) + Nz * Nf * b : -1;
    }
  }
}
template <int NC>
__device__ __forceinline__ void ph_stage(cplx* dst, const cplx* src, const int* off) {
#pragma unroll
  for (int u = 0; u < NC; u++) {
    if (off[u] == -2) continue;
    const bool ok = off[u] >= 0;
    ph_cp_async16(dst + threadIdx.x + u * blockDim.x, ok ? src + off[u] : src, ok);
  }
}

template <int OPT, int NR>
__global__ void __launch_bounds__(phir_max_threads(OPT, NR)) k_phir(PhirPtrs P, const cplx* __restrict__ expSqR,
                                               const int* __restrict__ symlist, const int* __restrict__ lsym,
                                               const double* __restrict__ lfac, int Nz, int Nf, int Nl, int NIBZ,
                                               int npairs, int slot0, int Nb, double inv_nx) {
  constexpr int SUB = PH_TI / OPT;
  extern __shared__ __align__(16) unsigned char phir_sm[];
  const int nl2 = Nl * Nl;
  cplx* sPhi = reinterpret_cast<cplx*>(phir_sm);          // [PH_STAGES][nl2][PH_TI]
  cplx* sE = sPhi + (size_t)PH_STAGES * nl2 * PH_TI;       // [npairs][NR]
  int* sSym = reinterpret_cast<int*>(sE + (size_t)npairs * NR);  // [npairs] symmetry of pair p
  int* sBeg = sSym + npairs;                               // [NIBZ + 1] first pair of Q
  int* sQ = sBeg + NIBZ + 1;                               // [NIBZ] momenta of this context at w
  // [NS][blockDim]: this thread's permuted offset per symmetry, sign in bit 31
  unsigned* sOff = reinterpret_cast<unsigned*>(sQ + NIBZ);
  __shared__ int sNq;

  const int ntile = (Nf + PH_TI - 1) / PH_TI;
  const int nj = blockIdx.x / ntile, ni0 = (blockIdx.x % ntile) * PH_TI;
  const int w = blockIdx.y, r = blockIdx.z;
  const int nh = Nf / 2;
  const int lane = threadIdx.x & 31;

  // star pairs with Q ascending (prefix sums of the star sizes) and the
  // momenta whose slot (Q, w) this context holds; first warp
  if (threadIdx.x < 32) {
    int base = 0, nq = 0;
    for (int Q0 = 0; Q0 < NIBZ; Q0 += 32) {
      const int Q = Q0 + lane;
      unsigned m = 0;
      bool mine = false;
      if (Q < NIBZ) {
#pragma unroll
        for (int sy = 0; sy < NS; sy++)
          if (symlist[NS * Q + sy]) m |= 1u << sy;
        const int lq = Q * nh + w - slot0;
        mine = lq >= 0 && lq < Nb;
      }
      const int c = __popc(m);
      int x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      if (Q < NIBZ) {
        sBeg[Q] = base + x - c;
        int p = base + x - c;
        for (int sy = 0; sy < NS; sy++)
          if (m >> sy & 1u) sSym[p++] = sy | (Q << 3);
      }
      const unsigned bal = __ballot_sync(0xffffffffu, mine);
      if (mine) sQ[nq + __popc(bal & ((1u << lane) - 1u))] = Q;
      nq += __popc(bal);
      base += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) {
      sBeg[NIBZ] = base;
      sNq = nq;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < npairs * NR; t += blockDim.x) {
    const int p = t / NR, R = t % NR;
    const int sy = sSym[p] & 7, Q = sSym[p] >> 3;
    sE[t] = expSqR[Q + (size_t)NIBZ * (R + (size_t)NR * sy)];
  }
  const int nq = sNq;

  // this thread's outputs: pair p, permuted-pair offsets and signs per symmetry
  const int p = threadIdx.x / SUB, c = threadIdx.x % SUB;
  const bool active = p < nl2;
  // (each thread reads back only its own entries: no barrier)
  if (active) {
    const int li = p % Nl, lj = p / Nl;
#pragma unroll
    for (int sy = 0; sy < NS; sy++) {
      const unsigned o = (unsigned)((lsym[sy + NS * li] + Nl * lsym[sy + NS * lj]) * PH_TI + c);
      const unsigned neg = lfac[sy + NS * li] * lfac[sy + NS * lj] < 0.0 ? 1u : 0u;
      sOff[sy * blockDim.x + threadIdx.x] = o | (neg << 31);
    }
  }
  cplx acc[OPT][NR];
#pragma unroll
  for (int k = 0; k < OPT; k++)
#pragma unroll
    for (int R = 0; R < NR; R++) acc[k][R] = cmk(0.0, 0.0);

  const size_t n2 = (size_t)Nz * Nz;
  // constant indices keep the parameter struct out of local memory
  const cplx* G = r == 0 ? P.G[0] : r == 1 ? P.G[1] : r == 2 ? P.G[2] : P.G[3];
  const int stage_elems = nl2 * PH_TI;
  const cplx* Gw = G + (size_t)Nz * nj;  // element (0, (0, nj)); column (b, nj) is Nz Nf b further
  // stage_elems = Nl^2 PH_TI <= OPT blockDim: at most OPT copies per thread
  int soff[OPT];
  ph_offsets<OPT>(soff, stage_elems, Nl, Nf, Nz, ni0);
  // three buffers, momenta staged two ahead: the barrier at the top of an
  // iteration both publishes this momentum's stage and ends every read of
  // the buffer the next copy overwrites, so one barrier per momentum
#pragma unroll
  for (int qq = 0; qq < PH_STAGES - 1; qq++) {
    if (qq < nq) ph_stage<OPT>(sPhi + (size_t)qq * stage_elems, Gw + n2 * (size_t)(sQ[qq] * nh + w - slot0), soff);
    asm volatile("cp.async.commit_group;\n" ::);
  }
  for (int qi = 0; qi < nq; qi++) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PH_STAGES - 2));
    __syncthreads();
    {
      const int qn = qi + PH_STAGES - 1;
      if (qn < nq)
        ph_stage<OPT>(sPhi + (size_t)(qn % PH_STAGES) * stage_elems, Gw + n2 * (size_t)(sQ[qn] * nh + w - slot0),
                      soff);
      asm volatile("cp.async.commit_group;\n" ::);
    }
    const cplx* S = sPhi + (size_t)(qi % PH_STAGES) * stage_elems;
    const int Q = sQ[qi];
    const int pe = sBeg[Q + 1];
    for (int pp = sBeg[Q]; pp < pe; pp++) {
      const int sy = sSym[pp] & 7;
      cplx e[NR];
#pragma unroll
      for (int R = 0; R < NR; R++) e[R] = sE[pp * NR + R];
      if (active) {
        const unsigned word = sOff[sy * blockDim.x + threadIdx.x];
        const unsigned off = word & 0x7fffffffu;
        const unsigned neg = word >> 31;
#pragma unroll
        for (int k = 0; k < OPT; k++) {
          cplx v = S[off + SUB * k];
          v.x = ph_sign(v.x, neg);
          v.y = ph_sign(v.y, neg);
#pragma unroll
          for (int R = 0; R < NR; R++) acc[k][R] = cfma(v, e[R], acc[k][R]);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::);
  if (!active) return;
  const int li = p % Nl, lj = p / Nl;
  cplx* out = r == 0 ? P.PhiR[0] : r == 1 ? P.PhiR[1] : r == 2 ? P.PhiR[2] : P.PhiR[3];
#pragma unroll
  for (int k = 0; k < OPT; k++) {
    const int ni = ni0 + c + SUB * k;
    if (ni >= Nf) continue;
    const size_t e = (size_t)(li * Nf + ni) + (size_t)Nz * (lj * Nf + nj);
#pragma unroll
    for (int R = 0; R < NR; R++) out[e + n2 * ((size_t)w + (size_t)nh * R)] = cscale(acc[k][R], inv_nx);
  }
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

// k_phir instantiations by outputs per thread (OPT) and NR; every candidate
// forms each output's sum in the same order, so all write the same bits.
typedef void (*PhirFn)(PhirPtrs, const cplx*, const int*, const int*, const double*, int, int, int, int, int, int,
                       int, double);
struct PhirCand {
  const char* name;
  int opt;
  PhirFn fn1, fn4, fn6;
};
static const PhirCand kPhirCands[] = {
    {"opt2", 2, k_phir<2, 1>, k_phir<2, 4>, k_phir<2, 6>},
    {"opt4", 4, k_phir<4, 1>, k_phir<4, 4>, k_phir<4, 6>},
    {"opt1", 1, k_phir<1, 1>, k_phir<1, 4>, k_phir<1, 6>},
};
constexpr int kNumPhirCands = sizeof(kPhirCands) / sizeof(kPhirCands[0]);

static int phir_threads(const tups_ctx* ctx, int cand) {
  const int opt = kPhirCands[cand].opt;
  return (ctx->d.Nl * ctx->d.Nl * (PH_TI / opt) + 31) / 32 * 32;
}

static bool phir_fits(const tups_ctx* ctx, int cand) {
  return phir_threads(ctx, cand) <= phir_max_threads(kPhirCands[cand].opt, ctx->d.NR);
}

static int phir_run(tups_ctx* ctx, const PhirPtrs& P, int cand) {
  const auto& d = ctx->d;
  const PhirCand& C = kPhirCands[cand];
  PhirFn fn = d.NR == 1 ? C.fn1 : d.NR == 4 ? C.fn4 : C.fn6;
  int npairs = 0;
  for (int v : ctx->symlist) npairs += v ? 1 : 0;
  const int nl2 = d.Nl * d.Nl;
  const int threads = phir_threads(ctx, cand);
  if (!phir_fits(ctx, cand)) return set_error(ctx, TUPS_ERR_BADDIM, "k_phir: too many form-factor pairs for one CTA");
  const size_t sm = (size_t)PH_STAGES * nl2 * PH_TI * sizeof(cplx) + (size_t)npairs * d.NR * sizeof(cplx) +
                    ((size_t)npairs + 2 * d.NIBZ + 1) * sizeof(int) + (size_t)NS * threads * sizeof(unsigned);
  if (sm > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return cuda_check(ctx, e, "k_phir smem attribute");
  }
  const int ntile = (d.Nf + PH_TI - 1) / PH_TI;
  dim3 grid(ntile * d.Nf, d.Nf / 2, 4);
  fn<<<grid, threads, sm, ctx->stream>>>(P, ctx->t.expSqR, ctx->t.symlist, ctx->t.lsym, ctx->t.lfac, d.Nz, d.Nf,
                                         d.Nl, d.NIBZ, npairs, ctx->slot0, d.Nb, 1.0 / d.Nx);
  return after_launch(ctx, "k_phir");
}

int launch_phir(tups_ctx* ctx) {
  const auto& d = ctx->d;
  PhirPtrs P;
  for (int r = 0; r < 4; r++) {
    P.G[r] = ctx->s.G[r];
    P.PhiR[r] = ctx->s.PhiR[r];
  }
  if (d.NR != 1 && d.NR != 4 && d.NR != 6) return set_error(ctx, TUPS_ERR_BADDIM, "k_phir: NR not in {1, 4, 6}");
  if (d.Nl > 16) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 16 not supported by k_phir");
  // the tuner: Phi(R) is a pure function of Gamma and the tables, so the
  // candidates run on the call's own operands
  const std::string key = "k_phir Nl=" + std::to_string(d.Nl) + " Nf=" + std::to_string(d.Nf) +
                          " NIBZ=" + std::to_string(d.NIBZ) + " Nb=" + std::to_string(d.Nb) +
                          " slot0=" + std::to_string(ctx->slot0);
  // the candidates whose CTA fits this Nl; the first one is the default
  std::vector<int> fit;
  std::vector<std::string> names;
  for (int c = 0; c < kNumPhirCands; c++)
    if (phir_fits(ctx, c)) {
      fit.push_back(c);
      names.push_back(kPhirCands[c].name);
    }
  if (fit.empty()) return set_error(ctx, TUPS_ERR_BADDIM, "k_phir: too many form-factor pairs for one CTA");
  int choice = 0;
  int rc = TUPS_OK;
  const int forced = tune_forced(key, names);
  if (forced >= 0) {
    choice = forced;
  } else if (ctx->autotune && !tune_get(key, &choice) && tune_allowed(ctx)) {
    rc = tune_pick(ctx, key, (int)fit.size(), names, [&](int c) { return phir_run(ctx, P, fit[c]); }, 2, &choice);
    if (rc) return rc;
  }
  if (choice < 0 || choice >= (int)fit.size()) choice = 0;
  rc = phir_run(ctx, P, fit[choice]);
  if (rc) return rc;
  // a sharded context summed over its own momenta: Phi(R) over all ranks
  const size_t n2 = (size_t)d.Nz * d.Nz;
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
