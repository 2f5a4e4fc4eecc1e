// Parquet equation: calculate_PAE (SRC/parquet_EQOuter.f90:16-118) with the
// eight crossing contributions of SRC/parquet_EQContribs.f90:44-524.
//
// The reference loops over source channel and w2 and scatter-adds every
// contribution into F.  Here the loop is turned around (output-stationary):
// for a target element F_a/F_b[(l1,nu1),(l2,nu2), q] each contribution type
// hits it for at most ONE w2, obtained by inverting the type's frequency map,
//   phbar_to_ph     w2 = nu2 - nu1 + 1          (F_d, F_m  <- Phi_d, Phi_m)
//   phbar_to_ph_TR  w2 = nu1 - nu2 + 1 (>1)
//   pp_to_ph        w2 = nu1 + nu2 + W - Nf - 1 (F_d, F_m  <- Phi_s, Phi_t)
//   pp_to_ph_TR     w2 = Nf + 3 - nu1 - nu2 - W (>1)
//   ph_to_pp        w2 = W - nu1 - nu2 + Nf + 1 (F_s, F_t  <- Phi_d, Phi_m)
//   ph_to_pp_TR     w2 = nu1 + nu2 - W - Nf + 1 (>1)
//   phbar_to_pp     w2 = nu2 - nu1 + 1          (F_s, F_t  <- Phi_d, Phi_m)
//   phbar_to_pp_TR  w2 = nu1 - nu2 + 1 (>1)
// (W = bosonic index of q, 1-based frequencies, w2 in 1..Nf/2).  So every F
// element is formed once, in registers, as Phi + Lambda*Nc + sum of <= 4
// contractions over (R, l3, l4), and written once: no atomics, deterministic.
// The two sources of a type are combined with the dispatch factors of
// SRC/parquet_EQOuter.f90:84-113 before the contraction.
#include "tups_device.cuh"

namespace tups {

constexpr int PAE_NLMAX = 13;

struct PaePtrs {
  const cplx* Phi[4];   // Phi_r (G arrays after the BSE), (Nz, Nz, Nb)
  const cplx* PhiR[4];  // (Nz*Nz, Nf/2, NR)
  const cplx* M[4];     // (Nl^4, NIBZ, NR)
  const cplx* L[4];     // (Nf, Nf, Nf/2)
  cplx* F[4];
};

__device__ __forceinline__ int clampnu(int x, int Nf) { return x < 1 ? 1 : (x > Nf ? Nf : x); }

// Frequency map of contribution type t of target pair `pair` for the target
// (nu1, nu2) at bosonic index W.  Returns false when the type does not reach
// this element; otherwise w2 and the source (row, column) frequencies a, b.
__device__ __forceinline__ bool pae_map(int pair, int t, int nu1, int nu2, int W, int Nf, int* w2, int* a, int* b) {
  const int nh = Nf / 2;
  int ww;
  if (pair == 0) {
    switch (t) {
      case 0:  // phbar_to_ph: nu2 = nu1 + w2 - 1, Phi_R[(l3,nu1),(l4,pick(nu1+W-1))]
        ww = nu2 - nu1 + 1;
        if (ww < 1 || ww > nh) return false;
        *a = nu1;
        *b = clampnu(nu1 + W - 1, Nf);
        break;
      case 1:  // phbar_to_ph_TR: nu2 = nu1 - w2 + 1, conj Phi_R[(l3,mF(nu1)),(l4,pick(mF(nu1+W-1)))]
        ww = nu1 - nu2 + 1;
        if (ww < 2 || ww > nh) return false;
        *a = Nf + 1 - nu1;
        *b = clampnu(Nf + 2 - nu1 - W, Nf);
        break;
      case 2:  // pp_to_ph: nu2 = BmBmF(w2, W, nu1), Phi_R[(l3,nu1),(l4,nu2)]
        ww = nu1 + nu2 + W - Nf - 1;
        if (ww < 1 || ww > nh) return false;
        *a = nu1;
        *b = nu2;
        break;
      default:  // pp_to_ph_TR: nu2 = mF(nu1+W+w2-2), conj Phi_R[(l3,mF(nu1)),(l4,mF(nu2))]
        ww = Nf + 3 - nu1 - nu2 - W;
        if (ww < 2 || ww > nh) return false;
        *a = Nf + 1 - nu1;
        *b = Nf + 1 - nu2;
        break;
    }
  } else {
    switch (t) {
      case 0:  // ph_to_pp: nu2 = BmBmF(W, w2, nu1), Phi_R[(l3,nu1),(l4,nu2)]
        ww = W - nu1 - nu2 + Nf + 1;
        if (ww < 1 || ww > nh) return false;
        *a = nu1;
        *b = nu2;
        break;
      case 1:  // ph_to_pp_TR: nu2 = BpBmF(W, w2, nu1), conj Phi_R[(l3,mF(nu1)),(l4,FmB(nu1,W+w2-1))]
        ww = nu1 + nu2 - W - Nf + 1;
        if (ww < 2 || ww > nh) return false;
        *a = Nf + 1 - nu1;
        *b = nu1 - (W + ww - 1) + 1;
        break;
      case 2:  // phbar_to_pp: nu2 = nu1 + w2 - 1, Phi_R[(l3,nu1),(l4,pick(BmBmF(W,w2,nu1)))]
        ww = nu2 - nu1 + 1;
        if (ww < 1 || ww > nh) return false;
        *a = nu1;
        *b = clampnu((W - 1) - (nu1 + ww - 1) + Nf + 1, Nf);
        break;
      default:  // phbar_to_pp_TR: nu2 = nu1 - w2 + 1, conj Phi_R[(l3,mF(nu1)),(l4,pick(FmB(nu1,W+w2-1)))]
        ww = nu1 - nu2 + 1;
        if (ww < 2 || ww > nh) return false;
        *a = Nf + 1 - nu1;
        *b = clampnu(nu1 - (W + ww - 1) + 1, Nf);
        break;
    }
  }
  *w2 = ww;
  return true;
}

// One CTA per (q slot, target pair, l1); threads over the (nu1, nu2) plane;
// each thread keeps F_a, F_b for all l2 of its element in registers.
__global__ void __launch_bounds__(256) k_pae(PaePtrs P, const int* __restrict__ ibz, const int* __restrict__ signs,
                                             int Nz, int Nf, int Nl, int NIBZ, int NR, double aux, double inv_nx) {
  const int q = blockIdx.x;
  const int pair = blockIdx.y;
  const int l1 = blockIdx.z;
  const int W = ibz[3 * q + 2];
  const int Qi = q / (Nf / 2);
  const int nh = Nf / 2;
  const size_t n2 = (size_t)Nz * Nz;
  const int nl2 = Nl * Nl, nl4 = nl2 * nl2;
  // targets and sources: pair 0 -> (F_d, F_m), sources (d,m) for types 0,1 and
  // (s,t) for types 2,3; pair 1 -> (F_s, F_t), sources (d,m) for all types
  const int ta = pair == 0 ? 0 : 2, tb = ta + 1;
  // dispatch factors (SRC/parquet_EQOuter.f90:84-113): [type][source][target]
  double fac[4][2][2];
  if (pair == 0) {
    const double f01[2][2] = {{-0.5, -0.5}, {-1.5, 0.5}};  // phbar_to_ph from d, m
    const double f23[2][2] = {{0.5, -0.5}, {1.5, 0.5}};    // pp_to_ph from s, t
    for (int s = 0; s < 2; s++)
      for (int g = 0; g < 2; g++) {
        fac[0][s][g] = fac[1][s][g] = f01[s][g];
        fac[2][s][g] = fac[3][s][g] = f23[s][g];
      }
  } else {
    const double f01[2][2] = {{0.5, 0.5}, {-1.5, 0.5}};    // ph_to_pp from d, m
    const double f23[2][2] = {{0.5, -0.5}, {-1.5, -0.5}};  // phbar_to_pp from d, m
    for (int s = 0; s < 2; s++)
      for (int g = 0; g < 2; g++) {
        fac[0][s][g] = fac[1][s][g] = f01[s][g];
        fac[2][s][g] = fac[3][s][g] = f23[s][g];
      }
  }
  // M type of each contribution
  const int mtype[4] = {pair == 0 ? 0 : 2, pair == 0 ? 0 : 2, pair == 0 ? 1 : 3, pair == 0 ? 1 : 3};

  for (int e = threadIdx.x; e < Nf * Nf; e += blockDim.x) {
    const int nu1 = e % Nf + 1, nu2 = e / Nf + 1;
    cplx acc_a[PAE_NLMAX], acc_b[PAE_NLMAX];
#pragma unroll
    for (int l2 = 0; l2 < PAE_NLMAX; l2++) acc_a[l2] = acc_b[l2] = cmk(0.0, 0.0);
    for (int t = 0; t < 4; t++) {
      int w2, a, b;
      if (!pae_map(pair, t, nu1, nu2, W, Nf, &w2, &a, &b)) continue;
      const bool tr = t & 1;
      const int s0 = (pair == 0 && t >= 2) ? 2 : 0;  // first source channel
      const cplx* X0 = P.PhiR[s0] + n2 * (w2 - 1);
      const cplx* X1 = P.PhiR[s0 + 1] + n2 * (w2 - 1);
      const cplx* Mt = P.M[mtype[t]] + (size_t)nl4 * Qi;
      const double fa0 = fac[t][0][0], fa1 = fac[t][1][0], fb0 = fac[t][0][1], fb1 = fac[t][1][1];
      for (int R = 0; R < NR; R++) {
        const size_t roff = n2 * nh * R;
        const cplx* MR = Mt + (size_t)nl4 * NIBZ * R;
        for (int l4 = 0; l4 < Nl; l4++)
          for (int l3 = 0; l3 < Nl; l3++) {
            const size_t xi = (size_t)(l3 * Nf + a - 1) + (size_t)Nz * (l4 * Nf + b - 1) + roff;
            cplx x0 = X0[xi], x1 = X1[xi];
            if (tr) {
              const double sg = (double)(signs[l3] * signs[l4]);
              x0 = cscale(cconj(x0), sg);
              x1 = cscale(cconj(x1), sg);
            }
            const cplx xa = cmk(fa0 * x0.x + fa1 * x1.x, fa0 * x0.y + fa1 * x1.y);
            const cplx xb = cmk(fb0 * x0.x + fb1 * x1.x, fb0 * x0.y + fb1 * x1.y);
            const cplx* Mrow = MR + l1 + (size_t)nl2 * (l3 + Nl * l4);
#pragma unroll
            for (int l2 = 0; l2 < PAE_NLMAX; l2++) {
              if (l2 < Nl) {
                const cplx m = __ldg(Mrow + Nl * l2);
                acc_a[l2] = cfma(m, xa, acc_a[l2]);
                acc_b[l2] = cfma(m, xb, acc_b[l2]);
              }
            }
          }
      }
    }
    // F = Phi + Lambda*Nc on the l=1 block + contributions/Nx
    const size_t i = (size_t)(l1 * Nf + nu1 - 1);
#pragma unroll
    for (int l2 = 0; l2 < PAE_NLMAX; l2++) {
      if (l2 < Nl) {
        const size_t idx = i + (size_t)Nz * (l2 * Nf + nu2 - 1) + n2 * q;
        cplx fa = P.Phi[ta][idx], fb = P.Phi[tb][idx];
        if (l1 == 0 && l2 == 0) {
          const size_t li = (size_t)(nu1 - 1) + (size_t)Nf * ((nu2 - 1) + (size_t)Nf * (W - 1));
          fa = cadd(fa, cscale(P.L[ta][li], aux));
          fb = cadd(fb, cscale(P.L[tb][li], aux));
        }
        P.F[ta][idx] = cadd(fa, cscale(acc_a[l2], inv_nx));
        P.F[tb][idx] = cadd(fb, cscale(acc_b[l2], inv_nx));
      }
    }
  }
}

int launch_pae(tups_ctx* ctx) {
  const auto& d = ctx->d;
  if (d.Nl > PAE_NLMAX) return set_error(ctx, TUPS_ERR_BADDIM, "Nl > 13 not supported by the crossing kernel");
  PaePtrs P;
  for (int r = 0; r < 4; r++) {
    P.Phi[r] = ctx->s.G[r];
    P.PhiR[r] = ctx->s.PhiR[r];
    P.M[r] = ctx->s.M[r];
    P.L[r] = ctx->t.L[r];
    P.F[r] = ctx->s.F[r];
  }
  dim3 grid(d.Nb, 2, d.Nl);
  k_pae<<<grid, 256, 0, ctx->stream>>>(P, ctx->t.ibz, ctx->t.signs, d.Nz, d.Nf, d.Nl, d.NIBZ, d.NR,
                                       std::fabs(1.0 / ctx->FF[0] * 1.0 / ctx->FF[0]), 1.0 / d.Nx);
  return after_launch(ctx, "k_pae");
}

}  // namespace tups
