// Compiled CPU port of two oracle phases (TEST AND BASELINE INFRASTRUCTURE
// ONLY: the timed CPU baseline of the benchmark and the checker of itself
// against the numpy oracle; nothing in the product calls it).
//
// The numpy oracle (oracle/tups_oracle.py) spends most of a parquet
// iteration in fancy-index gathers and scatter-adds: the crossing
// (calculate_PAE) and the Phi(q) -> Phi(R) transform (calc_PhiR).  The
// reference runs both as compiled Fortran loop nests (SRC/parquet_EQContribs.f90:
// 44-524, SRC/parquet_PhiR.f90:196-258), so this file restates them as C++
// loop nests with OpenMP over the output, in the oracle's conventions:
//  * port_crossing follows calculate_PAE / crossing_maps / crossing_contribution
//    of the oracle: for every target slot, source channel, w2, dispatch entry
//    (parquet_EQOuter.f90:84-113) and call (with its _TR twin for w2 > 1), the
//    frequency maps of parquet_EQContribs.f90 decide which nu1 contribute, the
//    Phi(R) entries are gathered (conjugated with signs(l3) signs(l4) for the
//    _TR calls) and contracted with M over (l3, l4, R);
//  * port_phir follows calc_PhiR / phir_at_w: Phi_r(R) = (1/Nx) sum over the
//    8 symmetries and the IBZ momenta of fac(i) PhiQ[src(i)] e^{i S(Q).R}.
// All arrays are the oracle's numpy arrays (Fortran order, complex128).
#include <complex>
#include <cstdint>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;

namespace {

// the eight calls: M index (0 phbar_to_ph, 1 pp_to_ph, 2 ph_to_pp, 3 phbar_to_pp),
// target pair (0: d, m; 1: s, t), time reversal
struct Call {
  int m, pair, tr;
  int kind;  // frequency map, see maps()
};

// dispatch of calculate_PAE: source channel -> (call kind, fac1, fac2)
struct Disp {
  int kind;
  double f1, f2;
};
// kinds: 0 phbar_to_ph, 1 pp_to_ph, 2 ph_to_pp, 3 phbar_to_pp (the _TR twin is kind + 4)
const Disp kDisp[4][3] = {
    {{0, -0.5, -0.5}, {2, 0.5, 0.5}, {3, 0.5, -0.5}},   // d
    {{0, -1.5, 0.5}, {2, -1.5, 0.5}, {3, -1.5, -0.5}},  // m
    {{1, 0.5, -0.5}, {-1, 0, 0}, {-1, 0, 0}},          // s
    {{1, 1.5, 0.5}, {-1, 0, 0}, {-1, 0, 0}},           // t
};
const int kDispN[4] = {3, 3, 1, 1};

inline int clampnu(int x, int Nf) { return x < 1 ? 1 : (x > Nf ? Nf : x); }

// crossing_maps of the oracle (1-based): returns false when the call does not
// reach nu1; t = target nu2, a, b = Phi(R) row / column frequencies
inline bool maps(int kind, int tr, int w2, int Om, int nu1, int Nf, int* t, int* a, int* b) {
  auto mF = [&](int x) { return -x + Nf + 1; };
  switch (kind * 2 + tr) {
    case 0:  // phbar_to_ph
      *t = nu1 + w2 - 1;
      *a = nu1;
      *b = clampnu(nu1 + Om - 1, Nf);
      return *t <= Nf;
    case 1:  // phbar_to_ph_TR
      *t = nu1 - w2 + 1;
      *a = mF(nu1);
      *b = clampnu(mF(nu1 + Om - 1), Nf);
      return *t <= Nf && *t >= 1;
    case 2:  // pp_to_ph
      *t = (w2 - 1) - (nu1 + Om - 1) + Nf + 1;
      *a = nu1;
      *b = *t;
      return *t <= Nf && *t >= 1;
    case 3: {  // pp_to_ph_TR
      const int v = nu1 + (Om + w2 - 1) - 1;
      *t = mF(v);
      *a = mF(nu1);
      *b = v;
      return v <= Nf && v >= 1;
    }
    case 4:  // ph_to_pp
      *t = (Om - 1) - (nu1 + w2 - 1) + Nf + 1;
      *a = nu1;
      *b = *t;
      return *t <= Nf && *t >= 1;
    case 5:  // ph_to_pp_TR
      *t = Om + w2 - 1 + (-nu1 + Nf + 1) - 1;
      *a = mF(nu1);
      *b = nu1 - (Om + w2 - 1) + 1;
      return *t <= Nf && *t >= 1;
    case 6:  // phbar_to_pp
      *t = nu1 + w2 - 1;
      *a = nu1;
      *b = clampnu((Om - 1) - (nu1 + w2 - 1) + Nf + 1, Nf);
      return *t <= Nf;
    case 7:  // phbar_to_pp_TR
      *t = nu1 - w2 + 1;
      *a = mF(nu1);
      *b = clampnu(nu1 - (Om + w2 - 1) + 1, Nf);
      return *t <= Nf && *t >= 1;
  }
  return false;
}

}  // namespace

extern "C" int port_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// F[r] (Nz, Nz, Nb) holds Phi_r + Lambda_r aux on entry (the first lines of
// calculate_PAE); the crossing contributions are added.  ibz: (Nb, 3) int64
// row-major (qx, qy, w); signs: (Nl) int64; M[r]: the oracle's M_ibz arrays
// (Nl, Nl, Nl, Nl, NIBZ, NR) Fortran order, in the order phbar_to_ph,
// pp_to_ph, ph_to_pp, phbar_to_pp; PhiR[r]: (Nz*Nz, Nf/2, NR).
extern "C" int port_crossing(int Nz, int Nf, int Nl, int Nb, int NR, int NIBZ, int Nx, const int64_t* ibz,
                             const int64_t* signs, const double* const* M_, const double* const* PhiR_,
                             double* const* F_) {
  const int nh = Nf / 2, nl2 = Nl * Nl, K = nl2 * NR;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* M[4];
  const cplx* PhiR[4];
  cplx* F[4];
  for (int r = 0; r < 4; r++) {
    M[r] = reinterpret_cast<const cplx*>(M_[r]);
    PhiR[r] = reinterpret_cast<const cplx*>(PhiR_[r]);
    F[r] = reinterpret_cast<cplx*>(F_[r]);
  }
  // M per (type, Q) as rows (l1, l2) x columns k = (l3, l4, R), row-major
  std::vector<cplx> Mq((size_t)4 * NIBZ * nl2 * K);
  for (int m = 0; m < 4; m++)
    for (int Q = 0; Q < NIBZ; Q++)
      for (int R = 0; R < NR; R++)
        for (int l34 = 0; l34 < nl2; l34++)
          for (int l12 = 0; l12 < nl2; l12++)
            Mq[(((size_t)m * NIBZ + Q) * nl2 + l12) * K + l34 + (size_t)nl2 * R] =
                M[m][l12 + (size_t)nl2 * (l34 + (size_t)nl2 * (Q + (size_t)NIBZ * R))];
  const double inv_nx = 1.0 / Nx;
#pragma omp parallel
  {
    std::vector<cplx> X(K), C(nl2);
#pragma omp for schedule(dynamic, 1)
    for (int q = 0; q < Nb; q++) {
      const int Om = (int)ibz[3 * q + 2];
      const int Q = q / nh;
      for (int src = 0; src < 4; src++)
        for (int w2 = 1; w2 <= nh; w2++) {
          const cplx* P = PhiR[src] + n2 * (size_t)(w2 - 1);
          for (int di = 0; di < kDispN[src]; di++) {
            const Disp& d = kDisp[src][di];
            const int pair = (d.kind == 0 || d.kind == 1) ? 0 : 1;
            const int mtype = d.kind;  // M order equals the kind order
            const cplx* Mm = Mq.data() + ((size_t)mtype * NIBZ + Q) * nl2 * K;
            for (int tr = 0; tr <= (w2 > 1 ? 1 : 0); tr++)
              for (int nu1 = 1; nu1 <= Nf; nu1++) {
                int t, a, b;
                if (!maps(d.kind, tr, w2, Om, nu1, Nf, &t, &a, &b)) continue;
                const int ai = clampnu(a, Nf) - 1, bi = clampnu(b, Nf) - 1;
                for (int R = 0; R < NR; R++)
                  for (int l4 = 0; l4 < Nl; l4++)
                    for (int l3 = 0; l3 < Nl; l3++) {
                      cplx x = P[(size_t)(l3 * Nf + ai) + (size_t)Nz * (l4 * Nf + bi) + n2 * nh * (size_t)R];
                      if (tr) x = (double)(signs[l3] * signs[l4]) * std::conj(x);
                      X[l3 + Nl * l4 + (size_t)nl2 * R] = x;
                    }
                for (int l12 = 0; l12 < nl2; l12++) {
                  const cplx* mr = Mm + (size_t)l12 * K;
                  double cr = 0.0, ci = 0.0;
                  for (int k = 0; k < K; k++) {
                    const double mrr = mr[k].real(), mri = mr[k].imag(), xr = X[k].real(), xi = X[k].imag();
                    cr += mrr * xr - mri * xi;
                    ci += mrr * xi + mri * xr;
                  }
                  C[l12] = cplx(cr, ci);
                }
                const int t1 = pair == 0 ? 0 : 2;
                for (int l2 = 0; l2 < Nl; l2++)
                  for (int l1 = 0; l1 < Nl; l1++) {
                    const size_t idx = (size_t)(l1 * Nf + nu1 - 1) + (size_t)Nz * (l2 * Nf + t - 1) + n2 * q;
                    const cplx c = C[l1 + Nl * l2];
                    F[t1][idx] += c * (d.f1 * inv_nx);
                    F[t1 + 1][idx] += c * (d.f2 * inv_nx);
                  }
              }
          }
        }
    }
  }
  return 0;
}

// PhiR[r] (Nz*Nz, Nf/2, NR) from PhiQ[r] (Nz*Nz, Nf/2, NIBZ) (G_r reshaped as
// the oracle does); src/fac: (8, Nz*Nz) symop_perm tables (int64 / double);
// expSqR: (NIBZ, NR, 8) Fortran order.
extern "C" int port_phir(int Nz, int Nf, int NIBZ, int NR, int Nx, const double* const* PhiQ_, const int64_t* src,
                         const double* fac, const double* expSqR_, double* const* PhiR_) {
  const int nh = Nf / 2;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* E = reinterpret_cast<const cplx*>(expSqR_);
  const double inv = 1.0 / Nx;
  for (int r = 0; r < 4; r++) {
    const cplx* PhiQ = reinterpret_cast<const cplx*>(PhiQ_[r]);
    cplx* out = reinterpret_cast<cplx*>(PhiR_[r]);
#pragma omp parallel
    {
      std::vector<cplx> acc(NR);
#pragma omp for schedule(static)
      for (long long iw = 0; iw < (long long)n2 * nh; iw++) {
        const size_t i = (size_t)(iw % (long long)n2);
        const int w = (int)(iw / (long long)n2);
        for (int R = 0; R < NR; R++) acc[R] = 0.0;
        for (int s = 0; s < 8; s++) {
          const double f = fac[(size_t)s * n2 + i];
          if (f == 0.0) continue;
          const size_t si = (size_t)src[(size_t)s * n2 + i];
          for (int Q = 0; Q < NIBZ; Q++) {
            const cplx v = f * PhiQ[si + n2 * ((size_t)w + (size_t)nh * Q)];
            for (int R = 0; R < NR; R++) acc[R] += v * E[Q + (size_t)NIBZ * (R + (size_t)NR * s)];
          }
        }
        for (int R = 0; R < NR; R++) out[i + n2 * ((size_t)w + (size_t)nh * R)] = acc[R] * inv;
      }
    }
  }
  return 0;
}
