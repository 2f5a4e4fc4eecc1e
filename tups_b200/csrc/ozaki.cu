// Split-precision complex GEMM on the int8 tensor cores (tcgen05.mma
// kind::i8), used by the BSE in its split mode and exported as a batched
// ZGEMM.  No counterpart in the reference (its BSE runs FP64 ZGEMMs,
// SRC/parquet_BSE.f90:72-128).
//
// Error-free splitting after Ozaki, Ogita, Oishi & Rump (Numer. Algorithms
// 59, 2012), with integer slices:
//   C = A B (complex, M x K times K x N) is the real product C' = A' B' with
//   A' = [Re A | Im A] (M x 2K) and B' whose column 2j is [Re B_j ; -Im B_j]
//   and column 2j+1 is [Im B_j ; Re B_j].  Every row of A' is scaled by 2^-e
//   (max |row| < 2^e) and cut into s int8 slices of 7 bits; every column of
//   B' likewise.  Slice products with i + j = d < s are summed exactly in
//   int32 on the tensor cores (|sum| <= s K' 127^2 < 2^31) and combined in
//   FP64: C' = 2^(e+f) sum_d 2^(-7(d+2)) D_d.
//
// Layout: slices of A' as rows of Kpad bytes (K-major), slices of B' as rows
// of Kpad bytes (one row per column of B'); Kpad = 2K rounded up to 128.
// The GEMM kernel reads 128-byte K chunks of both with TMA (128-byte
// swizzle), accumulates one diagonal d at a time in TMEM (two buffers, so
// the FP64 drain of diagonal d overlaps the MMAs of diagonal d+1), and
// folds each diagonal into an FP64 partial sum in global memory; the last
// diagonal applies the scales and the caller's epilogue.
#include <cuda.h>

#include <algorithm>
#include <cstdio>
#include <atomic>
#include <cstring>

#include "tups_device.cuh"

namespace tups {

constexpr int OZ_BM = 128;       // rows per tile (TMEM lanes)
constexpr int OZ_BK = 128;       // K bytes per pipeline stage
constexpr int OZ_STAGES = 6;     // 6 x (16 KB of A + <= 16 KB of B) in flight
constexpr int OZ_SLICE_BITS = 7;

// ---- splitting ---------------------------------------------------------------
// Operand: line = [X1 | X2] for rows of A, [Y1 ; Y2] for columns of B;
// part 2 may be absent (K2 = 0).  Instance b of a batch uses X1 + b*s1,
// X2 + b*s2, or, in BSE mode, the (q, r) vertex of the chunk.
__device__ __forceinline__ const cplx* oz_part(const OzOperand& o, int part, int inst) {
  const bool bse = part == 1 ? o.bse1 : o.bse2;
  if (bse) {
    const int q = o.q_begin + inst / 4, r = inst % 4;
    // constant indices keep the parameter struct out of local memory
    const cplx* Fr = r == 0 ? o.F[0] : r == 1 ? o.F[1] : r == 2 ? o.F[2] : o.F[3];
    return Fr + (size_t)o.Nz * o.Nz * q;
  }
  return part == 1 ? o.p1 + (size_t)o.s1 * inst : o.p2 + (size_t)o.s2 * inst;
}

// Per-instance view of an operand
struct OzLine {
  const cplx* p1;
  const cplx* p2;
  int ld1, ld2, K1;
};

__device__ __forceinline__ OzLine oz_view(const OzOperand& o, int inst) {
  OzLine v;
  v.ld1 = o.ld1;
  v.ld2 = o.ld2;
  v.K1 = o.K1;
  v.p1 = oz_part(o, 1, inst);
  v.p2 = o.K2 ? oz_part(o, 2, inst) : nullptr;
  return v;
}

// element (m, k) of a row operand (parts)
__device__ __forceinline__ cplx oz_a(const OzLine& v, int m, int k) {
  return k < v.K1 ? v.p1[m + (size_t)v.ld1 * k] : v.p2[m + (size_t)v.ld2 * (k - v.K1)];
}

// element (k, j) of a column operand (parts)
__device__ __forceinline__ cplx oz_b(const OzLine& v, int k, int j) {
  return k < v.K1 ? v.p1[k + (size_t)v.ld1 * j] : v.p2[(k - v.K1) + (size_t)v.ld2 * j];
}

__device__ __forceinline__ int oz_exponent(double maxabs) {
  int e = 0;
  if (maxabs > 0.0) frexp(maxabs, &e);
  return e;
}

// The s int8 slices of v 2^-e (|v 2^-e| < 1) are the base-128 digits, most
// significant first and carrying the sign of v, of t = trunc(v 2^(7s - e)):
// the same bytes as the repeated a = trunc(128 r), r = 128 r - a of the
// error-free splitting (all steps exact in FP64), with
// one scaling and one conversion instead of 4 s FP64 operations.  |t| <
// 2^(7s) <= 2^56, so t is an exact int64.
__device__ __forceinline__ long long oz_fixed(double v, int e, int s) {
  return __double2ll_rz(ldexp(v, OZ_SLICE_BITS * s - e));
}
// digit i (0 = most significant) of t as a byte
__device__ __forceinline__ uint32_t oz_digit(long long t, int i, int s) {
  const long long u = t < 0 ? -t : t;
  const int d = (int)((u >> (OZ_SLICE_BITS * (s - 1 - i))) & 127);
  return (uint32_t)(uint8_t)(int8_t)(t < 0 ? -d : d);
}

// Rows of A': one CTA per 32 rows of one instance.  out: [inst][s][M][Kpad].
// Pass 1 finds each row's scale (a warp per 8 columns at a time, four loads
// in flight per thread); pass 2 stages 32 x 64 complex tiles in shared
// memory (eight loads in flight per thread) and writes each row's slices as
// 8-byte runs.
constexpr int OZ_RT = 64;  // columns per staged tile of the row slicer
__global__ void __launch_bounds__(256, 3) k_oz_split_rows(OzOperand A, int M, int s, int Kpad, int8_t* __restrict__ out,
                                                       double* __restrict__ rscale) {
  const int inst = blockIdx.y;
  const int m0 = blockIdx.x * 32;
  const int Kc = A.K1 + A.K2;
  const OzLine V = oz_view(A, inst);
  __shared__ double smax[8][33];
  __shared__ int sexp[32];
  __shared__ cplx tile[OZ_RT][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  {
    const int m = m0 + lane;
    double mx0 = 0.0, mx1 = 0.0, mx2 = 0.0, mx3 = 0.0;
    if (m < M) {
      int k = w;
      for (; k + 24 < Kc; k += 32) {
        const cplx v0 = oz_a(V, m, k), v1 = oz_a(V, m, k + 8), v2 = oz_a(V, m, k + 16), v3 = oz_a(V, m, k + 24);
        mx0 = fmax(mx0, fmax(fabs(v0.x), fabs(v0.y)));
        mx1 = fmax(mx1, fmax(fabs(v1.x), fabs(v1.y)));
        mx2 = fmax(mx2, fmax(fabs(v2.x), fabs(v2.y)));
        mx3 = fmax(mx3, fmax(fabs(v3.x), fabs(v3.y)));
      }
      for (; k < Kc; k += 8) {
        const cplx v = oz_a(V, m, k);
        mx0 = fmax(mx0, fmax(fabs(v.x), fabs(v.y)));
      }
    }
    smax[w][lane] = fmax(fmax(mx0, mx1), fmax(mx2, mx3));
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    double mx = 0.0;
    for (int i = 0; i < 8; i++) mx = fmax(mx, smax[i][threadIdx.x]);
    const int e = oz_exponent(mx);
    sexp[threadIdx.x] = e;
    const int m = m0 + threadIdx.x;
    if (m < M) rscale[(size_t)inst * M + m] = ldexp(1.0, e);
  }
  __syncthreads();
  const size_t slice_stride = (size_t)M * Kpad;
  int8_t* base = out + (size_t)inst * s * slice_stride;
  // thread -> (row rr, 8 consecutive columns 8 cg .. 8 cg + 7): 8 groups x 32 rows
  const int cg = threadIdx.x & 7, rr = threadIdx.x >> 3;
  const int m = m0 + rr;
  const int e = sexp[rr];
  const bool vec = (Kc & 7) == 0;
  for (int k0 = 0; k0 < Kc; k0 += OZ_RT) {
    // load a 32 x 64 tile, rows fastest: eight independent loads per thread
    cplx v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int x = threadIdx.x + 256 * j;
      const int r = x & 31, c = x >> 5;
      const int mm = m0 + r, k = k0 + c;
      v[j] = (mm < M && k < Kc) ? oz_a(V, mm, k) : cmk(0.0, 0.0);
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int x = threadIdx.x + 256 * j;
      tile[x >> 5][x & 31] = v[j];
    }
    __syncthreads();
    const int k = k0 + cg * 8;
    if (m < M && k < Kc) {
      uint32_t lre[8], hre[8], lim[8], him[8];
#pragma unroll
      for (int i = 0; i < 8; i++) lre[i] = hre[i] = lim[i] = him[i] = 0u;
      // column c = (j + cg) & 7 at step j: the eight lanes of a quarter warp
      // (cg = 0..7, one row) then read eight different banks
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int c = (j + cg) & 7;
        const cplx x = (k + c < Kc) ? tile[cg * 8 + c][rr] : cmk(0.0, 0.0);
        const long long tr = oz_fixed(x.x, e, s), ti = oz_fixed(x.y, e, s);
        const int sh = 8 * (c & 3);
        const bool lo = c < 4;
#pragma unroll
        for (int i = 0; i < 8; i++)
          if (i < s) {
            const uint32_t dr = oz_digit(tr, i, s) << sh, di = oz_digit(ti, i, s) << sh;
            lre[i] |= lo ? dr : 0u;
            hre[i] |= lo ? 0u : dr;
            lim[i] |= lo ? di : 0u;
            him[i] |= lo ? 0u : di;
          }
      }
      int8_t* row = base + (size_t)m * Kpad;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        if (i >= s) continue;
        int8_t* dst = row + (size_t)i * slice_stride;
        if (vec && k + 7 < Kc) {
          *reinterpret_cast<uint2*>(dst + k) = make_uint2(lre[i], hre[i]);
          *reinterpret_cast<uint2*>(dst + Kc + k) = make_uint2(lim[i], him[i]);
        } else {
          for (int c = 0; c < 8 && k + c < Kc; c++) {
            dst[k + c] = (int8_t)((c < 4 ? lre[i] : hre[i]) >> (8 * (c & 3)));
            dst[Kc + k + c] = (int8_t)((c < 4 ? lim[i] : him[i]) >> (8 * (c & 3)));
          }
        }
      }
    }
    __syncthreads();
  }
  // zero the K padding [2 Kc, Kpad) of this CTA's rows
  const int pad = Kpad - 2 * Kc;
  for (int x = threadIdx.x; x < 32 * pad * s; x += 256) {
    const int b = x % pad, r = (x / pad) % 32, i = x / (pad * 32);
    if (m0 + r < M) base[(size_t)i * slice_stride + (size_t)(m0 + r) * Kpad + 2 * Kc + b] = 0;
  }
}

// Columns of B': one warp per complex column j of B (K1 + K2 long); writes
// rows 2j and 2j+1 of every slice.  out: [inst][s][2N][Kpad].  The column
// is read twice (scale, then slices); the second read hits L1.
__global__ void __launch_bounds__(256) k_oz_split_cols(OzOperand B, int N, int s, int Kpad, int8_t* __restrict__ out,
                                                       double* __restrict__ cscale) {
  const int inst = blockIdx.y;
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= N) return;
  const int Kc = B.K1 + B.K2;
  const OzLine V = oz_view(B, inst);
  double mx0 = 0.0, mx1 = 0.0, mx2 = 0.0, mx3 = 0.0;
  {
    int k = lane;
    for (; k + 96 < Kc; k += 128) {
      const cplx v0 = oz_b(V, k, j), v1 = oz_b(V, k + 32, j), v2 = oz_b(V, k + 64, j), v3 = oz_b(V, k + 96, j);
      mx0 = fmax(mx0, fmax(fabs(v0.x), fabs(v0.y)));
      mx1 = fmax(mx1, fmax(fabs(v1.x), fabs(v1.y)));
      mx2 = fmax(mx2, fmax(fabs(v2.x), fabs(v2.y)));
      mx3 = fmax(mx3, fmax(fabs(v3.x), fabs(v3.y)));
    }
    for (; k < Kc; k += 32) {
      const cplx v = oz_b(V, k, j);
      mx0 = fmax(mx0, fmax(fabs(v.x), fabs(v.y)));
    }
  }
  const double mx = warp_max(fmax(fmax(mx0, mx1), fmax(mx2, mx3)));
  const int e = oz_exponent(mx);
  if (lane == 0) cscale[(size_t)inst * N + j] = ldexp(1.0, e);
  const size_t slice_stride = (size_t)2 * N * Kpad;
  int8_t* r0 = out + (size_t)inst * s * slice_stride + (size_t)(2 * j) * Kpad;
  int8_t* r1 = r0 + Kpad;
  const bool vec = (Kc & 3) == 0;
  for (int k = lane * 4; k < Kc; k += 128) {
    cplx v[4];
#pragma unroll
    for (int c = 0; c < 4; c++) v[c] = k + c < Kc ? oz_b(V, k + c, j) : cmk(0.0, 0.0);
    uint32_t wre[8], wim[8];
#pragma unroll
    for (int i = 0; i < 8; i++) wre[i] = wim[i] = 0u;
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const long long tr = oz_fixed(v[c].x, e, s), ti = oz_fixed(v[c].y, e, s);
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (i < s) {
          wre[i] |= oz_digit(tr, i, s) << (8 * c);
          wim[i] |= oz_digit(ti, i, s) << (8 * c);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      if (i >= s) continue;
      int8_t* d0 = r0 + (size_t)i * slice_stride;
      int8_t* d1 = r1 + (size_t)i * slice_stride;
      // the slices of -Im are the negated slices of Im (truncation is odd):
      // a byte-wise negation of the packed digits
      const uint32_t wnim = __vneg4(wim[i]);
      if (vec && k + 3 < Kc) {
        *reinterpret_cast<uint32_t*>(d0 + k) = wre[i];
        *reinterpret_cast<uint32_t*>(d0 + Kc + k) = wnim;
        *reinterpret_cast<uint32_t*>(d1 + k) = wim[i];
        *reinterpret_cast<uint32_t*>(d1 + Kc + k) = wre[i];
      } else {
        for (int c = 0; c < 4 && k + c < Kc; c++) {
          d0[k + c] = (int8_t)(wre[i] >> (8 * c));
          d0[Kc + k + c] = (int8_t)(wnim >> (8 * c));
          d1[k + c] = (int8_t)(wim[i] >> (8 * c));
          d1[Kc + k + c] = (int8_t)(wre[i] >> (8 * c));
        }
      }
    }
  }
  // zero the K padding [2 Kc, Kpad) of rows 2j, 2j+1
  for (int i = 0; i < s; i++)
    for (int b = 2 * Kc + lane; b < Kpad; b += 32) {
      r0[(size_t)i * slice_stride + b] = 0;
      r1[(size_t)i * slice_stride + b] = 0;
    }
}

// ---- tcgen05 helpers ------------------------------------------------------------
__device__ __forceinline__ uint32_t oz_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(oz_smem(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(oz_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// SM cycles a wait of the work loop may take before the CTA gives up
// (about 2 s at 1.965 GHz); the waits of the abort path itself, for copies
// and MMAs already in flight, always use this default
constexpr long long OZ_WAIT_CYCLES = 4000000000LL;

// bounded wait: false when the CTA's abort flag is set (honor_abort) or
// `limit` SM cycles pass, in which case the abort flag is set
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                          bool honor_abort = true, long long limit = OZ_WAIT_CYCLES) {
  const long long t0 = clock64();
  for (uint32_t it = 0;; it++) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 255) {
      if (honor_abort && *abort_flag) return false;
      if (clock64() - t0 > limit) {
        *abort_flag = 1;
        return false;
      }
    }
  }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(oz_smem(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(oz_smem(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(oz_smem(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(oz_smem(bar))
               : "memory");
}

__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, int32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// K-major operand tile with 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t oz_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// ---- the GEMM ----------------------------------------------------------------------
// Persistent: each CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... of
// the list (instance, row tile, column tile), instance outermost.  Per tile
// and diagonal d the MMA warp accumulates the slice products (i, d - i) over
// K into one of OZ_NBUF TMEM buffers; the eight drain warps (two per TMEM
// lane quarter, each owning half of the tile's columns) fold the finished
// buffer into FP64 registers, acc += 2^(-7(d+2)) D_d, while the MMAs of the
// next diagonals proceed; after the last diagonal they apply the row and
// column scales and the epilogue, and the next tile starts.
enum { OZ_EPI_ZGEMM = 0, OZ_EPI_BSE = 1, OZ_EPI_SUB = 2 };

constexpr int OZ_NBUF = 4;            // TMEM accumulator buffers
constexpr int OZ_MAX_NT = 128;        // columns per tile
constexpr int OZ_HALF = OZ_MAX_NT / 2;
constexpr int OZ_DRAIN_WARPS = 8;
constexpr int OZ_THREADS2 = (OZ_DRAIN_WARPS + 2) * 32;  // + MMA warp + TMA warp

struct OzGemm {
  int M, N;            // complex output size; N' = 2N real columns
  int s;               // slices
  int kchunks;         // Kpad / 128
  int n_tile;          // real columns per tile (multiple of 16, <= 128)
  int m_tiles, n_tiles, tiles;
  const double* rscale;  // [inst][M]
  const double* cscale;  // [inst][N]
  double* status;        // set to status_code on a timed-out wait
  double status_code;
  int epi;
  cplx* C;               // OZ_EPI_ZGEMM: col-major M x N per instance; OZ_EPI_SUB: C -= A B
  int ldc;               // OZ_EPI_SUB: leading dimension and instance stride of C
  long long c_stride;
  cplx* F[4];            // OZ_EPI_BSE: Phi = scale[r] C + omf (F - G) over G
  cplx* G[4];
  double scale[4];
  double omf;
  int q_begin;
  long long wait_cycles;  // limit of the work loop's waits
  int stall_test;         // 1: the MMA warp first waits on a barrier nothing signals
};

__device__ __forceinline__ void tc_ld8(uint32_t taddr, int32_t* v) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}

__global__ void __launch_bounds__(OZ_THREADS2, 1)
    k_oz_gemm(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzGemm P) {
  extern __shared__ uint8_t oz_dyn[];
  __shared__ uint64_t full_bar[OZ_STAGES], empty_bar[OZ_STAGES], accf_bar[OZ_NBUF], acce_bar[OZ_NBUF], done_bar;
  __shared__ uint64_t never_bar;  // initialised, never arrived on: the stall test waits here
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ int issued_sh, consumed_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int Np = 2 * P.N;
  const uint32_t a_bytes = OZ_BM * OZ_BK, b_bytes = (uint32_t)P.n_tile * OZ_BK;
  const uint32_t dyn = (oz_smem(oz_dyn) + 1023u) & ~1023u;
  auto sA = [&](int st) { return dyn + (uint32_t)st * (a_bytes + b_bytes); };
  auto sB = [&](int st) { return dyn + (uint32_t)st * (a_bytes + b_bytes) + a_bytes; };
  const int per_inst = P.m_tiles * P.n_tiles;

  if (threadIdx.x == 0) {
    for (int i = 0; i < OZ_STAGES; i++) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < OZ_NBUF; i++) {
      mbar_init(&accf_bar[i], 1);
      mbar_init(&acce_bar[i], OZ_DRAIN_WARPS * 32);
    }
    mbar_init(&done_bar, 1);
    mbar_init(&never_bar, 1);
    abort_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == OZ_DRAIN_WARPS) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tmem_base_sh)),
                 "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp == OZ_DRAIN_WARPS + 1) {
    // ---- TMA producer ----
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < P.tiles && ok; t += gridDim.x) {
        const int inst = t / per_inst, rem = t % per_inst;
        const int m0 = (rem % P.m_tiles) * OZ_BM, n0 = (rem / P.m_tiles) * P.n_tile;
        for (int d = 0; d < P.s && ok; d++)
          for (int i = 0; i <= d && ok; i++) {
            const int ya = (inst * P.s + i) * P.M + m0;
            const int yb = (inst * P.s + (d - i)) * Np + n0;
            for (int kc = 0; kc < P.kchunks; kc++) {
              if (!mbar_wait(&empty_bar[stage], phase ^ 1u, &abort_sh, true, P.wait_cycles)) {
                ok = false;
                break;
              }
              mbar_expect_tx(&full_bar[stage], a_bytes + b_bytes);
              tma_load_2d(sA(stage), &tmA, kc * OZ_BK, ya, &full_bar[stage]);
              tma_load_2d(sB(stage), &tmB, kc * OZ_BK, yb, &full_bar[stage]);
              issued++;
              if (++stage == OZ_STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
          }
      }
      issued_sh = issued;
    }
  } else if (warp == OZ_DRAIN_WARPS) {
    // ---- MMA issuer ----
    if (lane == 0) {
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(P.n_tile >> 3) << 17) |
                             ((uint32_t)(OZ_BM >> 4) << 24);
      int stage = 0;
      uint32_t phase = 0;
      int consumed = 0;
      int nacc = 0;  // accumulations issued so far (one per tile and diagonal)
      bool ok = true;
      // failure-path test: a wait that can only run out, before any MMA
      if (P.stall_test) ok = mbar_wait(&never_bar, 0, &abort_sh, true, P.wait_cycles);
      for (int t = blockIdx.x; t < P.tiles && ok; t += gridDim.x)
        for (int d = 0; d < P.s && ok; d++, nacc++) {
          const int buf = nacc % OZ_NBUF;
          if (nacc >= OZ_NBUF &&
              !mbar_wait(&acce_bar[buf], (uint32_t)((nacc - OZ_NBUF) / OZ_NBUF) & 1u, &abort_sh, true,
                         P.wait_cycles)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dtm = tmem + (uint32_t)(buf * OZ_MAX_NT);
          uint32_t accum = 0;
          for (int i = 0; i <= d && ok; i++)
            for (int kc = 0; kc < P.kchunks; kc++) {
              if (!mbar_wait(&full_bar[stage], phase, &abort_sh, true, P.wait_cycles)) {
                ok = false;
                break;
              }
              consumed++;
              tc_fence_after();
              const uint64_t da = oz_desc(sA(stage)), db = oz_desc(sB(stage));
#pragma unroll
              for (int kk = 0; kk < OZ_BK / 32; kk++) {
                tc_mma_i8(dtm, da + 2 * kk, db + 2 * kk, idesc, accum);
                accum = 1;
              }
              tc_commit(&empty_bar[stage]);
              if (++stage == OZ_STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
          if (ok) tc_commit(&accf_bar[buf]);
        }
      consumed_sh = consumed;
      tc_commit(&done_bar);
      mbar_wait(&done_bar, 0, &abort_sh, false);
    }
  } else {
    // ---- drain: warp w reads TMEM lanes 32 (w % 4) .. + 31 and columns
    //      [h n_tile/2, (h+1) n_tile/2), h = w / 4 ----
    const int quarter = warp & 3, h = warp >> 2;
    const int half = P.n_tile >> 1;
    const int row = quarter * 32 + lane;
    double acc[OZ_HALF];
    int nacc = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < P.tiles && ok; t += gridDim.x) {
      const int inst = t / per_inst, rem = t % per_inst;
      const int m0 = (rem % P.m_tiles) * OZ_BM, n0 = (rem / P.m_tiles) * P.n_tile;
      const int m = m0 + row;
      const bool mok = m < P.M;
#pragma unroll
      for (int c = 0; c < OZ_HALF; c++) acc[c] = 0.0;
      for (int d = 0; d < P.s; d++, nacc++) {
        const int buf = nacc % OZ_NBUF;
        if (!mbar_wait(&accf_bar[buf], (uint32_t)(nacc / OZ_NBUF) & 1u, &abort_sh, true, P.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const double w = ldexp(1.0, -OZ_SLICE_BITS * (d + 2));
        const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * OZ_MAX_NT + h * half);
#pragma unroll
        for (int c = 0; c < OZ_HALF; c += 8) {
          if (c < half) {
            int32_t v[8];
            tc_ld8(tb + (uint32_t)c, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 8; e++) acc[c + e] = fma((double)v[e], w, acc[c + e]);
          }
        }
        tc_fence_before();
        mbar_arrive(&acce_bar[buf]);
      }
      if (!ok) break;
      if (!mok) continue;
      // scales and the epilogue; complex column jc = (n0 + h half + c) / 2
      const double rs = P.rscale[(size_t)inst * P.M + m];
      cplx* Cq = nullptr;
      const cplx* Fq = nullptr;
      cplx* Gq = nullptr;
      int r = 0;
      if (P.epi == OZ_EPI_BSE) {
        const int q = P.q_begin + inst / 4;
        r = inst % 4;
        Fq = P.F[r] + (size_t)P.M * P.M * q;
        Gq = P.G[r] + (size_t)P.M * P.M * q;
      } else if (P.epi == OZ_EPI_SUB) {
        Cq = P.C + (size_t)inst * P.c_stride;
      } else {
        Cq = P.C + (size_t)inst * P.M * P.N;
      }
#pragma unroll
      for (int c = 0; c < OZ_HALF; c += 2) {
        const int np = n0 + h * half + c;
        if (c < half && np < Np) {
          const int jc = np >> 1;
          const double sc = rs * P.cscale[(size_t)inst * P.N + jc];
          const double cre = acc[c] * sc, cim = acc[c + 1] * sc;
          if (P.epi == OZ_EPI_SUB) {
            const size_t ix = m + (size_t)P.ldc * jc;
            const cplx c0 = Cq[ix];
            Cq[ix] = cmk(c0.x - cre, c0.y - cim);
            continue;
          }
          const size_t idx = m + (size_t)P.M * jc;
          if (P.epi == OZ_EPI_ZGEMM) {
            Cq[idx] = cmk(cre, cim);
          } else {
            const cplx f = Fq[idx], g = Gq[idx];
            const double sr = P.scale[r];
            Gq[idx] = cmk(__dadd_rn(__dmul_rn(sr, cre), __dmul_rn(P.omf, __dsub_rn(f.x, g.x))),
                          __dadd_rn(__dmul_rn(sr, cim), __dmul_rn(P.omf, __dsub_rn(f.y, g.y))));
          }
        }
      }
    }
  }

  __syncthreads();
  if (threadIdx.x == 0 && abort_sh) {
    *P.status = P.status_code;
    // wait for the TMA copies that were issued but never consumed
    int stage = consumed_sh % OZ_STAGES;
    uint32_t phase = (uint32_t)(consumed_sh / OZ_STAGES) & 1u;
    for (int k = consumed_sh; k < issued_sh; k++) {
      mbar_wait(&full_bar[stage], phase, &abort_sh, false);
      if (++stage == OZ_STAGES) {
        stage = 0;
        phase ^= 1u;
      }
    }
  }
  __syncthreads();
  if (warp == OZ_DRAIN_WARPS) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
  }
}

// ---- the GEMM on CTA pairs (tcgen05 cta_group::2) ------------------------------
// The same tiles, diagonal schedule and FP64 folding as k_oz_gemm (so the
// same bits), but a cluster of two CTAs computes a 256 x n_tile tile with
// one M = 256 MMA per K step: CTA r stages rows 128 r .. 128 r + 127 of the
// pair's A rows and half of the tile's B columns (n_tile / 2 rows of B'), so
// each SM's tensor core reads 4 KB + n_tile x 16 B of operands per MMA
// instead of 4 KB + n_tile x 32 B.  The leader (cluster rank 0) issues the
// MMAs and owns the stage-full barriers (both CTAs' copies complete there);
// the MMA completions reach both CTAs' stage-empty and accumulator-full
// barriers by multicast commits; each CTA's drain warps read their own TMEM
// rows and arrive on the leader's accumulator-empty barrier.  Only the
// tensor maps of this GPU's own memory are read, and no copy multicasts.
constexpr int OZ2_STAGES = 8;  // 8 x (16 KB of A + <= 8 KB of B)

__device__ __forceinline__ uint32_t oz_cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// the shared::cluster address of `addr` (a shared::cta address) in CTA `rank`
__device__ __forceinline__ uint32_t oz_mapa(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void oz_cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_cl(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(oz_smem(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait with cluster-scope acquire (barriers that other CTAs signal)
__device__ __forceinline__ bool mbar_wait_cl(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                             bool honor_abort = true, long long limit = OZ_WAIT_CYCLES) {
  const long long t0 = clock64();
  for (uint32_t it = 0;; it++) {
    if (mbar_try_cl(bar, parity)) return true;
    if ((it & 255) == 255) {
      if (honor_abort && *abort_flag) return false;
      if (clock64() - t0 > limit) {
        *abort_flag = 1;
        return false;
      }
    }
  }
}
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr) : "memory");
}
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t bar_cluster) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar_cluster)
      : "memory");
}
// MMA completion to the barrier at this offset in the CTAs of `mask`
__device__ __forceinline__ void tc_commit_pair(uint64_t* bar, uint16_t mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          oz_smem(bar)),
      "h"(mask)
      : "memory");
}
__device__ __forceinline__ void tc_mma_i8_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                               uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u), "r"(0u),
      "r"(0u), "r"(0u));
}

// P.m_tiles counts 256-row pair tiles here
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(OZ_THREADS2, 1)
    k_oz_gemm2(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzGemm P) {
  extern __shared__ uint8_t oz_dyn[];
  __shared__ uint64_t full_bar[OZ2_STAGES], empty_bar[OZ2_STAGES], accf_bar[OZ_NBUF], acce_bar[OZ_NBUF], done_bar;
  __shared__ uint64_t never_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ volatile int abort_sh;
  __shared__ int issued_sh, consumed_sh;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t crank = oz_cluster_rank();
  const bool leader = crank == 0;
  const int Np = 2 * P.N;
  const int NT = P.n_tile, HB = NT >> 1;  // B' rows staged by each CTA
  const uint32_t a_bytes = OZ_BM * OZ_BK, b_bytes = (uint32_t)HB * OZ_BK;
  const uint32_t dyn = (oz_smem(oz_dyn) + 1023u) & ~1023u;
  auto sA = [&](int st) { return dyn + (uint32_t)st * (a_bytes + b_bytes); };
  auto sB = [&](int st) { return dyn + (uint32_t)st * (a_bytes + b_bytes) + a_bytes; };
  const int per_inst = P.m_tiles * P.n_tiles;
  const int cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;

  if (threadIdx.x == 0) {
    for (int i = 0; i < OZ2_STAGES; i++) {
      mbar_init(&full_bar[i], 1);
      mbar_init(&empty_bar[i], 1);
    }
    for (int i = 0; i < OZ_NBUF; i++) {
      mbar_init(&accf_bar[i], 1);
      mbar_init(&acce_bar[i], 2 * OZ_DRAIN_WARPS * 32);
    }
    mbar_init(&done_bar, 1);
    mbar_init(&never_bar, 1);
    abort_sh = 0;
    issued_sh = 0;
    consumed_sh = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == OZ_DRAIN_WARPS) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(oz_smem(&tmem_base_sh)),
                 "r"(512u));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  // both CTAs' barriers exist before either CTA signals the other's
  oz_cluster_sync();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp == OZ_DRAIN_WARPS + 1) {
    // ---- TMA producer (both CTAs): own rows of A, own half of B' ----
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int issued = 0;
      bool ok = true;
      for (int t = cid; t < P.tiles && ok; t += ncl) {
        const int inst = t / per_inst, rem = t % per_inst;
        const int m0 = (rem % P.m_tiles) * (2 * OZ_BM) + (int)crank * OZ_BM;
        const int n0 = (rem / P.m_tiles) * NT + (int)crank * HB;
        for (int d = 0; d < P.s && ok; d++)
          for (int i = 0; i <= d && ok; i++) {
            const int ya = (inst * P.s + i) * P.M + m0;
            const int yb = (inst * P.s + (d - i)) * Np + n0;
            for (int kc = 0; kc < P.kchunks; kc++) {
              if (!mbar_wait_cl(&empty_bar[stage], phase ^ 1u, &abort_sh, true, P.wait_cycles)) {
                ok = false;
                break;
              }
              // the leader's stage-full barrier counts both CTAs' bytes
              if (leader) mbar_expect_tx(&full_bar[stage], 2 * (a_bytes + b_bytes));
              const uint32_t fb = oz_mapa(oz_smem(&full_bar[stage]), 0);
              tma_load_2d_pair(sA(stage), &tmA, kc * OZ_BK, ya, fb);
              tma_load_2d_pair(sB(stage), &tmB, kc * OZ_BK, yb, fb);
              issued++;
              if (++stage == OZ2_STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
          }
      }
      issued_sh = issued;
    }
  } else if (warp == OZ_DRAIN_WARPS) {
    // ---- MMA issuer: the leader only ----
    if (lane == 0 && leader) {
      const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) |
                             ((uint32_t)((2 * OZ_BM) >> 4) << 24);
      int stage = 0;
      uint32_t phase = 0;
      int consumed = 0;
      int nacc = 0;
      bool ok = true;
      if (P.stall_test) ok = mbar_wait(&never_bar, 0, &abort_sh, true, P.wait_cycles);
      for (int t = cid; t < P.tiles && ok; t += ncl)
        for (int d = 0; d < P.s && ok; d++, nacc++) {
          const int buf = nacc % OZ_NBUF;
          if (nacc >= OZ_NBUF &&
              !mbar_wait_cl(&acce_bar[buf], (uint32_t)((nacc - OZ_NBUF) / OZ_NBUF) & 1u, &abort_sh, true,
                            P.wait_cycles)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dtm = tmem + (uint32_t)(buf * OZ_MAX_NT);
          uint32_t accum = 0;
          for (int i = 0; i <= d && ok; i++)
            for (int kc = 0; kc < P.kchunks; kc++) {
              if (!mbar_wait_cl(&full_bar[stage], phase, &abort_sh, true, P.wait_cycles)) {
                ok = false;
                break;
              }
              consumed++;
              tc_fence_after();
              const uint64_t da = oz_desc(sA(stage)), db = oz_desc(sB(stage));
#pragma unroll
              for (int kk = 0; kk < OZ_BK / 32; kk++) {
                tc_mma_i8_pair(dtm, da + 2 * kk, db + 2 * kk, idesc, accum);
                accum = 1;
              }
              tc_commit_pair(&empty_bar[stage], 0x3);
              if (++stage == OZ2_STAGES) {
                stage = 0;
                phase ^= 1u;
              }
            }
          if (ok) tc_commit_pair(&accf_bar[buf], 0x3);
        }
      consumed_sh = consumed;
      tc_commit_pair(&done_bar, 0x1);
      mbar_wait_cl(&done_bar, 0, &abort_sh, false);
    }
  } else {
    // ---- drain (both CTAs): own TMEM lanes = own 128 rows of the pair tile ----
    const int quarter = warp & 3, h = warp >> 2;
    const int half = NT >> 1;
    const int row = quarter * 32 + lane;
    const uint32_t acce_leader0 = oz_mapa(oz_smem(&acce_bar[0]), 0);
    double acc[OZ_HALF];
    int nacc = 0;
    bool ok = true;
    for (int t = cid; t < P.tiles && ok; t += ncl) {
      const int inst = t / per_inst, rem = t % per_inst;
      const int m0 = (rem % P.m_tiles) * (2 * OZ_BM) + (int)crank * OZ_BM;
      const int n0 = (rem / P.m_tiles) * NT;
      const int m = m0 + row;
      const bool mok = m < P.M;
#pragma unroll
      for (int c = 0; c < OZ_HALF; c++) acc[c] = 0.0;
      for (int d = 0; d < P.s; d++, nacc++) {
        const int buf = nacc % OZ_NBUF;
        if (!mbar_wait_cl(&accf_bar[buf], (uint32_t)(nacc / OZ_NBUF) & 1u, &abort_sh, true, P.wait_cycles)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const double w = ldexp(1.0, -OZ_SLICE_BITS * (d + 2));
        const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * OZ_MAX_NT + h * half);
#pragma unroll
        for (int c = 0; c < OZ_HALF; c += 8) {
          if (c < half) {
            int32_t v[8];
            tc_ld8(tb + (uint32_t)c, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 8; e++) acc[c + e] = fma((double)v[e], w, acc[c + e]);
          }
        }
        tc_fence_before();
        mbar_arrive_remote(acce_leader0 + (uint32_t)(buf * sizeof(uint64_t)));
      }
      if (!ok) break;
      if (!mok) continue;
      const double rs = P.rscale[(size_t)inst * P.M + m];
      cplx* Cq = nullptr;
      const cplx* Fq = nullptr;
      cplx* Gq = nullptr;
      int r = 0;
      if (P.epi == OZ_EPI_BSE) {
        const int q = P.q_begin + inst / 4;
        r = inst % 4;
        const cplx* Fr = r == 0 ? P.F[0] : r == 1 ? P.F[1] : r == 2 ? P.F[2] : P.F[3];
        cplx* Gr = r == 0 ? P.G[0] : r == 1 ? P.G[1] : r == 2 ? P.G[2] : P.G[3];
        Fq = Fr + (size_t)P.M * P.M * q;
        Gq = Gr + (size_t)P.M * P.M * q;
      } else if (P.epi == OZ_EPI_SUB) {
        Cq = P.C + (size_t)inst * P.c_stride;
      } else {
        Cq = P.C + (size_t)inst * P.M * P.N;
      }
      const double sr = r == 0 ? P.scale[0] : r == 1 ? P.scale[1] : r == 2 ? P.scale[2] : P.scale[3];
#pragma unroll
      for (int c = 0; c < OZ_HALF; c += 2) {
        const int np = n0 + h * half + c;
        if (c < half && np < Np) {
          const int jc = np >> 1;
          const double sc = rs * P.cscale[(size_t)inst * P.N + jc];
          const double cre = acc[c] * sc, cim = acc[c + 1] * sc;
          if (P.epi == OZ_EPI_SUB) {
            const size_t ix = m + (size_t)P.ldc * jc;
            const cplx c0 = Cq[ix];
            Cq[ix] = cmk(c0.x - cre, c0.y - cim);
            continue;
          }
          const size_t idx = m + (size_t)P.M * jc;
          if (P.epi == OZ_EPI_ZGEMM) {
            Cq[idx] = cmk(cre, cim);
          } else {
            const cplx f = Fq[idx], g = Gq[idx];
            Gq[idx] = cmk(__dadd_rn(__dmul_rn(sr, cre), __dmul_rn(P.omf, __dsub_rn(f.x, g.x))),
                          __dadd_rn(__dmul_rn(sr, cim), __dmul_rn(P.omf, __dsub_rn(f.y, g.y))));
          }
        }
      }
    }
  }

  __syncthreads();
  if (threadIdx.x == 0 && abort_sh) {
    *P.status = P.status_code;
    if (leader) {
      // wait for the stages whose copies were issued but never consumed
      int stage = consumed_sh % OZ2_STAGES;
      uint32_t phase = (uint32_t)(consumed_sh / OZ2_STAGES) & 1u;
      for (int k = consumed_sh; k < issued_sh; k++) {
        mbar_wait_cl(&full_bar[stage], phase, &abort_sh, false);
        if (++stage == OZ2_STAGES) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
  }
  __syncthreads();
  // neither CTA frees its shared or tensor memory while the other may still use it
  oz_cluster_sync();
  if (warp == OZ_DRAIN_WARPS) {
    __syncwarp();
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u));
  }
}

// ---- host side ----------------------------------------------------------------------
// the work loop's wait limit (0: OZ_WAIT_CYCLES) and a pending stall test,
// set by tups_set_split_wait; the stall test applies to the next launch only
static std::atomic<long long> g_oz_wait_cycles{0};
static std::atomic<int> g_oz_stall_test{0};
static std::atomic<int> g_oz_n_tile{0};  // 0: oz_n_tile
static std::atomic<int> g_oz_pairs{0};   // 1: k_oz_gemm2 (CTA pairs) for M >= 256

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 2-D byte tensor [rows][Kpad], boxes of 128 bytes x box_rows, 128-byte swizzle
static bool make_map(CUtensorMap* map, const int8_t* base, long long rows, int Kpad, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return false;
  if (((uintptr_t)base & 15) || (Kpad % OZ_BK) || box_rows < 1 || box_rows > 256) return false;
  cuuint64_t dims[2] = {(cuuint64_t)Kpad, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)Kpad};
  cuuint32_t box[2] = {(cuuint32_t)OZ_BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int oz_kpad(int K) { return (int)(((long long)2 * K + OZ_BK - 1) / OZ_BK * OZ_BK); }

// columns per tile: multiple of 16, <= 128; cost = tiles x (columns + 64),
// the 64 standing for the per-tile cost of streaming the A rows
int oz_n_tile(int N) {
  const int Np = 2 * N;
  int best = 16;
  long long best_cost = -1;
  for (int t = 16; t <= OZ_MAX_NT; t += 16) {
    const long long cost = (long long)((Np + t - 1) / t) * (t + 64);
    if (best_cost < 0 || cost < best_cost || (cost == best_cost && t > best)) {
      best = t;
      best_cost = cost;
    }
  }
  return best;
}

size_t oz_smem_bytes(int n_tile) {
  size_t s = (size_t)OZ_STAGES * (OZ_BM * OZ_BK + (size_t)n_tile * OZ_BK) + 1024;
  return std::max<size_t>(s, 120 * 1024);  // one CTA per SM: the CTA owns all 512 TMEM columns
}

OzWork oz_work_layout(int batch, int M, int N, int K, int s) {
  OzWork w;
  w.Kpad = oz_kpad(K);
  w.a_bytes = (size_t)batch * s * M * w.Kpad;
  w.b_bytes = (size_t)batch * s * 2 * N * w.Kpad;
  w.rs_bytes = (size_t)batch * M * sizeof(double);
  w.cs_bytes = (size_t)batch * N * sizeof(double);
  w.acc_bytes = 0;  // the FP64 sums live in registers
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  w.total = up(w.a_bytes) + up(w.b_bytes) + up(w.rs_bytes) + up(w.cs_bytes) + up(w.acc_bytes) + 256;
  return w;
}

void oz_bind_work(OzRun& R, const OzWork& w, void* base) {
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  uint8_t* p = (uint8_t*)(((uintptr_t)base + 255) & ~(uintptr_t)255);
  R.a_slices = (int8_t*)p;
  p += up(w.a_bytes);
  R.b_slices = (int8_t*)p;
  p += up(w.b_bytes);
  R.rscale = (double*)p;
  p += up(w.rs_bytes);
  R.cscale = (double*)p;
  R.acc = nullptr;
}

// a failed CUDA step of oz_run on stderr (the batched ZGEMM entry point has no
// context to keep a message in)
static int oz_fail(const char* step, cudaError_t e) {
  std::fprintf(stderr, "tups split GEMM: %s failed: %s\n", step, e == cudaSuccess ? "-" : cudaGetErrorString(e));
  return TUPS_ERR_CUDA;
}

int oz_run(OzRun& R, cudaStream_t stream, long long* launches) {
  const int M = R.M, N = R.N, s = R.s, batch = R.batch;
  if (s < 1 || s > 8) return TUPS_ERR_BADARG;
  if (R.A.K1 + R.A.K2 != R.B.K1 + R.B.K2) return TUPS_ERR_BADDIM;
  const int K = R.A.K1 + R.A.K2;
  // exactness of the int32 sums: s K' 127^2 < 2^31
  if ((long long)s * 2 * K * 127 * 127 >= (1LL << 31)) return TUPS_ERR_BADDIM;
  const int Kpad = oz_kpad(K);
  if ((long long)batch * s * std::max(M, 2 * N) >= (1LL << 31)) return TUPS_ERR_BADDIM;
  // rows of the split kernels
  {
    dim3 g((M + 31) / 32, batch);
    k_oz_split_rows<<<g, 256, 0, stream>>>(R.A, M, s, Kpad, R.a_slices, R.rscale);
    if (launches) (*launches)++;
    dim3 gc((N + 7) / 8, batch);
    k_oz_split_cols<<<gc, 256, 0, stream>>>(R.B, N, s, Kpad, R.b_slices, R.cscale);
    if (launches) (*launches)++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return oz_fail("slice kernels launch", e);
  }
  OzGemm P;
  std::memset(&P, 0, sizeof(P));
  P.M = M;
  P.N = N;
  P.s = s;
  P.kchunks = Kpad / OZ_BK;
  const bool pairs = g_oz_pairs.load() != 0 && M >= 2 * OZ_BM;
  {
    const int nt = g_oz_n_tile.load();
    P.n_tile = nt > 0 ? nt : oz_n_tile(N);
    // CTA pairs: each CTA stages n_tile / 2 rows of B', a multiple of 16
    if (pairs) P.n_tile = std::min(OZ_MAX_NT, (P.n_tile + 31) / 32 * 32);
  }
  P.m_tiles = pairs ? (M + 2 * OZ_BM - 1) / (2 * OZ_BM) : (M + OZ_BM - 1) / OZ_BM;
  P.n_tiles = (2 * N + P.n_tile - 1) / P.n_tile;
  if ((long long)batch * P.m_tiles * P.n_tiles >= (1LL << 31)) return TUPS_ERR_BADDIM;
  P.tiles = batch * P.m_tiles * P.n_tiles;
  P.rscale = R.rscale;
  P.cscale = R.cscale;
  P.status = R.status;
  P.status_code = R.status_code;
  P.epi = R.epi;
  P.C = R.C;
  P.ldc = R.ldc;
  P.c_stride = R.c_stride;
  for (int r = 0; r < 4; r++) {
    P.F[r] = R.F[r];
    P.G[r] = R.G[r];
    P.scale[r] = R.scale[r];
  }
  P.omf = R.omf;
  P.q_begin = R.q_begin;
  {
    const long long lim = g_oz_wait_cycles.load();
    P.wait_cycles = lim > 0 ? lim : OZ_WAIT_CYCLES;
    P.stall_test = g_oz_stall_test.exchange(0);
  }
  CUtensorMap ta, tb;
  if (!make_map(&ta, R.a_slices, (long long)batch * s * M, Kpad, OZ_BM))
    return oz_fail("tensor map of the A slices", cudaSuccess);
  if (!make_map(&tb, R.b_slices, (long long)batch * s * 2 * N, Kpad, pairs ? P.n_tile / 2 : P.n_tile))
    return oz_fail("tensor map of the B slices", cudaSuccess);
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e;
  if (pairs) {
    const size_t smem = (size_t)OZ2_STAGES * (OZ_BM * OZ_BK + (size_t)(P.n_tile / 2) * OZ_BK) + 1024;
    e = cudaFuncSetAttribute(k_oz_gemm2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return oz_fail("k_oz_gemm2 shared memory attribute", e);
    const int grid = 2 * std::max(1, std::min(P.tiles, sms / 2));
    k_oz_gemm2<<<grid, OZ_THREADS2, smem, stream>>>(ta, tb, P);
    if (launches) (*launches)++;
    e = cudaGetLastError();
    return e == cudaSuccess ? TUPS_OK : oz_fail("k_oz_gemm2 launch", e);
  }
  const size_t smem = oz_smem_bytes(P.n_tile);
  e = cudaFuncSetAttribute(k_oz_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return oz_fail("k_oz_gemm shared memory attribute", e);
  const int grid = std::max(1, std::min(P.tiles, sms));
  k_oz_gemm<<<grid, OZ_THREADS2, smem, stream>>>(ta, tb, P);
  if (launches) (*launches)++;
  e = cudaGetLastError();
  return e == cudaSuccess ? TUPS_OK : oz_fail("k_oz_gemm launch", e);
}

}  // namespace tups

// ---- C-ABI: batched split-precision ZGEMM ---------------------------------------------
extern "C" size_t tups_zgemm_split_workspace(int batch, int M, int N, int K, int slices) {
  if (batch < 1 || M < 1 || N < 1 || K < 1 || slices < 1 || slices > 8) return 0;
  return tups::oz_work_layout(batch, M, N, K, slices).total + 256;
}

extern "C" int tups_zgemm_split(int batch, int M, int N, int K, const double* A, const double* B, double* C,
                                int slices, void* work, size_t work_bytes, void* stream) {
  using namespace tups;
  if (batch < 1 || M < 1 || N < 1 || K < 1 || !A || !B || !C || !work) return TUPS_ERR_BADARG;
  if (slices < 1 || slices > 8) return TUPS_ERR_BADARG;
  const OzWork w = oz_work_layout(batch, M, N, K, slices);
  if (work_bytes < w.total + 256) return TUPS_ERR_BADARG;
  cudaStream_t st = (cudaStream_t)stream;
  OzRun R;
  R.batch = batch;
  R.M = M;
  R.N = N;
  R.s = slices;
  R.A.p1 = (const cplx*)A;
  R.A.s1 = (long long)M * K;
  R.A.ld1 = M;
  R.A.K1 = K;
  R.B.p1 = (const cplx*)B;
  R.B.s1 = (long long)K * N;
  R.B.ld1 = K;
  R.B.K1 = K;
  oz_bind_work(R, w, work);
  // the status slot sits after the carved buffers
  double* status = (double*)((uint8_t*)work + w.total);
  status = (double*)(((uintptr_t)status + 7) & ~(uintptr_t)7);
  if ((uint8_t*)(status + 1) > (uint8_t*)work + work_bytes) return TUPS_ERR_BADARG;
  if (cudaMemsetAsync(status, 0, sizeof(double), st) != cudaSuccess) return TUPS_ERR_CUDA;
  R.status = status;
  R.status_code = 1.0;
  R.epi = 0;
  R.C = (cplx*)C;
  int rc = oz_run(R, st, nullptr);
  if (rc) return rc;
  double flag = 0.0;
  cudaError_t e = cudaMemcpyAsync(&flag, status, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return oz_fail("split ZGEMM completion", e);
  return flag != 0.0 ? TUPS_ERR_TIMEOUT : TUPS_OK;
}

// Failure detection of the split GEMM's bounded device waits.  cycles > 0
// sets how many SM cycles a wait of the work loop may take (0 restores the
// default, about 2 s); stall_test = 1 makes the next split GEMM launch wait
// first on a barrier that nothing signals, so its bounded wait runs out: the
// kernel then drains its copies in flight, frees its tensor memory, returns,
// and the call reports TUPS_ERR_TIMEOUT; the launch after it runs normally.
extern "C" int tups_set_split_wait(long long cycles, int stall_test) {
  if (cycles < 0) return TUPS_ERR_BADARG;
  tups::g_oz_wait_cycles.store(cycles);
  tups::g_oz_stall_test.store(stall_test ? 1 : 0);
  return TUPS_OK;
}

extern "C" int tups_set_split_tile(int n_tile) {
  if (n_tile < 0 || n_tile > tups::OZ_MAX_NT || n_tile % 16) return TUPS_ERR_BADARG;
  tups::g_oz_n_tile.store(n_tile);
  return TUPS_OK;
}

// The split GEMM on CTA pairs (tcgen05 cta_group::2, M = 256 over two SMs)
// for row counts >= 256: 1 enables, 0 restores one CTA per 128-row tile.
// Both forms give the same bits.  Process-wide; no counterpart in the
// reference.
extern "C" int tups_set_split_cta_pairs(int enable) {
  tups::g_oz_pairs.store(enable ? 1 : 0);
  return TUPS_OK;
}
