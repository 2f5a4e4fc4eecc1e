// Device pieces shared by the batched LU kernels (lu.cu, lu_split.cu):
// complex 1-norm for pivoting and the rank-K (K <= 32) update on the FP64
// tensor cores.
#pragma once

#include "tups_device.cuh"

namespace tups {
namespace lud {

constexpr int kRankMaxK = 32;

static __device__ __forceinline__ double cabs1(cplx a) { return fabs(a.x) + fabs(a.y); }

static __device__ __forceinline__ void dmma8(double* c, const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// C[m x p] -= A[m x K] B[K x p], K <= 32, column-major with leading dim ld
// (all three inside the same n x n matrix or RHS block).  Warp tiles of
// 16 x 32 on the FP64 tensor cores, fragments straight from global memory.
static __device__ void rank_update(cplx* C, const cplx* A, const cplx* B, int m, int p, int K, int ldc, int lda,
                                   int ldb) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  const int tm = (m + 15) / 16, tp = (p + 31) / 32;
  for (int t = warp; t < tm * tp; t += nwarps) {
    const int r0 = (t % tm) * 16, c0 = (t / tm) * 32;
    double cre[4][4], cim[4][4];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int r = r0 + gid + (x >= 2 ? 8 : 0), c = c0 + j * 8 + 2 * tig + (x & 1);
        cplx v = (r < m && c < p) ? C[r + (size_t)ldc * c] : cmk(0.0, 0.0);
        cre[j][x] = v.x;
        cim[j][x] = v.y;
      }
#pragma unroll
    for (int k8 = 0; k8 < kRankMaxK; k8 += 8) {
      if (k8 >= K) break;
      double are[4], aim[4], apos[4];
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int r = r0 + gid + (x & 1 ? 8 : 0), k = k8 + tig + (x >= 2 ? 4 : 0);
        cplx v = (r < m && k < K) ? A[r + (size_t)lda * k] : cmk(0.0, 0.0);
        // C -= A B  ==  C += (-A) B
        are[x] = -v.x;
        aim[x] = -v.y;
        apos[x] = v.y;
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = c0 + j * 8 + gid;
        const int k0 = k8 + tig, k1 = k8 + tig + 4;
        cplx w0 = (c < p && k0 < K) ? B[k0 + (size_t)ldb * c] : cmk(0.0, 0.0);
        cplx w1 = (c < p && k1 < K) ? B[k1 + (size_t)ldb * c] : cmk(0.0, 0.0);
        const double bre[2] = {w0.x, w1.x}, bim[2] = {w0.y, w1.y};
        dmma8(cre[j], are, bre);   // -Are Bre
        dmma8(cre[j], apos, bim);  // +Aim Bim
        dmma8(cim[j], are, bim);   // -Are Bim
        dmma8(cim[j], aim, bre);   // -Aim Bre
      }
    }
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int r = r0 + gid + (x >= 2 ? 8 : 0), c = c0 + j * 8 + 2 * tig + (x & 1);
        if (r < m && c < p) C[r + (size_t)ldc * c] = cmk(cre[j][x], cim[j][x]);
      }
  }
}

}  // namespace lud
}  // namespace tups
