// Device helpers: complex128 arithmetic on double2 and reductions.
#pragma once

#include <cuda_runtime.h>

#include "tups_internal.h"

namespace tups {

__host__ __device__ __forceinline__ cplx cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ cplx cconj(cplx a) { return cmk(a.x, -a.y); }
// acc += a*b
__host__ __device__ __forceinline__ cplx cfma(cplx a, cplx b, cplx acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// 1/z
__host__ __device__ __forceinline__ cplx crecip(cplx z) {
  double d = z.x * z.x + z.y * z.y;
  return cmk(z.x / d, -z.y / d);
}
__host__ __device__ __forceinline__ double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Matsubara frequency get_freq(nu) (SRC/parquet_util.f90:1332-1339), 1-based
// nu, any integer: the imaginary part pi/beta*(2(nu-Nf/2-1)+1)
__host__ __device__ __forceinline__ double matsubara(int nu, int Nf, double beta) {
  return M_PI / beta * (2.0 * (double)(nu - Nf / 2 - 1) + 1.0);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// block-wide sum; all threads get the result; `sh` holds >= 32 doubles
__device__ __forceinline__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  for (int i = 0; i < nw; i++) r += sh[i];
  __syncthreads();
  return r;
}

// atomic max for non-negative doubles (bit pattern order == value order)
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
  unsigned long long nv = __double_as_longlong(v);
  unsigned long long old = *a;
  while (__longlong_as_double(old) < v) {
    unsigned long long assumed = old;
    old = atomicCAS(a, assumed, nv);
    if (old == assumed) break;
  }
}

inline int cdiv(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace tups
