// Batched BSE update that allocates no device memory.
//
// The regular BSE path (bse.cu) keeps its Gamma*chi / chi*Gamma scratch in a
// buffer that tups_ctx_create obtains with cudaMalloc.  Some callers cannot
// allocate device memory when they call into this library: a Fortran/MPI
// host that hands the whole device memory to its own arena at start-up, or
// an embedding whose driver loop must not trigger the implicit device-wide
// synchronisation and possible failure of cudaMalloc/cudaFree.  This entry
// point takes only caller-owned inputs and outputs and keeps its scratch in
// a fixed-size array in the library's own static device memory.
//
// The scratch is a file-scope __device__ array of kScratchComplex complex128
// (32 MiB), present on every GPU that loads the library until the process
// exits.  Host code cannot use the array's name as a device address; the
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call made on the device, so that first call
// should come before any stream capture.  The address is kept for the life
// of the process: after a cudaDeviceReset the device's module, and with it
// the array, is loaded anew, so a process that resets a device must not call
// this entry point on that device again.  All calls share the array and it
// keeps the last call's contents; every element a call reads is written by
// that call first.  Calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on the array.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "tups_device.cuh"

namespace {

using tups::cplx;

constexpr size_t kScratchComplex = (size_t)2 << 20;  // 2 Mi complex128 = 32 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double2 g_bse_scratch[kScratchComplex];

std::mutex g_mu;
cplx* g_scratch_ptr[kMaxDevices] = {};

// device address of g_bse_scratch on the current device, looked up once
int scratch_address(int dev, cplx** out) {
  if (dev < 0 || dev >= kMaxDevices) return TUPS_ERR_BADARG;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_bse_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return TUPS_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<cplx*>(p);
  }
  *out = g_scratch_ptr[dev];
  return TUPS_OK;
}

// A = Gamma chi, B = chi Gamma for instances [i0, i0+n) into the scratch
__global__ void k_noalloc_prep(const cplx* __restrict__ G, const cplx* __restrict__ chi, cplx* __restrict__ A,
                               cplx* __restrict__ B, int i0, int Nz, int Nf, int Nl) {
  const int li = blockIdx.y;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* Gm = G + n2 * (i0 + li);
  const cplx* ch = chi + (size_t)Nl * Nl * Nf * (i0 + li);
  cplx* Ai = A + n2 * li;
  cplx* Bi = B + n2 * li;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (size_t)gridDim.x * blockDim.x) {
    const int row = (int)(e % Nz), col = (int)(e / Nz);
    const int l2 = col / Nf, nu = col % Nf;
    cplx acc = tups::cmk(0.0, 0.0);
    for (int l1 = 0; l1 < Nl; l1++)
      acc = tups::cfma(Gm[row + (size_t)Nz * (l1 * Nf + nu)], ch[l1 + Nl * (l2 + (size_t)Nl * nu)], acc);
    Ai[e] = acc;
    const int r1 = row / Nf, rnu = row % Nf;
    cplx acb = tups::cmk(0.0, 0.0);
    for (int l = 0; l < Nl; l++)
      acb = tups::cfma(ch[r1 + Nl * (l + (size_t)Nl * rnu)], Gm[(l * Nf + rnu) + (size_t)Nz * col], acb);
    Bi[e] = acb;
  }
}

__device__ __forceinline__ void na_cp_async16(void* sdst, const void* gsrc, bool valid) {
  unsigned sz = valid ? 16u : 0u;
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(sz));
}

__device__ __forceinline__ void na_dmma(double* c, const double* a, const double* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Phi = s [A | F] [F ; B] + (1-f)(F - Gamma) over Gamma, 32x32 complex tiles,
// 4 warps of 16x16, two-stage cp.async pipeline, K step 16
constexpr int NB_BM = 32, NB_BN = 32, NB_BK = 16, NB_LDL = NB_BM + 2, NB_LDR = NB_BK + 4;

__global__ void __launch_bounds__(128) k_noalloc_gemm(cplx* __restrict__ G, const cplx* __restrict__ F,
                                                      const cplx* __restrict__ A, const cplx* __restrict__ B, int i0,
                                                      int Nz, double s, double one_minus_f) {
  __shared__ __align__(16) cplx sL[2][NB_BK][NB_LDL];
  __shared__ __align__(16) cplx sR[2][NB_BN][NB_LDR];
  const int li = blockIdx.y;
  const size_t n2 = (size_t)Nz * Nz;
  const cplx* Ai = A + n2 * li;
  const cplx* Bi = B + n2 * li;
  const cplx* Fi = F + n2 * (i0 + li);
  cplx* Gi = G + n2 * (i0 + li);
  const int tiles_m = (Nz + NB_BM - 1) / NB_BM;
  const int m0 = (blockIdx.x % tiles_m) * NB_BM, n0 = (blockIdx.x / tiles_m) * NB_BN;
  const int K = 2 * Nz, ktiles = (K + NB_BK - 1) / NB_BK;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm0 = (warp % 2) * 16, wn0 = (warp / 2) * 16;
  const int gid = lane >> 2, tig = lane & 3;
  auto load = [&](int st, int kt) {
    const int k0 = kt * NB_BK;
    for (int e = tid; e < NB_BK * NB_BM; e += 128) {
      const int m = e % NB_BM, kk = e / NB_BM, gm = m0 + m, gk = k0 + kk;
      const bool ok = gm < Nz && gk < K;
      const cplx* src = Ai;
      if (ok) src = gk < Nz ? Ai + gm + (size_t)Nz * gk : Fi + gm + (size_t)Nz * (gk - Nz);
      na_cp_async16(&sL[st][kk][m], src, ok);
    }
    for (int e = tid; e < NB_BK * NB_BN; e += 128) {
      const int kk = e % NB_BK, n = e / NB_BK, gn = n0 + n, gk = k0 + kk;
      const bool ok = gn < Nz && gk < K;
      const cplx* src = Fi;
      if (ok) src = gk < Nz ? Fi + gk + (size_t)Nz * gn : Bi + (gk - Nz) + (size_t)Nz * gn;
      na_cp_async16(&sR[st][n][kk], src, ok);
    }
    asm volatile("cp.async.commit_group;\n" ::);
  };
  double cre[2][4] = {}, cim[2][4] = {};
  load(0, 0);
  for (int kt = 0; kt < ktiles; kt++) {
    const int cur = kt & 1;
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncthreads();
    if (kt + 1 < ktiles) load(cur ^ 1, kt + 1);
#pragma unroll
    for (int k8 = 0; k8 < NB_BK; k8 += 8) {
      const int mb = wm0 + gid;
      const cplx v0 = sL[cur][k8 + tig][mb], v1 = sL[cur][k8 + tig][mb + 8];
      const cplx v2 = sL[cur][k8 + tig + 4][mb], v3 = sL[cur][k8 + tig + 4][mb + 8];
      const double are[4] = {v0.x, v1.x, v2.x, v3.x}, aim[4] = {v0.y, v1.y, v2.y, v3.y};
      const double anim[4] = {-v0.y, -v1.y, -v2.y, -v3.y};
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int nb = wn0 + j * 8 + gid;
        const cplx w0 = sR[cur][nb][k8 + tig], w1 = sR[cur][nb][k8 + tig + 4];
        const double bre[2] = {w0.x, w1.x}, bim[2] = {w0.y, w1.y};
        na_dmma(cre[j], are, bre);
        na_dmma(cre[j], anim, bim);
        na_dmma(cim[j], are, bim);
        na_dmma(cim[j], aim, bre);
      }
    }
  }
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int row = m0 + wm0 + gid + (x >= 2 ? 8 : 0), col = n0 + wn0 + j * 8 + 2 * tig + (x & 1);
      if (row < Nz && col < Nz) {
        const size_t idx = row + (size_t)Nz * col;
        const cplx f = Fi[idx], g = Gi[idx];
        Gi[idx] = tups::cmk(s * cre[j][x] + one_minus_f * (f.x - g.x), s * cim[j][x] + one_minus_f * (f.y - g.y));
      }
    }
}

}  // namespace

extern "C" int tups_bse_noalloc(int n_inst, int Nz, int Nf, int Nl, double* gamma_phi, const double* F,
                                const double* chi, double scale, double f_damping, void* stream) {
  if (n_inst < 1 || Nf < 1 || Nl < 1 || Nz != Nl * Nf || !gamma_phi || !F || !chi) return TUPS_ERR_BADARG;
  const size_t per = 2 * (size_t)Nz * Nz;
  if (per > kScratchComplex) {
    std::fprintf(stderr,
                 "tups_bse_noalloc: Nz = %d needs %zu bytes of scratch per instance; the static scratch holds %zu "
                 "bytes (Nz <= 1024)\n",
                 Nz, per * sizeof(cplx), kScratchComplex * sizeof(cplx));
    return TUPS_ERR_BADDIM;
  }
  // an error left by an earlier, unrelated call would otherwise be reported
  // as this call's launch failure
  (void)cudaGetLastError();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return TUPS_ERR_CUDA;
  }
  cplx* scratch = nullptr;
  int rc = scratch_address(dev, &scratch);
  if (rc != TUPS_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // instances per pass through the scratch; the instance index is gridDim.y
  // of both kernels, at most 65535
  const int chunk = (int)std::min<size_t>(kScratchComplex / per, 65535);
  cplx* A = scratch;
  cplx* B = scratch + (size_t)chunk * Nz * Nz;
  const size_t n2 = (size_t)Nz * Nz;
  const int tiles = ((Nz + NB_BM - 1) / NB_BM) * ((Nz + NB_BN - 1) / NB_BN);
  for (int i0 = 0; i0 < n_inst; i0 += chunk) {
    const int n = n_inst - i0 < chunk ? n_inst - i0 : chunk;
    dim3 pg((unsigned)(n2 < 256 * 1024 ? (n2 + 255) / 256 : 1024), n);
    k_noalloc_prep<<<pg, 256, 0, st>>>(reinterpret_cast<const cplx*>(gamma_phi), reinterpret_cast<const cplx*>(chi), A,
                                       B, i0, Nz, Nf, Nl);
    if (cudaGetLastError() != cudaSuccess) return TUPS_ERR_CUDA;
    k_noalloc_gemm<<<dim3(tiles, n), 128, 0, st>>>(reinterpret_cast<cplx*>(gamma_phi), reinterpret_cast<const cplx*>(F),
                                                   A, B, i0, Nz, scale, 1.0 - f_damping);
    if (cudaGetLastError() != cudaSuccess) return TUPS_ERR_CUDA;
  }
  return TUPS_OK;
}
