// Multilayer perceptron of the learned warm start: forward, backward and Adam
// in FP32 on the device.  No counterpart in the reference.
//
// Network: n_in -> H -> ... -> H (n_layers hidden layers, SiLU) -> n_out
// (linear).  Layer l holds W_l (out_l, in_l) row-major and b_l (out_l); the
// flat parameter vector is [W_0, b_0, W_1, b_1, ...].  Loss: mean squared
// error over batch x n_out.  Batches are row-major (batch, features).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/tups_b200.h"

struct tups_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  long long launches = 0;
  int n_in = 0, n_hidden = 0, n_layers = 0, n_out = 0, max_batch = 0;
  std::vector<int> width;      // n_layers + 2 entries: n_in, H, ..., H, n_out
  std::vector<size_t> w_off;   // offset of W_l in the flat vector
  std::vector<size_t> b_off;   // offset of b_l
  size_t n_params = 0;
  float* params = nullptr;
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  long long adam_t = 0;
  float* x = nullptr;          // input batch (max_batch, n_in)
  float* t = nullptr;          // target batch (max_batch, n_out)
  std::vector<float*> z, a;    // per hidden layer: pre-activation, activation
  float* y = nullptr;          // output (max_batch, n_out)
  float* dz[2] = {};           // backward ping-pong (max_batch, max width)
  double* loss = nullptr;      // device loss slots
  int loss_slots = 0;
  float* data_x = nullptr;     // resident training set
  float* data_t = nullptr;
  int data_n = 0;
  int* idx = nullptr;          // minibatch row indices
  std::vector<void*> allocs;
};

namespace {

int mlp_error(tups_mlp* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  return code;
}

int mlp_cuda(tups_mlp* m, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TUPS_OK;
  return mlp_error(m, e == cudaErrorMemoryAllocation ? TUPS_ERR_OOM : TUPS_ERR_CUDA,
                   std::string(what) + ": " + cudaGetErrorString(e));
}

#define MTRY(x)                     \
  do {                              \
    int _rc = (x);                  \
    if (_rc != TUPS_OK) return _rc; \
  } while (0)

int launched(tups_mlp* m, const char* name) {
  m->launches++;
  return mlp_cuda(m, cudaGetLastError(), name);
}

template <typename T>
int mlp_alloc(tups_mlp* m, T** p, size_t count) {
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T) + 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return mlp_error(m, TUPS_ERR_OOM, "MLP device allocation failed");
  }
  m->allocs.push_back(*p);
  return TUPS_OK;
}

__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

// Epilogues of the tiled GEMM
enum { EPI_STORE = 0, EPI_BIAS_SILU = 1, EPI_BIAS = 2, EPI_DSILU = 3 };

// C(m, n) = sum_k A(m, k) B(k, n) with A(m, k) = A[m*sam + k*sak] and
// B(k, n) = B[k*sbk + n*sbn]; 64 x 64 tile per CTA, 4 x 4 per thread.
//   EPI_STORE:     C = acc
//   EPI_BIAS_SILU: C = acc + bias[n] (pre-activation), C2 = silu(C)
//   EPI_BIAS:      C = acc + bias[n]
//   EPI_DSILU:     C = acc * silu'(aux[m, n])
template <int EPI>
__global__ void __launch_bounds__(256) k_mlp_gemm(int M, int N, int K, const float* __restrict__ A, int sam, int sak,
                                                  const float* __restrict__ B, int sbk, int sbn,
                                                  const float* __restrict__ bias, const float* __restrict__ aux,
                                                  float* __restrict__ C, float* __restrict__ C2) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ float As[BK][BM + 4];
  __shared__ float Bs[BK][BN + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
  const bool a_kfast = sak == 1, b_kfast = sbk == 1;
  for (int k0 = 0; k0 < K; k0 += BK) {
    for (int e = threadIdx.x; e < BK * BM; e += 256) {
      const int kk = a_kfast ? e % BK : e / BM;
      const int mm = a_kfast ? e / BK : e % BM;
      const int gm = m0 + mm, gk = k0 + kk;
      As[kk][mm] = (gm < M && gk < K) ? A[(size_t)gm * sam + (size_t)gk * sak] : 0.0f;
      const int kb = b_kfast ? e % BK : e / BN;
      const int nn = b_kfast ? e / BK : e % BN;
      const int gn = n0 + nn, gkb = k0 + kb;
      Bs[kb][nn] = (gn < N && gkb < K) ? B[(size_t)gkb * sbk + (size_t)gn * sbn] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk++) {
      float av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; i++) av[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) bv[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int m = m0 + ty + 16 * i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int n = n0 + tx + 16 * j;
      if (n >= N) continue;
      const size_t o = (size_t)m * N + n;
      float v = acc[i][j];
      if (EPI == EPI_BIAS_SILU) {
        v += bias[n];
        C[o] = v;
        C2[o] = v * sigmoid(v);
      } else if (EPI == EPI_BIAS) {
        C[o] = v + bias[n];
      } else if (EPI == EPI_DSILU) {
        const float z = aux[o];
        const float s = sigmoid(z);
        C[o] = v * (s * (1.0f + z * (1.0f - s)));
      } else {
        C[o] = v;
      }
    }
  }
}

// db[n] = sum_m dz[m, n]
__global__ void k_mlp_colsum(const float* __restrict__ dz, float* __restrict__ db, int M, int N) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = 0; m < M; m++) s += dz[(size_t)m * N + n];
  db[n] = s;
}

// dy = 2 (y - t) / (M N); loss[slot] += sum (y - t)^2 / (M N)
__global__ void k_mlp_mse(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                          size_t n, double inv, double* loss) {
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = (float)(2.0 * inv) * d;
    s += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double sh[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += sh[w];
    atomicAdd(loss, tot * inv);
  }
}

// Adam (Kingma & Ba 2015) with bias-corrected step size lr_t
__global__ void k_mlp_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                           float* __restrict__ v, size_t n, float lr_t, float b1, float b2, float eps_t) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr_t * mi / (sqrtf(vi) + eps_t);
  }
}

__global__ void k_mlp_scale(float* __restrict__ p, size_t n, float f) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] *= f;
}

// rows of a resident set: out[i, :] = src[idx[i], :]
__global__ void k_mlp_gather(const float* __restrict__ src, const int* __restrict__ idx, float* __restrict__ out,
                             int rows, int cols) {
  const size_t n = (size_t)rows * cols;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int r = (int)(e / cols), c = (int)(e % cols);
    out[e] = src[(size_t)idx[r] * cols + c];
  }
}

unsigned grid1d(size_t n, int threads) {
  const size_t b = (n + threads - 1) / threads;
  return (unsigned)std::min<size_t>(std::max<size_t>(b, 1), 148 * 8);
}

template <int EPI>
int gemm(tups_mlp* m, int M, int N, int K, const float* A, int sam, int sak, const float* B, int sbk, int sbn,
         const float* bias, const float* aux, float* C, float* C2) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  k_mlp_gemm<EPI><<<grid, 256, 0, m->stream>>>(M, N, K, A, sam, sak, B, sbk, sbn, bias, aux, C, C2);
  return launched(m, "k_mlp_gemm");
}

int n_linear(const tups_mlp* m) { return m->n_layers + 1; }

// forward of the batch in m->x (batch rows) into m->y
int forward(tups_mlp* m, int batch) {
  const float* in = m->x;
  for (int l = 0; l < n_linear(m); l++) {
    const int fin = m->width[l], fout = m->width[l + 1];
    const float* W = m->params + m->w_off[l];
    const float* b = m->params + m->b_off[l];
    // Z = in W^T + b: A(m, k) = in[m*fin + k], B(k, n) = W[n*fin + k]
    if (l < m->n_layers) {
      MTRY(gemm<EPI_BIAS_SILU>(m, batch, fout, fin, in, fin, 1, W, 1, fin, b, nullptr, m->z[l], m->a[l]));
      in = m->a[l];
    } else {
      MTRY(gemm<EPI_BIAS>(m, batch, fout, fin, in, fin, 1, W, 1, fin, b, nullptr, m->y, nullptr));
    }
  }
  return TUPS_OK;
}

// loss into m->loss[slot] and gradients of the batch in m->x / m->t into m->grads
int backward(tups_mlp* m, int batch, int slot) {
  const size_t ny = (size_t)batch * m->n_out;
  float* dcur = m->dz[0];
  k_mlp_mse<<<grid1d(ny, 256), 256, 0, m->stream>>>(m->y, m->t, dcur, ny, 1.0 / (double)ny, m->loss + slot);
  MTRY(launched(m, "k_mlp_mse"));
  for (int l = n_linear(m) - 1; l >= 0; l--) {
    const int fin = m->width[l], fout = m->width[l + 1];
    const float* in = l == 0 ? m->x : m->a[l - 1];
    // dW(o, i) = sum_b dZ[b, o] in[b, i]: A(m=o, k=b) = dZ[b*fout + o], B(k=b, n=i) = in[b*fin + i]
    MTRY(gemm<EPI_STORE>(m, fout, fin, batch, dcur, 1, fout, in, fin, 1, nullptr, nullptr, m->grads + m->w_off[l],
                         nullptr));
    k_mlp_colsum<<<(fout + 127) / 128, 128, 0, m->stream>>>(dcur, m->grads + m->b_off[l], batch, fout);
    MTRY(launched(m, "k_mlp_colsum"));
    if (l > 0) {
      // dZ_{l-1}(b, i) = sum_o dZ[b, o] W[o, i] * silu'(Z_{l-1}(b, i))
      float* dnext = dcur == m->dz[0] ? m->dz[1] : m->dz[0];
      const float* W = m->params + m->w_off[l];
      MTRY(gemm<EPI_DSILU>(m, batch, fin, fout, dcur, fout, 1, W, fin, 1, nullptr, m->z[l - 1], dnext, nullptr));
      dcur = dnext;
    }
  }
  return TUPS_OK;
}

int adam_step(tups_mlp* m, float lr, float b1, float b2, float eps) {
  m->adam_t++;
  const double bc1 = 1.0 - std::pow((double)b1, (double)m->adam_t);
  const double bc2 = 1.0 - std::pow((double)b2, (double)m->adam_t);
  // step with bias correction folded into the step size and epsilon
  const float lr_t = (float)(lr * std::sqrt(bc2) / bc1);
  const float eps_t = (float)(eps * std::sqrt(bc2));
  k_mlp_adam<<<grid1d(m->n_params, 256), 256, 0, m->stream>>>(m->params, m->grads, m->adam_m, m->adam_v,
                                                               m->n_params, lr_t, b1, b2, eps_t);
  return launched(m, "k_mlp_adam");
}

int h2d(tups_mlp* m, void* dst, const void* src, size_t bytes) {
  if (!src) return mlp_error(m, TUPS_ERR_BADARG, "NULL host buffer");
  return mlp_cuda(m, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, m->stream), "H2D");
}

int d2h(tups_mlp* m, void* dst, const void* src, size_t bytes) {
  if (!dst) return mlp_error(m, TUPS_ERR_BADARG, "NULL host buffer");
  MTRY(mlp_cuda(m, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, m->stream), "D2H"));
  return mlp_cuda(m, cudaStreamSynchronize(m->stream), "synchronize");
}

int set_dev(tups_mlp* m) { return mlp_cuda(m, cudaSetDevice(m->device), "cudaSetDevice"); }

int check_batch(tups_mlp* m, int batch) {
  if (batch < 1 || batch > m->max_batch) return mlp_error(m, TUPS_ERR_BADDIM, "batch outside 1..max_batch");
  return TUPS_OK;
}

// splitmix64 for the minibatch shuffles
uint64_t mix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

void free_mlp(tups_mlp* m) {
  for (void* p : m->allocs) cudaFree(p);
  m->allocs.clear();
  if (m->stream) cudaStreamDestroy(m->stream);
  m->stream = nullptr;
}

}  // namespace

extern "C" int tups_mlp_create(int n_in, int n_hidden, int n_layers, int n_out, int max_batch, int device,
                               tups_mlp** out) {
  if (!out) return TUPS_ERR_BADARG;
  *out = nullptr;
  if (n_in < 1 || n_hidden < 1 || n_layers < 1 || n_out < 1 || max_batch < 1 || n_layers > 16)
    return TUPS_ERR_BADDIM;
  tups_mlp* m = new tups_mlp();
  m->device = device;
  m->n_in = n_in;
  m->n_hidden = n_hidden;
  m->n_layers = n_layers;
  m->n_out = n_out;
  m->max_batch = max_batch;
  m->width.push_back(n_in);
  for (int l = 0; l < n_layers; l++) m->width.push_back(n_hidden);
  m->width.push_back(n_out);
  size_t off = 0;
  for (int l = 0; l <= n_layers; l++) {
    m->w_off.push_back(off);
    off += (size_t)m->width[l] * m->width[l + 1];
    m->b_off.push_back(off);
    off += (size_t)m->width[l + 1];
  }
  m->n_params = off;
  int rc = set_dev(m);
  if (!rc) rc = mlp_cuda(m, cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "stream");
  const int wmax = std::max(std::max(n_in, n_hidden), n_out);
  if (!rc) rc = mlp_alloc(m, &m->params, m->n_params);
  if (!rc) rc = mlp_alloc(m, &m->grads, m->n_params);
  if (!rc) rc = mlp_alloc(m, &m->adam_m, m->n_params);
  if (!rc) rc = mlp_alloc(m, &m->adam_v, m->n_params);
  if (!rc) rc = mlp_alloc(m, &m->x, (size_t)max_batch * n_in);
  if (!rc) rc = mlp_alloc(m, &m->t, (size_t)max_batch * n_out);
  if (!rc) rc = mlp_alloc(m, &m->y, (size_t)max_batch * n_out);
  m->z.assign(n_layers, nullptr);
  m->a.assign(n_layers, nullptr);
  for (int l = 0; l < n_layers && !rc; l++) {
    rc = mlp_alloc(m, &m->z[l], (size_t)max_batch * n_hidden);
    if (!rc) rc = mlp_alloc(m, &m->a[l], (size_t)max_batch * n_hidden);
  }
  if (!rc) rc = mlp_alloc(m, &m->dz[0], (size_t)max_batch * wmax);
  if (!rc) rc = mlp_alloc(m, &m->dz[1], (size_t)max_batch * wmax);
  if (!rc) rc = mlp_cuda(m, cudaMemsetAsync(m->params, 0, m->n_params * sizeof(float), m->stream), "memset");
  if (!rc) rc = mlp_cuda(m, cudaMemsetAsync(m->adam_m, 0, m->n_params * sizeof(float), m->stream), "memset");
  if (!rc) rc = mlp_cuda(m, cudaMemsetAsync(m->adam_v, 0, m->n_params * sizeof(float), m->stream), "memset");
  if (!rc) rc = mlp_cuda(m, cudaStreamSynchronize(m->stream), "synchronize");
  if (rc) {
    free_mlp(m);
    delete m;
    return rc;
  }
  *out = m;
  return TUPS_OK;
}

extern "C" int tups_mlp_destroy(tups_mlp* m) {
  if (!m) return TUPS_OK;
  cudaSetDevice(m->device);
  free_mlp(m);
  delete m;
  return TUPS_OK;
}

extern "C" const char* tups_mlp_last_error(const tups_mlp* m) { return m ? m->err.c_str() : "NULL MLP"; }

extern "C" long long tups_mlp_num_params(const tups_mlp* m) { return m ? (long long)m->n_params : -1; }

extern "C" long long tups_mlp_kernel_launches(const tups_mlp* m) { return m ? m->launches : -1; }

extern "C" int tups_mlp_set_params(tups_mlp* m, const float* host) {
  if (!m) return TUPS_ERR_BADARG;
  MTRY(set_dev(m));
  MTRY(h2d(m, m->params, host, m->n_params * sizeof(float)));
  // a new parameter set restarts the optimiser
  MTRY(mlp_cuda(m, cudaMemsetAsync(m->adam_m, 0, m->n_params * sizeof(float), m->stream), "memset"));
  MTRY(mlp_cuda(m, cudaMemsetAsync(m->adam_v, 0, m->n_params * sizeof(float), m->stream), "memset"));
  m->adam_t = 0;
  return mlp_cuda(m, cudaStreamSynchronize(m->stream), "synchronize");
}

extern "C" int tups_mlp_get_params(tups_mlp* m, float* host) {
  if (!m) return TUPS_ERR_BADARG;
  MTRY(set_dev(m));
  return d2h(m, host, m->params, m->n_params * sizeof(float));
}

extern "C" int tups_mlp_forward(tups_mlp* m, const float* x, int batch, float* y) {
  if (!m) return TUPS_ERR_BADARG;
  MTRY(set_dev(m));
  MTRY(check_batch(m, batch));
  MTRY(h2d(m, m->x, x, (size_t)batch * m->n_in * sizeof(float)));
  MTRY(forward(m, batch));
  return d2h(m, y, m->y, (size_t)batch * m->n_out * sizeof(float));
}

extern "C" int tups_mlp_gradients(tups_mlp* m, const float* x, const float* t, int batch, float* grad,
                                  double* loss) {
  if (!m) return TUPS_ERR_BADARG;
  MTRY(set_dev(m));
  MTRY(check_batch(m, batch));
  if (m->loss_slots < 1) {
    MTRY(mlp_alloc(m, &m->loss, 1));
    m->loss_slots = 1;
  }
  MTRY(h2d(m, m->x, x, (size_t)batch * m->n_in * sizeof(float)));
  MTRY(h2d(m, m->t, t, (size_t)batch * m->n_out * sizeof(float)));
  MTRY(mlp_cuda(m, cudaMemsetAsync(m->loss, 0, sizeof(double), m->stream), "memset"));
  MTRY(forward(m, batch));
  MTRY(backward(m, batch, 0));
  if (loss) MTRY(d2h(m, loss, m->loss, sizeof(double)));
  if (grad) MTRY(d2h(m, grad, m->grads, m->n_params * sizeof(float)));
  return mlp_cuda(m, cudaStreamSynchronize(m->stream), "synchronize");
}

extern "C" int tups_mlp_train(tups_mlp* m, const float* x, const float* t, int n_samples, int batch, int epochs,
                              float lr, float weight_decay, unsigned long long seed, double* loss_per_epoch) {
  if (!m) return TUPS_ERR_BADARG;
  if (n_samples < 1 || epochs < 0 || lr <= 0.0f || weight_decay < 0.0f)
    return mlp_error(m, TUPS_ERR_BADARG, "bad training arguments");
  MTRY(set_dev(m));
  batch = std::min(batch, n_samples);
  MTRY(check_batch(m, batch));
  if (n_samples > m->data_n) {
    MTRY(mlp_alloc(m, &m->data_x, (size_t)n_samples * m->n_in));
    MTRY(mlp_alloc(m, &m->data_t, (size_t)n_samples * m->n_out));
    MTRY(mlp_alloc(m, &m->idx, (size_t)n_samples));
    m->data_n = n_samples;
  }
  if (m->loss_slots < epochs) {
    MTRY(mlp_alloc(m, &m->loss, (size_t)epochs));
    m->loss_slots = epochs;
  }
  MTRY(h2d(m, m->data_x, x, (size_t)n_samples * m->n_in * sizeof(float)));
  MTRY(h2d(m, m->data_t, t, (size_t)n_samples * m->n_out * sizeof(float)));
  if (epochs > 0) MTRY(mlp_cuda(m, cudaMemsetAsync(m->loss, 0, (size_t)epochs * sizeof(double), m->stream), "memset"));
  const int per_epoch = (n_samples + batch - 1) / batch;
  std::vector<int> perm(n_samples);
  std::vector<int> all_idx((size_t)epochs * n_samples);
  uint64_t s = seed;
  for (int e = 0; e < epochs; e++) {
    for (int i = 0; i < n_samples; i++) perm[i] = i;
    for (int i = n_samples - 1; i > 0; i--) std::swap(perm[i], perm[(int)(mix64(s) % (uint64_t)(i + 1))]);
    std::memcpy(all_idx.data() + (size_t)e * n_samples, perm.data(), n_samples * sizeof(int));
  }
  for (int e = 0; e < epochs; e++) {
    // index upload per epoch: the host vector stays alive for the whole call
    MTRY(h2d(m, m->idx, all_idx.data() + (size_t)e * n_samples, n_samples * sizeof(int)));
    for (int b = 0; b < per_epoch; b++) {
      const int r0 = b * batch, rows = std::min(batch, n_samples - r0);
      k_mlp_gather<<<grid1d((size_t)rows * m->n_in, 256), 256, 0, m->stream>>>(m->data_x, m->idx + r0, m->x, rows,
                                                                              m->n_in);
      MTRY(launched(m, "k_mlp_gather"));
      k_mlp_gather<<<grid1d((size_t)rows * m->n_out, 256), 256, 0, m->stream>>>(m->data_t, m->idx + r0, m->t, rows,
                                                                               m->n_out);
      MTRY(launched(m, "k_mlp_gather"));
      MTRY(forward(m, rows));
      MTRY(backward(m, rows, e));
      if (weight_decay > 0.0f) {
        // decoupled weight decay (Loshchilov & Hutter 2019) on the weights only
        for (int l = 0; l < n_linear(m); l++) {
          const size_t nw = (size_t)m->width[l] * m->width[l + 1];
          k_mlp_scale<<<grid1d(nw, 256), 256, 0, m->stream>>>(m->params + m->w_off[l], nw, 1.0f - lr * weight_decay);
          MTRY(launched(m, "k_mlp_scale"));
        }
      }
      MTRY(adam_step(m, lr, 0.9f, 0.999f, 1e-8f));
    }
  }
  if (loss_per_epoch && epochs > 0) {
    MTRY(d2h(m, loss_per_epoch, m->loss, (size_t)epochs * sizeof(double)));
    for (int e = 0; e < epochs; e++) loss_per_epoch[e] /= per_epoch;
  }
  return mlp_cuda(m, cudaStreamSynchronize(m->stream), "synchronize");
}
