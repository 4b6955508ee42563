// The learned start vector's network: a 3-layer MLP (n_in -> width -> width -> n_out,
// SiLU between layers) with FP32 weights and BF16 hidden activations, trained and
// evaluated on the GPU by the kernels of this file.  It maps the coefficients of an
// interaction variant to the compressed ground state (weights on the dominant
// proton x neutron sub-blocks) that seeds the Lanczos start vector.  The reference
// has no counterpart: its start vector is always the seeded random one
// (src/NuLnz/NuCoreX.f90:625-654).
//
// Parameter layout (one flat FP32 array, also the layout of the gradients and of
// the Adam moments): W1 [width x n_in] row-major, b1 [width], W2 [width x width],
// b2 [width], W3 [n_out x width], b3 [n_out].
//
// Arithmetic: every product accumulates in FP32; the hidden activations a1, a2
// are rounded to BF16 (round to nearest even) when stored, as the forward pass
// keeps them for the backward pass; pre-activations z stay FP32.  Reductions
// (bias gradients, loss) run in a fixed order, so results are deterministic.
#include <cuda_bf16.h>
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>
#include "nsx.h"

namespace {

struct Err {
  int code;
  std::string msg;
};
thread_local std::string g_mlp_err;

void mcheck(cudaError_t e, const char *what) {
  if (e != cudaSuccess)
    throw Err{e == cudaErrorMemoryAllocation ? NSX_E_NOMEM : NSX_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e)};
}
#define MCUDA(x) mcheck((x), #x)

// Makes the network's device current for one entry point and restores the caller's device.
struct MDevice {
  int prev = -1;
  explicit MDevice(int device) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) MCUDA(cudaSetDevice(device));
  }
  ~MDevice() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <typename F>
int mguard(F &&f) {
  try {
    f();
    return NSX_OK;
  } catch (const Err &e) {
    g_mlp_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    g_mlp_err = "host allocation failed";
    return NSX_E_NOMEM;
  } catch (const std::exception &e) {
    g_mlp_err = e.what();
    return NSX_E_ARG;
  }
}

__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }

// C(m, n) = [C(m, n) +] sum_k A(m, k) B(k, n) [+ bias(n)], all strides in elements.
// 32 x 32 output tile per CTA of 256 threads (4 outputs per thread), K staged in
// chunks of 32 through shared memory.
template <typename TA, typename TB>
__global__ void __launch_bounds__(256) k_mlp_gemm(int M, int N, int K, const TA *__restrict__ A, int64_t as_m,
                                                  int64_t as_k, const TB *__restrict__ B, int64_t bs_k, int64_t bs_n,
                                                  float *__restrict__ C, int64_t cs_m, int64_t cs_n,
                                                  const float *__restrict__ bias, int accumulate) {
  __shared__ float As[32][33];
  __shared__ float Bs[32][33];
  const int m0 = blockIdx.y * 32, n0 = blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // ty 0..7: rows ty, ty+8, ty+16, ty+24
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k0 = 0; k0 < K; k0 += 32) {
    for (int e = threadIdx.x; e < 32 * 32; e += 256) {
      const int r = e >> 5, c = e & 31;
      const int m = m0 + r, k = k0 + c;
      As[r][c] = (m < M && k < K) ? to_f(A[(int64_t)m * as_m + (int64_t)k * as_k]) : 0.f;
      const int kk = k0 + r, n = n0 + c;
      Bs[r][c] = (kk < K && n < N) ? to_f(B[(int64_t)kk * bs_k + (int64_t)n * bs_n]) : 0.f;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const float b = Bs[k][tx];
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[i] = fmaf(As[ty + 8 * i][k], b, acc[i]);
    }
    __syncthreads();
  }
  const int n = n0 + tx;
  if (n >= N) return;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty + 8 * i;
    if (m >= M) continue;
    float v = acc[i] + (bias ? bias[n] : 0.f);
    float *c = C + (int64_t)m * cs_m + (int64_t)n * cs_n;
    *c = accumulate ? *c + v : v;
  }
}

__device__ __forceinline__ float sigmoidf_(float z) { return 1.f / (1.f + expf(-z)); }

// a = bf16(silu(z))
__global__ void k_mlp_act(const float *__restrict__ z, __nv_bfloat16 *__restrict__ a, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sigmoidf_(z[i]);
    a[i] = __float2bfloat16_rn(z[i] * s);
  }
}

// dz = da * silu'(z), silu'(z) = s (1 + z (1 - s))
__global__ void k_mlp_dact(const float *__restrict__ da, const float *__restrict__ z, float *__restrict__ dz, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sigmoidf_(z[i]);
    dz[i] = da[i] * s * (1.f + z[i] * (1.f - s));
  }
}

// db[n] = sum_b dz[b, n] (fixed order)
__global__ void k_mlp_colsum(const float *__restrict__ dz, float *__restrict__ db, int B, int N) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int b = 0; b < B; ++b) s += dz[(int64_t)b * N + n];
  db[n] = s;
}

// Mean squared error over B x N and its gradient dy = 2 (y - t) / (B N); one CTA of
// 1024 threads, fixed reduction order.
__global__ void __launch_bounds__(1024) k_mlp_mse(const float *__restrict__ y, const float *__restrict__ t,
                                                  float *__restrict__ dy, float *__restrict__ loss, int64_t n) {
  __shared__ float red[1024];
  float s = 0.f;
  const float g = 2.f / (float)n;
  for (int64_t i = threadIdx.x; i < n; i += 1024) {
    const float d = y[i] - t[i];
    dy[i] = g * d;
    s += d * d;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = red[0] / (float)n;
}

// Adam with bias corrections c1 = 1 / (1 - beta1^t), c2 = 1 / (1 - beta2^t).
__global__ void k_mlp_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                           float *__restrict__ v, int64_t n, float lr, float b1, float b2, float eps, float c1,
                           float c2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

unsigned grid_1d(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8); }

template <typename TA, typename TB>
void gemm(int M, int N, int K, const TA *A, int64_t as_m, int64_t as_k, const TB *B, int64_t bs_k, int64_t bs_n,
          float *C, int64_t cs_m, int64_t cs_n, const float *bias, bool accumulate) {
  if (M <= 0 || N <= 0) return;
  dim3 grid((N + 31) / 32, (M + 31) / 32);
  k_mlp_gemm<TA, TB><<<grid, 256>>>(M, N, K, A, as_m, as_k, B, bs_k, bs_n, C, cs_m, cs_n, bias, accumulate ? 1 : 0);
  MCUDA(cudaGetLastError());
}

}  // namespace

struct nsx_mlp {
  int device = 0;
  int n_in = 0, width = 0, n_out = 0;
  int64_t np = 0;
  int64_t o_w1 = 0, o_b1 = 0, o_w2 = 0, o_b2 = 0, o_w3 = 0, o_b3 = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // params, gradients, Adam moments
  int64_t adam_t = 0;
  // batch workspace
  int cap = 0;
  float *x = nullptr, *t = nullptr, *z1 = nullptr, *z2 = nullptr, *y = nullptr;
  __nv_bfloat16 *a1 = nullptr, *a2 = nullptr;
  float *dy = nullptr, *da = nullptr, *dz = nullptr, *loss = nullptr;

  void free_batch() {
    for (void *q : {(void *)x, (void *)t, (void *)z1, (void *)z2, (void *)y, (void *)a1, (void *)a2, (void *)dy,
                    (void *)da, (void *)dz})
      if (q) cudaFree(q);
    x = t = z1 = z2 = y = dy = da = dz = nullptr;
    a1 = a2 = nullptr;
    cap = 0;
  }
  void ensure_batch(int B) {
    if (B <= cap) return;
    free_batch();
    const int w = width;
    MCUDA(cudaMalloc(&x, sizeof(float) * (size_t)B * n_in));
    MCUDA(cudaMalloc(&t, sizeof(float) * (size_t)B * n_out));
    MCUDA(cudaMalloc(&z1, sizeof(float) * (size_t)B * w));
    MCUDA(cudaMalloc(&z2, sizeof(float) * (size_t)B * w));
    MCUDA(cudaMalloc(&y, sizeof(float) * (size_t)B * n_out));
    MCUDA(cudaMalloc(&a1, sizeof(__nv_bfloat16) * (size_t)B * w));
    MCUDA(cudaMalloc(&a2, sizeof(__nv_bfloat16) * (size_t)B * w));
    MCUDA(cudaMalloc(&dy, sizeof(float) * (size_t)B * n_out));
    MCUDA(cudaMalloc(&da, sizeof(float) * (size_t)B * w));
    MCUDA(cudaMalloc(&dz, sizeof(float) * (size_t)B * w));
    cap = B;
  }

  void forward(int B) {
    const int w = width;
    gemm<float, float>(B, w, n_in, x, n_in, 1, p + o_w1, 1, n_in, z1, w, 1, p + o_b1, false);
    k_mlp_act<<<grid_1d((int64_t)B * w), 256>>>(z1, a1, (int64_t)B * w);
    gemm<__nv_bfloat16, float>(B, w, w, a1, w, 1, p + o_w2, 1, w, z2, w, 1, p + o_b2, false);
    k_mlp_act<<<grid_1d((int64_t)B * w), 256>>>(z2, a2, (int64_t)B * w);
    gemm<__nv_bfloat16, float>(B, n_out, w, a2, w, 1, p + o_w3, 1, w, y, n_out, 1, p + o_b3, false);
    MCUDA(cudaGetLastError());
  }

  // loss and gradients of the batch held in x, t
  void backward(int B) {
    const int w = width;
    k_mlp_mse<<<1, 1024>>>(y, t, dy, loss, (int64_t)B * n_out);
    // layer 3: dW3 = dy^T a2, db3 = colsum dy, da2 = dy W3
    gemm<float, __nv_bfloat16>(n_out, w, B, dy, 1, n_out, a2, w, 1, g + o_w3, w, 1, nullptr, false);
    k_mlp_colsum<<<(n_out + 127) / 128, 128>>>(dy, g + o_b3, B, n_out);
    gemm<float, float>(B, w, n_out, dy, n_out, 1, p + o_w3, w, 1, da, w, 1, nullptr, false);
    k_mlp_dact<<<grid_1d((int64_t)B * w), 256>>>(da, z2, dz, (int64_t)B * w);
    // layer 2: dW2 = dz2^T a1, db2, da1 = dz2 W2
    gemm<float, __nv_bfloat16>(w, w, B, dz, 1, w, a1, w, 1, g + o_w2, w, 1, nullptr, false);
    k_mlp_colsum<<<(w + 127) / 128, 128>>>(dz, g + o_b2, B, w);
    gemm<float, float>(B, w, w, dz, w, 1, p + o_w2, w, 1, da, w, 1, nullptr, false);
    k_mlp_dact<<<grid_1d((int64_t)B * w), 256>>>(da, z1, dz, (int64_t)B * w);
    // layer 1: dW1 = dz1^T x, db1
    gemm<float, float>(w, n_in, B, dz, 1, w, x, n_in, 1, g + o_w1, n_in, 1, nullptr, false);
    k_mlp_colsum<<<(w + 127) / 128, 128>>>(dz, g + o_b1, B, w);
    MCUDA(cudaGetLastError());
  }

  void adam(float lr, float b1, float b2, float eps) {
    ++adam_t;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)adam_t));
    const float c2 = 1.f / (1.f - std::pow(b2, (float)adam_t));
    k_mlp_adam<<<grid_1d(np), 256>>>(p, g, m, v, np, lr, b1, b2, eps, c1, c2);
    MCUDA(cudaGetLastError());
  }
};

namespace {
void upload_batch(nsx_mlp *q, const float *x, const float *t, int B) {
  q->ensure_batch(B);
  MCUDA(cudaMemcpy(q->x, x, sizeof(float) * (size_t)B * q->n_in, cudaMemcpyHostToDevice));
  if (t) MCUDA(cudaMemcpy(q->t, t, sizeof(float) * (size_t)B * q->n_out, cudaMemcpyHostToDevice));
}
void check_handle(const nsx_mlp *q) {
  if (!q) throw Err{NSX_E_ARG, "null network handle"};
}
void check_batch(int B) {
  if (B <= 0 || B > (1 << 20)) throw Err{NSX_E_ARG, "batch size out of range (1 .. 2^20)"};
}
}  // namespace

extern "C" {

const char *nsx_mlp_last_error(void) { return g_mlp_err.c_str(); }

int nsx_mlp_create(int32_t n_in, int32_t width, int32_t n_out, uint64_t seed, int device, nsx_mlp **out) {
  if (!out) {
    g_mlp_err = "null output handle pointer";
    return NSX_E_ARG;
  }
  *out = nullptr;
  nsx_mlp *q = new (std::nothrow) nsx_mlp();
  if (!q) {
    g_mlp_err = "host allocation failed";
    return NSX_E_NOMEM;
  }
  int rc = mguard([&] {
    if (n_in <= 0 || width <= 0 || n_out <= 0 || n_in > 4096 || width > 4096 || n_out > 4096)
      throw Err{NSX_E_ARG, "layer sizes out of range (1 .. 4096)"};
    q->device = device;
    MDevice dg(device);
    q->n_in = n_in;
    q->width = width;
    q->n_out = n_out;
    int64_t o = 0;
    q->o_w1 = o; o += (int64_t)width * n_in;
    q->o_b1 = o; o += width;
    q->o_w2 = o; o += (int64_t)width * width;
    q->o_b2 = o; o += width;
    q->o_w3 = o; o += (int64_t)n_out * width;
    q->o_b3 = o; o += n_out;
    q->np = o;
    // initial weights: uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) from a 64-bit LCG, zero biases
    std::vector<float> h((size_t)o, 0.f);
    uint64_t s = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
      s = s * 6364136223846793005ull + 1442695040888963407ull;
      return (float)((double)(s >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    auto fill = [&](int64_t off, int64_t n, int fan_in) {
      const float a = 1.f / std::sqrt((float)fan_in);
      for (int64_t i = 0; i < n; ++i) h[off + i] = a * uni();
    };
    fill(q->o_w1, (int64_t)width * n_in, n_in);
    fill(q->o_w2, (int64_t)width * width, width);
    fill(q->o_w3, (int64_t)n_out * width, width);
    MCUDA(cudaMalloc(&q->p, sizeof(float) * o));
    MCUDA(cudaMalloc(&q->g, sizeof(float) * o));
    MCUDA(cudaMalloc(&q->m, sizeof(float) * o));
    MCUDA(cudaMalloc(&q->v, sizeof(float) * o));
    MCUDA(cudaMalloc(&q->loss, sizeof(float)));
    MCUDA(cudaMemcpy(q->p, h.data(), sizeof(float) * o, cudaMemcpyHostToDevice));
    MCUDA(cudaMemset(q->g, 0, sizeof(float) * o));
    MCUDA(cudaMemset(q->m, 0, sizeof(float) * o));
    MCUDA(cudaMemset(q->v, 0, sizeof(float) * o));
  });
  if (rc != NSX_OK) {
    nsx_mlp_destroy(q);
    return rc;
  }
  *out = q;
  return NSX_OK;
}

int64_t nsx_mlp_param_count(const nsx_mlp *q) { return q ? q->np : 0; }

int nsx_mlp_set_params(nsx_mlp *q, const float *params, int64_t n) {
  return mguard([&] {
    check_handle(q);
    if (!params || n != q->np) throw Err{NSX_E_ARG, "parameter count mismatch"};
    MDevice dg(q->device);
    MCUDA(cudaMemcpy(q->p, params, sizeof(float) * n, cudaMemcpyHostToDevice));
    MCUDA(cudaMemset(q->m, 0, sizeof(float) * n));
    MCUDA(cudaMemset(q->v, 0, sizeof(float) * n));
    q->adam_t = 0;
  });
}

int nsx_mlp_get_params(const nsx_mlp *q, float *params, int64_t n) {
  return mguard([&] {
    check_handle(q);
    if (!params || n != q->np) throw Err{NSX_E_ARG, "parameter count mismatch"};
    MDevice dg(q->device);
    MCUDA(cudaMemcpy(params, q->p, sizeof(float) * n, cudaMemcpyDeviceToHost));
  });
}

int nsx_mlp_forward(nsx_mlp *q, const float *x, int32_t batch, float *y) {
  return mguard([&] {
    check_handle(q);
    check_batch(batch);
    if (!x || !y) throw Err{NSX_E_ARG, "null argument"};
    MDevice dg(q->device);
    upload_batch(q, x, nullptr, batch);
    q->forward(batch);
    MCUDA(cudaMemcpy(y, q->y, sizeof(float) * (size_t)batch * q->n_out, cudaMemcpyDeviceToHost));
  });
}

int nsx_mlp_gradients(nsx_mlp *q, const float *x, const float *t, int32_t batch, float *loss, float *grad) {
  return mguard([&] {
    check_handle(q);
    check_batch(batch);
    if (!x || !t) throw Err{NSX_E_ARG, "null argument"};
    MDevice dg(q->device);
    upload_batch(q, x, t, batch);
    q->forward(batch);
    q->backward(batch);
    if (loss) MCUDA(cudaMemcpy(loss, q->loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (grad) MCUDA(cudaMemcpy(grad, q->g, sizeof(float) * q->np, cudaMemcpyDeviceToHost));
  });
}

int nsx_mlp_train(nsx_mlp *q, const float *x, const float *t, int32_t batch, int32_t steps, float lr, float *loss) {
  return mguard([&] {
    check_handle(q);
    check_batch(batch);
    if (!x || !t || steps < 0) throw Err{NSX_E_ARG, "bad argument"};
    MDevice dg(q->device);
    upload_batch(q, x, t, batch);
    for (int s = 0; s < steps; ++s) {
      q->forward(batch);
      q->backward(batch);
      q->adam(lr, 0.9f, 0.999f, 1e-8f);
    }
    q->forward(batch);
    k_mlp_mse<<<1, 1024>>>(q->y, q->t, q->dy, q->loss, (int64_t)batch * q->n_out);
    MCUDA(cudaGetLastError());
    if (loss) MCUDA(cudaMemcpy(loss, q->loss, sizeof(float), cudaMemcpyDeviceToHost));
  });
}

void nsx_mlp_destroy(nsx_mlp *q) {
  if (!q) return;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  cudaSetDevice(q->device);
  q->free_batch();
  for (void *ptr : {(void *)q->p, (void *)q->g, (void *)q->m, (void *)q->v, (void *)q->loss})
    if (ptr) cudaFree(ptr);
  if (prev >= 0 && prev != q->device) cudaSetDevice(prev);
  delete q;
}

}  // extern "C"
