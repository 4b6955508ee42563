// Thick-restart Lanczos in FP64 on the GPU (the reference's Lnz_OP / lnzort,
// src/NuLnz/NuCoreX.f90:240-791).
//
// Differences from the reference, by design:
// * all basis vectors stay in HBM (the reference keeps them in direct-access
//   disk records and reads every one back per iteration);
// * full classical Gram-Schmidt with a second pass (CGS2) against the whole
//   basis every step; the projected matrix T = V^T H V is assembled from the
//   Gram-Schmidt coefficients themselves, so after a thick restart the arrowhead
//   row appears without special cases (the reference's i == no_keep+1 branch,
//   NuCoreX.f90:351-355);
// * convergence is tested on Ritz residuals |beta_m s_mj| <= tol, not on the
//   stagnation of Ritz values between checks (NuCoreX.f90:719-737);
// * the small symmetric eigenproblem is solved on the GPU by a one-CTA parallel
//   cyclic Jacobi method (the reference uses Numerical Recipes tred2/tqli on the
//   host, ICommon.FI:188-597);
// * breakdown (beta below 1e-7 relative) restarts from a fresh random direction
//   orthogonalised against the basis, with a zero coupling, as the reference
//   does at NuCoreX.f90:368-382.
#include <algorithm>
#include <mutex>
#include <set>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>
#include "nsx_internal.h"

namespace nsx {

static constexpr int RED_CTAS = 592;   // 148 SMs x 4
static thread_local int64_t *g_launches = nullptr;  // the solving handle's launch counter
static inline void count_launch() {
  if (g_launches) ++*g_launches;
}
static constexpr int JT = 8;           // vectors per pass of the dot kernel

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// x[n] = U(-0.5, 0.5) on entries of the requested parity, 0 elsewhere
// (the reference's start vector, NuCoreX.f90:625-632, with its own generator).
__global__ void k_rand(double *x, const uint8_t *mask, int64_t n, uint64_t seed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double u = (double)(splitmix(seed * 0x100000001B3ull + (uint64_t)i) >> 11) * (1.0 / 9007199254740992.0);
    x[i] = mask[i] ? 0.5 - u : 0.0;
  }
}

// partial[cta][j] = sum over this CTA's slice of V[j0+j][i] * w[i], j < cnt (<= JT)
__global__ void __launch_bounds__(256) k_dots(const double *__restrict__ V, int64_t ldv, int j0, int cnt,
                                              const double *__restrict__ w, int64_t n, double *__restrict__ partial) {
  double acc[JT];
#pragma unroll
  for (int j = 0; j < JT; ++j) acc[j] = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double wi = w[i];
#pragma unroll
    for (int j = 0; j < JT; ++j)
      if (j < cnt) acc[j] = fma(V[(int64_t)(j0 + j) * ldv + i], wi, acc[j]);
  }
  __shared__ double red[JT][8];
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
#pragma unroll
  for (int j = 0; j < JT; ++j) {
    double v = acc[j];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[j][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < JT && threadIdx.x < cnt) {
    double s = 0.0;
    for (int k = 0; k < 8; ++k) s += red[threadIdx.x][k];
    partial[(int64_t)blockIdx.x * JT + threadIdx.x] = s;
  }
}
// out[j0+j] (+)= sum_cta partial[cta][j]   (fixed order: deterministic)
__global__ void k_dots_reduce(const double *__restrict__ partial, int nparts, int cnt, double *__restrict__ out,
                              int j0, int accumulate) {
  const int j = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (j >= cnt) return;
  double s = 0.0;
  for (int p = lane; p < nparts; p += 32) s += partial[(int64_t)p * JT + j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) out[j0 + j] = accumulate ? out[j0 + j] + s : s;
}
// w -= sum_{j<cnt} V[j] h[j]
__global__ void __launch_bounds__(256) k_sub(const double *__restrict__ V, int64_t ldv, int cnt,
                                             const double *__restrict__ h, double *__restrict__ w, int64_t n) {
  __shared__ double hs[256];
  for (int j = threadIdx.x; j < cnt && j < 256; j += blockDim.x) hs[j] = h[j];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s = w[i];
    for (int j = 0; j < cnt; ++j) s = fma(-hs[j], V[(int64_t)j * ldv + i], s);
    w[i] = s;
  }
}
// ---- classical Gram-Schmidt with a second pass (CGS2): four passes over the basis ----
// k_cg_dot:    h = V^T w                 (V and w read once)
// k_cg_subnrm: w -= V h                  (V read once, w read and written)
// k_cg_dot:    h2 = V^T w
// k_cg_subnrm: w -= V h2, ||w||^2
// Each pass streams the basis at the HBM roof; a fused subtract-and-dot pass (the second read
// of each chunk from L2) measured 3x one pass, more than the two passes it replaced.
// Per-CTA partial sums go to partial[cta][CG_MAXJ] and are added in a fixed order by
// k_cg_reduce (deterministic).
constexpr int CG_MAXJ = 128;   // basis vectors per pass (the window is capped below it)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Pass 1: each CTA takes row chunks of `chunk` rows (chunk <= CG_CHUNK_MAX; one chunk per CTA
// when the vector allows), stages w's chunk in shared memory, and warp q forms the chunk's
// dots with vectors q, q + 8, ..., reading each vector's chunk once with 32-lane coalesced
// loads; the lanes' sums stay in registers until the CTA's last chunk.
__global__ void __launch_bounds__(256) k_cg_dot(const double *__restrict__ V, int64_t ldv, int cnt,
                                                const double *__restrict__ w, int64_t n, int chunk,
                                                double *__restrict__ partial) {
  extern __shared__ double cg_sm[];   // [chunk]
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr int JW = CG_MAXJ / 8;     // vectors per warp
  double acc[JW];
#pragma unroll
  for (int jj = 0; jj < JW; ++jj) acc[jj] = 0.0;
  for (int64_t base = (int64_t)blockIdx.x * chunk; base < n; base += (int64_t)gridDim.x * chunk) {
    const int rows = (int)(n - base < chunk ? n - base : chunk);
    __syncthreads();
    for (int r = tid; r < rows; r += 256) cg_sm[r] = w[base + r];
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < JW; ++jj) {
      const int j = warp + 8 * jj;
      if (j < cnt) {
        const double *vj = V + (int64_t)j * ldv + base;
        double a0 = 0.0, a1 = 0.0;
        int r = lane;
        for (; r + 32 < rows; r += 64) {
          a0 = fma(vj[r], cg_sm[r], a0);
          a1 = fma(vj[r + 32], cg_sm[r + 32], a1);
        }
        if (r < rows) a0 = fma(vj[r], cg_sm[r], a0);
        acc[jj] += a0 + a1;
      }
    }
  }
#pragma unroll
  for (int jj = 0; jj < JW; ++jj) {
    const int j = warp + 8 * jj;
    const double v = warp_sum(acc[jj]);
    if (lane == 0 && j < cnt) partial[(int64_t)blockIdx.x * CG_MAXJ + j] = v;
  }
}

__global__ void __launch_bounds__(256) k_cg_subnrm(const double *__restrict__ V, int64_t ldv, int cnt,
                                                   const double *__restrict__ h, double *__restrict__ w, int64_t n,
                                                   double *__restrict__ partial) {
  __shared__ double hs[CG_MAXJ];
  __shared__ double red[8];
  const int tid = threadIdx.x;
  for (int j = tid; j < cnt; j += 256) hs[j] = h[j];
  __syncthreads();
  double nrm = 0.0;
  for (int64_t r = (int64_t)blockIdx.x * 256 + tid; r < n; r += (int64_t)gridDim.x * 256) {
    // four independent chains
    double s0 = w[r], s1 = 0.0, s2 = 0.0, s3 = 0.0;
    const double *vr = V + r;
    int j = 0;
    for (; j + 8 <= cnt; j += 8) {   // eight loads issued before their FMAs
      double v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = vr[(int64_t)(j + q) * ldv];
      s0 = fma(-hs[j], v[0], s0);
      s1 = fma(-hs[j + 1], v[1], s1);
      s2 = fma(-hs[j + 2], v[2], s2);
      s3 = fma(-hs[j + 3], v[3], s3);
      s0 = fma(-hs[j + 4], v[4], s0);
      s1 = fma(-hs[j + 5], v[5], s1);
      s2 = fma(-hs[j + 6], v[6], s2);
      s3 = fma(-hs[j + 7], v[7], s3);
    }
    for (; j < cnt; ++j) s0 = fma(-hs[j], vr[(int64_t)j * ldv], s0);
    const double sv = (s0 + s1) + (s2 + s3);
    w[r] = sv;
    nrm = fma(sv, sv, nrm);
  }
  nrm = warp_sum(nrm);
  if ((tid & 31) == 0) red[tid >> 5] = nrm;
  __syncthreads();
  if (tid == 0) {
    double v = 0.0;
    for (int q = 0; q < 8; ++q) v += red[q];
    partial[(int64_t)blockIdx.x * CG_MAXJ] = v;
  }
}

// out[j] = sum_cta partial[cta][j], j < cnt: one warp per j, fixed order
__global__ void __launch_bounds__(256) k_cg_reduce(const double *__restrict__ partial, int nparts, int cnt,
                                                   double *__restrict__ out) {
  const int j = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (j >= cnt) return;
  double v = 0.0;
  for (int p = lane; p < nparts; p += 32) v += partial[(int64_t)p * CG_MAXJ + j];
  v = warp_sum(v);
  if (lane == 0) out[j] = v;
}

// v = w / sqrt(nrm2[0]) (zero if nrm2 == 0)
__global__ void k_scale(const double *__restrict__ w, double *__restrict__ v, const double *__restrict__ nrm2,
                        int64_t n) {
  double b = sqrt(nrm2[0]);
  double s = b > 0.0 ? 1.0 / b : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = w[i] * s;
}
// out[c] = sum_{j<m} V[j] S[j + m c], c < k  (Ritz rotation, the reference's NuCoreX.f90:455-470)
__global__ void __launch_bounds__(256) k_rotate(const double *__restrict__ V, int64_t ldv, int m,
                                                const double *__restrict__ S, int k, double *__restrict__ out,
                                                int64_t n) {
  extern __shared__ double ss[];  // m*k
  for (int e = threadIdx.x; e < m * k; e += blockDim.x) ss[e] = S[e];
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int c0 = 0; c0 < k; c0 += 16) {
      double acc[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) acc[c] = 0.0;
      for (int j = 0; j < m; ++j) {
        double v = V[(int64_t)j * ldv + i];
#pragma unroll
        for (int c = 0; c < 16; ++c)
          if (c0 + c < k) acc[c] = fma(v, ss[j + m * (c0 + c)], acc[c]);
      }
#pragma unroll
      for (int c = 0; c < 16; ++c)
        if (c0 + c < k) out[(int64_t)(c0 + c) * ldv + i] = acc[c];
    }
  }
}

// One-CTA parallel cyclic Jacobi for a symmetric m x m matrix A (column-major,
// lda = m).  Tournament (round-robin) ordering: each round rotates m/2 disjoint
// (p, q) pairs, rows first, then columns.  Outputs eigenvalues (unsorted) in
// evals and eigenvectors as columns of Vout.  Sweeps stop when the off-diagonal
// Frobenius norm falls below 1e-13 of the total, at most 60 sweeps; status[0]
// = sweeps used, or -1 if not converged (the host reports NSX_E_NUMERIC).
__global__ void __launch_bounds__(512) k_jacobi(const double *__restrict__ Ain, int m, double *__restrict__ evals,
                                                double *__restrict__ Vout, int *__restrict__ status) {
  extern __shared__ double sm[];
  const int mp = m + (m & 1);   // even size (a dummy index when m is odd)
  double *A = sm;               // mp x mp
  double *Q = A + mp * mp;      // mp x mp
  double *cs = Q + mp * mp;     // [mp/2] cos
  double *sn = cs + mp / 2;     // [mp/2] sin
  int *perm = reinterpret_cast<int *>(sn + mp / 2);  // [mp]
  __shared__ double offn, totn;
  for (int e = threadIdx.x; e < mp * mp; e += blockDim.x) {
    int r = e % mp, c = e / mp;
    A[e] = (r < m && c < m) ? Ain[r + m * c] : 0.0;
    Q[e] = r == c ? 1.0 : 0.0;
  }
  for (int e = threadIdx.x; e < mp; e += blockDim.x) perm[e] = e;
  __syncthreads();
  int sweep = 0;
  for (; sweep < 60; ++sweep) {
    if (threadIdx.x == 0) {
      offn = 0.0;
      totn = 0.0;
    }
    __syncthreads();
    double lo = 0.0, lt = 0.0;
    for (int e = threadIdx.x; e < mp * mp; e += blockDim.x) {
      double v = A[e] * A[e];
      lt += v;
      if (e % mp != e / mp) lo += v;
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo += __shfl_down_sync(0xffffffffu, lo, o);
      lt += __shfl_down_sync(0xffffffffu, lt, o);
    }
    if (threadIdx.x % 32 == 0) {
      atomicAdd(&offn, lo);
      atomicAdd(&totn, lt);
    }
    __syncthreads();
    if (offn <= 1e-26 * totn || totn == 0.0) break;
    __syncthreads();
    for (int round = 0; round < mp - 1; ++round) {
      // circle-method pairs (perm[i], perm[mp-1-i]): every pair once per sweep
      for (int i = threadIdx.x; i < mp / 2; i += blockDim.x) {
        int p = perm[i], q = perm[mp - 1 - i];
        if (p > q) { int t = p; p = q; q = t; }
        double apq = A[p + mp * q];
        double c = 1.0, s = 0.0;
        double app = A[p + mp * p], aqq = A[q + mp * q];
        if (fabs(apq) > 1e-18 * (fabs(app) + fabs(aqq)) && apq != 0.0) {
          double tau = (aqq - app) / (2.0 * apq);
          double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        cs[i] = c;
        sn[i] = s;
      }
      __syncthreads();
      // rows: A <- J^T A
      for (int e = threadIdx.x; e < (mp / 2) * mp; e += blockDim.x) {
        int i = e / mp, k = e % mp;
        int p = perm[i], q = perm[mp - 1 - i];
        if (p > q) { int t = p; p = q; q = t; }
        double c = cs[i], s = sn[i];
        double ap = A[p + mp * k], aq = A[q + mp * k];
        A[p + mp * k] = c * ap - s * aq;
        A[q + mp * k] = s * ap + c * aq;
      }
      __syncthreads();
      // columns: A <- A J ; Q <- Q J
      for (int e = threadIdx.x; e < (mp / 2) * mp; e += blockDim.x) {
        int i = e / mp, k = e % mp;
        int p = perm[i], q = perm[mp - 1 - i];
        if (p > q) { int t = p; p = q; q = t; }
        double c = cs[i], s = sn[i];
        double ap = A[k + mp * p], aq = A[k + mp * q];
        A[k + mp * p] = c * ap - s * aq;
        A[k + mp * q] = s * ap + c * aq;
        double qp = Q[k + mp * p], qq = Q[k + mp * q];
        Q[k + mp * p] = c * qp - s * qq;
        Q[k + mp * q] = s * qp + c * qq;
      }
      __syncthreads();
      // next tournament round: keep perm[0], rotate the rest
      if (threadIdx.x == 0) {
        int last = perm[mp - 1];
        for (int e = mp - 1; e > 1; --e) perm[e] = perm[e - 1];
        perm[1] = last;
      }
      __syncthreads();
    }
  }
  for (int e = threadIdx.x; e < m; e += blockDim.x) evals[e] = A[e + mp * e];
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    int r = e % m, c = e / m;
    Vout[e] = Q[r + mp * c];
  }
  if (threadIdx.x == 0) status[0] = sweep < 60 ? sweep : -1;
}

// ---------------------------------------------------------------------------
// Device workspace of the solver, kept by the handle between solves (allocated by the first
// solve and grown when a later one needs more), so that a solve allocates nothing once the
// handle has solved a problem of its size: the basis V, the residual w, the rotation buffer,
// the refinement's H Y, the reduction partials and the small matrices.
struct Workspace {
  int64_t n = 0;
  int vcap = 0, tcap = 0, mcap = 0, hycap = 0;
  double *V = nullptr, *w = nullptr, *tmp = nullptr, *HY = nullptr, *partial = nullptr, *h = nullptr,
         *h2 = nullptr;
  double *T = nullptr, *ev = nullptr, *S = nullptr;
  int *status = nullptr;
  uint8_t *mask = nullptr;
  void free_all() {
    void *p[] = {V, w, tmp, HY, partial, h, h2, T, ev, S, status, mask};
    for (void *q : p)
      if (q) cudaFree(q);
    *this = Workspace();
  }
};

void release_lanczos(nsx_handle *h) {
  if (!h->lws) return;
  Workspace *ws = static_cast<Workspace *>(h->lws);
  ws->free_all();
  delete ws;
  h->lws = nullptr;
}

// The handle's workspace with room for a window of m, keep kept vectors and nev pairs.
static Workspace &workspace(nsx_handle *h, int m, int keep, int nev, cudaStream_t s) {
  if (!h->lws) h->lws = new Workspace();
  Workspace &ws = *static_cast<Workspace *>(h->lws);
  const int64_t n = h->no_state;
  const int vneed = std::max(m + 1, 2 * nev), tneed = std::max(keep, nev);
  if (ws.n == n && ws.vcap >= vneed && ws.tcap >= tneed && ws.mcap >= m && ws.hycap >= nev) return ws;
  NSX_CUDA(cudaStreamSynchronize(s));
  ws.free_all();
  ws.n = n;
  ws.vcap = vneed;
  ws.tcap = tneed;
  ws.mcap = m;
  ws.hycap = nev;
  NSX_CUDA(cudaMalloc(&ws.V, sizeof(double) * n * vneed));
  NSX_CUDA(cudaMalloc(&ws.w, sizeof(double) * n));
  NSX_CUDA(cudaMalloc(&ws.tmp, sizeof(double) * n * tneed));
  NSX_CUDA(cudaMalloc(&ws.HY, sizeof(double) * n * nev));
  NSX_CUDA(cudaMalloc(&ws.partial, sizeof(double) * RED_CTAS * std::max(JT, CG_MAXJ)));
  NSX_CUDA(cudaMalloc(&ws.h, sizeof(double) * (m + 8)));
  NSX_CUDA(cudaMalloc(&ws.h2, sizeof(double) * (m + 8)));
  NSX_CUDA(cudaMalloc(&ws.T, sizeof(double) * m * m));
  NSX_CUDA(cudaMalloc(&ws.ev, sizeof(double) * m));
  NSX_CUDA(cudaMalloc(&ws.S, sizeof(double) * m * m));
  NSX_CUDA(cudaMalloc(&ws.status, sizeof(int)));
  NSX_CUDA(cudaMalloc(&ws.mask, n));
  NSX_CUDA(cudaMemcpyAsync(ws.mask, h->lcoef.data(), n, cudaMemcpyHostToDevice, s));
  NSX_CUDA(cudaStreamSynchronize(s));   // the mask copy from pageable memory has landed
  return ws;
}

// Rows per chunk of k_cg_dot: the vector over RED_CTAS chunks, whole warps, at most CG_CHUNK_MAX.
constexpr int CG_CHUNK_MAX = 4096;
static int cg_chunk(int64_t n) {
  const int64_t per = (n + RED_CTAS - 1) / RED_CTAS;
  return (int)std::min<int64_t>(CG_CHUNK_MAX, std::max<int64_t>(32, (per + 31) / 32 * 32));
}

// CGS2 of w against the first cnt basis vectors: h = V^T w, w -= V h, h2 = V^T w, w -= V h2,
// nrm2 = ||w||^2 (four passes over V, seven launches).
static void cgs2(Workspace &ws, int cnt, double *h, double *h2, double *nrm2, cudaStream_t s) {
  const int64_t n = ws.n;
  const double *V = ws.V;
  const int chunk = cg_chunk(n);
  for (int pass = 0; pass < 2; ++pass) {
    double *hp = pass == 0 ? h : h2;
    count_launch();
    k_cg_dot<<<RED_CTAS, 256, sizeof(double) * chunk, s>>>(V, n, cnt, ws.w, n, chunk, ws.partial);
    count_launch();
    k_cg_reduce<<<(cnt + 7) / 8, 256, 0, s>>>(ws.partial, RED_CTAS, cnt, hp);
    count_launch();
    k_cg_subnrm<<<RED_CTAS, 256, 0, s>>>(V, n, cnt, hp, ws.w, n, ws.partial);
  }
  count_launch();
  k_cg_reduce<<<1, 256, 0, s>>>(ws.partial, RED_CTAS, 1, nrm2);
  NSX_CUDA(cudaGetLastError());
}

static unsigned grid_for(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, RED_CTAS); }

// h[0..cnt) = V[0..cnt)^T w  (or +=)
static void dots(Workspace &ws, const double *V, int64_t ld, int cnt, const double *w, int64_t n, double *h,
                 bool acc, cudaStream_t s) {
  for (int j0 = 0; j0 < cnt; j0 += JT) {
    int c = std::min(JT, cnt - j0);
    count_launch();
    k_dots<<<RED_CTAS, 256, 0, s>>>(V, ld, j0, c, w, n, ws.partial);
    count_launch();
    k_dots_reduce<<<1, 32 * JT, 0, s>>>(ws.partial, RED_CTAS, c, h, j0, acc ? 1 : 0);
  }
}
static void subtract(const double *V, int64_t ld, int cnt, const double *h, double *w, int64_t n, cudaStream_t s) {
  for (int j0 = 0; j0 < cnt; j0 += 256) {
    int c = std::min(256, cnt - j0);
    count_launch();
    k_sub<<<grid_for(n), 256, 0, s>>>(V + (int64_t)j0 * ld, ld, c, h + j0, w, n);
  }
}

// Largest window (k_jacobi keeps two m x m FP64 matrices in shared memory) and the
// shared-memory caps it implies.  The caps are kernel attributes shared by every host
// thread, so they are set once per device to these maxima (never per launch: a
// concurrent solve could otherwise lower the cap between another solve's setting and
// its launch).
constexpr int MAX_WINDOW = 112;
constexpr size_t JACOBI_SMEM_MAX = sizeof(double) * (2 * (size_t)MAX_WINDOW * MAX_WINDOW + MAX_WINDOW) +
                                   sizeof(int) * MAX_WINDOW;
constexpr size_t ROTATE_SMEM_MAX = sizeof(double) * (size_t)MAX_WINDOW * MAX_WINDOW;

static void ensure_kernel_attributes(int device) {
  static std::mutex mu;
  static std::set<int> done;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count(device)) return;
  NSX_CUDA(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)JACOBI_SMEM_MAX));
  NSX_CUDA(cudaFuncSetAttribute(k_rotate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROTATE_SMEM_MAX));
  done.insert(device);
}

static void jacobi(Workspace &ws, int m, const std::vector<double> &T, std::vector<double> &evals,
                   std::vector<double> &evecs, cudaStream_t s) {
  NSX_CUDA(cudaMemcpyAsync(ws.T, T.data(), sizeof(double) * m * m, cudaMemcpyHostToDevice, s));
  int mp = m + (m & 1);
  size_t smem = sizeof(double) * (2 * (size_t)mp * mp + mp) + sizeof(int) * mp;
  count_launch();
  k_jacobi<<<1, 512, smem, s>>>(ws.T, m, ws.ev, ws.S, ws.status);
  NSX_CUDA(cudaGetLastError());
  std::vector<double> e(m), q((size_t)m * m);
  int st = 0;
  NSX_CUDA(cudaMemcpyAsync(e.data(), ws.ev, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaMemcpyAsync(q.data(), ws.S, sizeof(double) * m * m, cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaMemcpyAsync(&st, ws.status, sizeof(int), cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaStreamSynchronize(s));
  if (st < 0) fail(NSX_E_NUMERIC, "Jacobi eigensolver did not converge");
  std::vector<int> idx(m);
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return e[a] < e[b]; });
  evals.resize(m);
  evecs.resize((size_t)m * m);
  for (int c = 0; c < m; ++c) {
    evals[c] = e[idx[c]];
    for (int r = 0; r < m; ++r) evecs[r + (size_t)m * c] = q[r + (size_t)m * idx[c]];
  }
}

static double host_norm2(Workspace &ws, const double *w, int64_t n, cudaStream_t s) {
  dots(ws, w, 0, 1, w, n, ws.h2, false, s);
  double v = 0;
  NSX_CUDA(cudaMemcpyAsync(&v, ws.h2, sizeof(double), cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaStreamSynchronize(s));
  return v;
}

struct Timer {
  nsx_handle *h;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> evs;
  double total = 0;
  void matvec(const double *x, double *y, int prec, cudaStream_t s) {
    cudaEvent_t a, b;
    NSX_CUDA(cudaEventCreate(&a));
    NSX_CUDA(cudaEventCreate(&b));
    NSX_CUDA(cudaEventRecord(a, s));
    matvec_device(h, x, y, prec, s);
    NSX_CUDA(cudaEventRecord(b, s));
    evs.push_back({a, b});
  }
  void flush() {
    for (auto &p : evs) {
      float ms = 0;
      NSX_CUDA(cudaEventSynchronize(p.second));
      NSX_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
      total += ms * 1e-3;
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
    evs.clear();
  }
  ~Timer() {
    for (auto &p : evs) {
      cudaEventDestroy(p.first);
      cudaEventDestroy(p.second);
    }
  }
};

void solve(nsx_handle *h, const nsx_params *P, const nsx_state *resume, nsx_state *state_out, double *evals_out,
           double *evecs_out, nsx_report *rep) {
  auto t0 = std::chrono::steady_clock::now();
  const int64_t n = h->no_state;
  int64_t nallowed = 0;
  for (auto c : h->lcoef) nallowed += c;
  if (P->nev <= 0 || P->nev > 64) fail(NSX_E_ARG, "nev must be in 1..64");
  if (nallowed == 0) fail(NSX_E_ARG, "no basis states of the requested parity");
  const int nev = (int)std::min<int64_t>(P->nev, nallowed);
  int m = P->window > 0 ? P->window : 100;
  m = (int)std::min<int64_t>(m, nallowed);
  m = std::min(m, MAX_WINDOW);
  if (m < nev + 1 && m < nallowed) fail(NSX_E_ARG, "window must exceed nev");
  int keep = P->keep > 0 ? P->keep : std::max(nev + 10, m / 3);
  keep = std::min(keep, m - 2);
  if (keep < nev) keep = std::min(nev, m - 1);
  const int max_iter = P->max_iter > 0 ? P->max_iter : 2000;
  const double tol = P->tol > 0 ? P->tol : 1e-6;
  const int prec = P->precision;
  ensure_precision(h, prec);
  ensure_kernel_attributes(h->device);
  cudaStream_t s = solve_stream(h);  // the handle's own non-blocking stream: solves of different handles overlap
  struct CounterScope {
    CounterScope(int64_t *p) { g_launches = p; }
    ~CounterScope() { g_launches = nullptr; }
  } counter_scope(&h->launches);

  // basis (m+1 vectors; the FP64 refinement reuses it for 2*nev rotated vectors), kept by the handle
  Workspace &ws = workspace(h, m, keep, nev, s);
  Timer tm{h};
  int matvecs = 0, iters = 0, restarts = 0;
  auto V = [&](int j) { return ws.V + (int64_t)j * n; };

  std::vector<double> T((size_t)m * m, 0.0), theta, Sm;
  std::vector<double> hcol(m + 2), h2(m + 2);
  int i = 0, nconv = 0;
  constexpr int CHECK_MIN = 10, CHECK_MAX = 50;   // steps between convergence checks
  int next_check = 0, last_check_it = -1;
  double last_dist = 0.0;
  if (resume) {
    // a thick restart from a saved state (the reference's TRL resume, NuCoreX.f90:266-292): the
    // lowest `keep` Ritz vectors of the saved basis, then the saved next vector
    const int mr = resume->m;
    if (mr < 1 || mr > m || !resume->V || !resume->T || !resume->next)
      fail(NSX_E_ARG, "resume state: bad size (1.." + std::to_string(m) + " basis vectors) or null arrays");
    NSX_CUDA(cudaMemcpyAsync(ws.V, resume->V, sizeof(double) * n * mr, cudaMemcpyHostToDevice, s));
    std::vector<double> Tr(resume->T, resume->T + (size_t)mr * mr);
    for (int c = 0; c < mr; ++c)
      for (int r = 0; r < c; ++r) {
        const double a = 0.5 * (Tr[r + (size_t)mr * c] + Tr[c + (size_t)mr * r]);
        if (!std::isfinite(a)) fail(NSX_E_ARG, "resume state: T is not finite");
        Tr[r + (size_t)mr * c] = Tr[c + (size_t)mr * r] = a;
      }
    jacobi(ws, mr, Tr, theta, Sm, s);
    const int k = std::min(keep, mr);
    std::vector<double> Sk((size_t)mr * k);
    for (int c = 0; c < k; ++c)
      for (int r = 0; r < mr; ++r) Sk[r + (size_t)mr * c] = Sm[r + (size_t)mr * c];
    NSX_CUDA(cudaMemcpyAsync(ws.S, Sk.data(), sizeof(double) * Sk.size(), cudaMemcpyHostToDevice, s));
    count_launch();
    k_rotate<<<grid_for(n), 256, sizeof(double) * mr * k, s>>>(ws.V, n, mr, ws.S, k, ws.tmp, n);
    NSX_CUDA(cudaMemcpyAsync(ws.V, ws.tmp, sizeof(double) * n * k, cudaMemcpyDeviceToDevice, s));
    // A stored basis carries its storage's rounding (the reference's .trl records are FP32), so
    // the rotated vectors are orthonormalised again in FP64 and their projection V_k^T H V_k is
    // formed from k products instead of being taken as the stored matrix's Ritz values: the
    // resumed recurrence then converges to the exact eigenvalues, not to those of the rounded
    // state.
    for (int j = 0; j < k; ++j) {
      NSX_CUDA(cudaMemcpyAsync(ws.w, V(j), sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      if (j == 0)
        dots(ws, ws.w, 0, 1, ws.w, n, ws.h2, false, s);
      else
        cgs2(ws, j, ws.h, ws.h2, ws.h2 + j, s);
      count_launch();
      k_scale<<<grid_for(n), 256, 0, s>>>(ws.w, V(j), ws.h2 + j, n);
    }
    for (int j = 0; j < k; ++j) {
      tm.matvec(V(j), ws.w, prec, s);
      ++matvecs;
      dots(ws, ws.V, n, j + 1, ws.w, n, ws.h, false, s);
      NSX_CUDA(cudaMemcpyAsync(hcol.data(), ws.h, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
      NSX_CUDA(cudaStreamSynchronize(s));
      for (int r = 0; r <= j; ++r) {
        if (!std::isfinite(hcol[r])) fail(NSX_E_NUMERIC, "non-finite projection of a resumed basis vector");
        T[r + (size_t)m * j] = T[j + (size_t)m * r] = hcol[r];
      }
    }
    NSX_CUDA(cudaMemcpyAsync(ws.w, resume->next, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    cgs2(ws, k, ws.h, ws.h2, ws.h2 + k, s);   // the next vector, orthogonal to the kept ones
    double nn2 = 0;
    NSX_CUDA(cudaMemcpyAsync(&nn2, ws.h2 + k, sizeof(double), cudaMemcpyDeviceToHost, s));
    NSX_CUDA(cudaStreamSynchronize(s));
    if (!(nn2 > 1e-20) || !std::isfinite(nn2)) fail(NSX_E_ARG, "resume state: the next vector lies in the basis");
    count_launch();
    k_scale<<<grid_for(n), 256, 0, s>>>(ws.w, V(k), ws.h2 + k, n);
    NSX_CUDA(cudaGetLastError());
    i = k;
    iters = std::max(resume->iterations, 0);
    restarts = std::max(resume->restarts, 0) + 1;
  }
  // start vector
  if (resume) {
  } else if (P->start) {
    NSX_CUDA(cudaMemcpyAsync(V(0), P->start, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  } else {
    count_launch();
    k_rand<<<grid_for(n), 256, 0, s>>>(V(0), ws.mask, n, P->seed ? P->seed : 5);
  }
  if (!resume) {
    double nn = host_norm2(ws, V(0), n, s);
    if (!(nn > 0) || !std::isfinite(nn)) fail(NSX_E_ARG, "start vector is zero or not finite");
    count_launch();
    k_scale<<<grid_for(n), 256, 0, s>>>(V(0), V(0), ws.h2, n);
  }
  for (int it = 0; !resume && it < P->pre_iter; ++it) {  // power pre-iterations (NuCoreX.f90:639-654)
    tm.matvec(V(0), ws.w, prec, s);
    ++matvecs;
    dots(ws, ws.w, 0, 1, ws.w, n, ws.h2, false, s);
    count_launch();
    k_scale<<<grid_for(n), 256, 0, s>>>(ws.w, V(0), ws.h2, n);
  }
  NSX_CUDA(cudaGetLastError());

  std::vector<double> res(nev, 0.0);
  for (;;) {
    // ---- one Lanczos step on basis vector i: column i of T, v_{i+1} ----
    tm.matvec(V(i), ws.w, prec, s);
    ++matvecs;
    ++iters;
    cgs2(ws, i + 1, ws.h, ws.h2, ws.h2 + (i + 1), s);   // full reorthogonalisation, two passes
    NSX_CUDA(cudaMemcpyAsync(hcol.data(), ws.h, sizeof(double) * (i + 1), cudaMemcpyDeviceToHost, s));
    NSX_CUDA(cudaMemcpyAsync(h2.data(), ws.h2, sizeof(double) * (i + 2), cudaMemcpyDeviceToHost, s));
    NSX_CUDA(cudaStreamSynchronize(s));
    double scale = 0;
    for (int j = 0; j <= i; ++j) {
      double v = hcol[j] + h2[j];
      if (!std::isfinite(v)) fail(NSX_E_NUMERIC, "non-finite Lanczos coefficient");
      T[j + (size_t)m * i] = v;  // full projection V^T H v_i (arrowhead row after a restart included)
      T[i + (size_t)m * j] = v;
      scale = std::max(scale, std::fabs(v));
    }
    double beta = std::sqrt(std::max(h2[i + 1], 0.0));
    const bool exhausted = i + 1 >= nallowed;  // Krylov space complete: the projection is exact
    if (exhausted) beta = 0.0;
    const bool full = i + 1 == m;
    const bool limit = iters >= max_iter;
    if (!exhausted && !full && beta <= 1e-7 * std::max(scale, 1.0)) {
      // breakdown: a random direction orthogonal to the basis, zero coupling (NuCoreX.f90:368-382)
      count_launch();
      k_rand<<<grid_for(n), 256, 0, s>>>(ws.w, ws.mask, n, 0xA5A5A5A5ull + (uint64_t)iters);
      for (int pass = 0; pass < 2; ++pass) {
        dots(ws, ws.V, n, i + 1, ws.w, n, ws.h, false, s);
        subtract(ws.V, n, i + 1, ws.h, ws.w, n, s);
      }
      dots(ws, ws.w, 0, 1, ws.w, n, ws.h2 + (i + 1), false, s);
      beta = 0.0;
    }
    if (!full && !exhausted) {
      count_launch();
      k_scale<<<grid_for(n), 256, 0, s>>>(ws.w, V(i + 1), ws.h2 + (i + 1), n);
      NSX_CUDA(cudaGetLastError());
      T[(i + 1) + (size_t)m * i] = beta;
      T[i + (size_t)m * (i + 1)] = beta;
    }
    const bool check = full || exhausted || limit || (iters >= next_check && i + 1 >= nev + 2);
    if (!check) {
      ++i;
      continue;
    }
    // ---- Ritz pairs of the leading (i+1) x (i+1) block ----
    const int mm = i + 1;
    std::vector<double> Tm((size_t)mm * mm);
    for (int c = 0; c < mm; ++c)
      for (int r = 0; r < mm; ++r) Tm[r + (size_t)mm * c] = T[r + (size_t)m * c];
    jacobi(ws, mm, Tm, theta, Sm, s);
    nconv = 0;
    double dist = 0.0;   // log(residual / tol) of the slowest unconverged pair
    for (int j = 0; j < nev && j < mm; ++j) {
      res[j] = std::fabs(beta * Sm[(mm - 1) + (size_t)mm * j]);
      if (res[j] <= tol && nconv == j) ++nconv;
      if (res[j] > tol) dist = std::max(dist, std::log(res[j] / tol));
    }
    // The next check: every check is a Jacobi solve of the projected matrix, so instead of a
    // fixed interval the residuals' decay since the last check is extrapolated and the next
    // check placed at 70 % of the steps it predicts to convergence (10 to 50 steps on).
    {
      int step = CHECK_MIN;
      if (last_check_it >= 0 && dist < last_dist && iters > last_check_it) {
        const double rate = (last_dist - dist) / (double)(iters - last_check_it);
        step = (int)std::min<double>(CHECK_MAX, std::max<double>(CHECK_MIN, 0.7 * dist / rate));
      }
      last_dist = dist;
      last_check_it = iters;
      next_check = iters + step;
    }
    if (nconv >= nev || exhausted || limit) {
      // Ritz vectors y_c = V S[:, c], c < nev, into ws.tmp
      const int ne = std::min(nev, mm);
      std::vector<double> Sk((size_t)mm * nev, 0.0);
      for (int c = 0; c < ne; ++c)
        for (int r = 0; r < mm; ++r) Sk[r + (size_t)mm * c] = Sm[r + (size_t)mm * c];
      NSX_CUDA(cudaMemcpyAsync(ws.S, Sk.data(), sizeof(double) * Sk.size(), cudaMemcpyHostToDevice, s));
      size_t smem = sizeof(double) * mm * nev;
      count_launch();
      k_rotate<<<grid_for(n), 256, smem, s>>>(ws.V, n, mm, ws.S, nev, ws.tmp, n);
      NSX_CUDA(cudaGetLastError());
      if (state_out) {   // the basis, its projection and the next vector: H V = V T + beta next e_m^T
        if (state_out->m < mm || !state_out->V || !state_out->T || !state_out->next)
          fail(NSX_E_ARG, "state output: room for " + std::to_string(mm) + " basis vectors needed");
        NSX_CUDA(cudaMemcpyAsync(state_out->V, ws.V, sizeof(double) * n * mm, cudaMemcpyDeviceToHost, s));
        for (int c = 0; c < mm; ++c)
          for (int r = 0; r < mm; ++r) state_out->T[r + (size_t)mm * c] = T[r + (size_t)m * c];
        const bool scaled = !full && !exhausted;   // V(i+1) = w / beta was formed above
        NSX_CUDA(cudaMemcpyAsync(state_out->next, scaled ? V(i + 1) : ws.w, sizeof(double) * n,
                                 cudaMemcpyDeviceToHost, s));
        NSX_CUDA(cudaStreamSynchronize(s));
        if (!scaled) {
          const double b = std::sqrt(std::max(h2[i + 1], 0.0));
          for (int64_t e = 0; e < n; ++e) state_out->next[e] = b > 0 ? state_out->next[e] / b : 0.0;
        }
        state_out->m = mm;
        state_out->beta = beta;
        state_out->iterations = iters;
        state_out->restarts = restarts;
      }
      break;
    }
    if (!full) {
      ++i;
      continue;
    }
    // ---- thick restart: keep the lowest `keep` Ritz vectors, continue from the residual ----
    ++restarts;
    std::vector<double> Sk((size_t)m * keep);
    for (int c = 0; c < keep; ++c)
      for (int r = 0; r < m; ++r) Sk[r + (size_t)m * c] = Sm[r + (size_t)m * c];
    NSX_CUDA(cudaMemcpyAsync(ws.S, Sk.data(), sizeof(double) * Sk.size(), cudaMemcpyHostToDevice, s));
    size_t smem = sizeof(double) * m * keep;
    count_launch();
    k_rotate<<<grid_for(n), 256, smem, s>>>(ws.V, n, m, ws.S, keep, ws.tmp, n);
    NSX_CUDA(cudaMemcpyAsync(ws.V, ws.tmp, sizeof(double) * n * keep, cudaMemcpyDeviceToDevice, s));
    count_launch();
    k_scale<<<grid_for(n), 256, 0, s>>>(ws.w, V(keep), ws.h2 + (i + 1), n);
    NSX_CUDA(cudaGetLastError());
    std::fill(T.begin(), T.end(), 0.0);
    for (int c = 0; c < keep; ++c) T[c + (size_t)m * c] = theta[c];
    i = keep;
  }
  tm.flush();
  // results
  for (int c = 0; c < nev; ++c) evals_out[c] = theta[c];
  if (P->refine) {
    // FP64 Rayleigh-Ritz on the Ritz vectors: G = Y^T H Y, eigen-decompose, rotate
    double *HY = ws.HY;
    for (int c = 0; c < nev; ++c) {
      tm.matvec(ws.tmp + (int64_t)c * n, HY + (int64_t)c * n, NSX_FP64, s);
      ++matvecs;
    }
    std::vector<double> G((size_t)nev * nev), Yo((size_t)nev * nev);
    for (int c = 0; c < nev; ++c) {
      dots(ws, ws.tmp, n, nev, HY + (int64_t)c * n, n, ws.h, false, s);
      dots(ws, ws.tmp, n, nev, ws.tmp + (int64_t)c * n, n, ws.h2, false, s);
      NSX_CUDA(cudaMemcpyAsync(G.data() + (size_t)nev * c, ws.h, sizeof(double) * nev, cudaMemcpyDeviceToHost, s));
      NSX_CUDA(cudaMemcpyAsync(Yo.data() + (size_t)nev * c, ws.h2, sizeof(double) * nev, cudaMemcpyDeviceToHost, s));
    }
    NSX_CUDA(cudaStreamSynchronize(s));
    for (int c = 0; c < nev; ++c)
      for (int r = 0; r < c; ++r) {
        double a = 0.5 * (G[r + (size_t)nev * c] + G[c + (size_t)nev * r]);
        G[r + (size_t)nev * c] = G[c + (size_t)nev * r] = a;
      }
    std::vector<double> th2, S2;
    jacobi(ws, nev, G, th2, S2, s);
    for (int c = 0; c < nev; ++c) evals_out[c] = th2[c];
    // rotate Ritz vectors and their images; residuals in FP64
    NSX_CUDA(cudaMemcpyAsync(ws.S, S2.data(), sizeof(double) * nev * nev, cudaMemcpyHostToDevice, s));
    size_t smem = sizeof(double) * nev * nev;
    count_launch();
    k_rotate<<<grid_for(n), 256, smem, s>>>(ws.tmp, n, nev, ws.S, nev, ws.V, n);
    count_launch();
    k_rotate<<<grid_for(n), 256, smem, s>>>(HY, n, nev, ws.S, nev, ws.V + (int64_t)nev * n, n);
    NSX_CUDA(cudaMemcpyAsync(ws.tmp, ws.V, sizeof(double) * n * nev, cudaMemcpyDeviceToDevice, s));
    for (int c = 0; c < nev; ++c) {
      // r = H y - theta y
      NSX_CUDA(cudaMemcpyAsync(ws.w, ws.V + (int64_t)(nev + c) * n, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      NSX_CUDA(cudaMemcpyAsync(ws.h, &th2[c], sizeof(double), cudaMemcpyHostToDevice, s));
      subtract(ws.tmp + (int64_t)c * n, n, 1, ws.h, ws.w, n, s);
      res[c] = std::sqrt(std::max(host_norm2(ws, ws.w, n, s), 0.0));
    }
    tm.flush();
    nconv = 0;
    for (int c = 0; c < nev; ++c)
      if (res[c] <= tol && nconv == c) ++nconv;
  }
  if (evecs_out) NSX_CUDA(cudaMemcpyAsync(evecs_out, ws.tmp, sizeof(double) * n * nev, cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaStreamSynchronize(s));
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->iterations = iters;
    rep->matvecs = matvecs;
    rep->restarts = restarts;
    rep->converged = nconv;
    rep->matvec_seconds = tm.total;
    for (int c = 0; c < nev && c < 64; ++c) rep->residual[c] = res[c];
    rep->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
}

}  // namespace nsx
