// H.v on the GPU for the pn-factorised J-scheme Hamiltonian.
//
// The reference computes the product as multiplyx (pn), multiplya (pp) and
// multiplyb (nn) in src/NuLnz/NuCoreX.f90:76-226 with axpy loops over density
// sub-blocks (src/NuCommonX/NuCommonX.f90:745-919, 1009-1104).  Here it is
// three stream-ordered kernels, each output element owned by exactly one CTA
// (no atomics, no per-thread vector copies):
//
//   k_like : out_b  = H_pp(Ja) C_b + C_b H_nn(Jb)              (dense tiled GEMM)
//   k_y    : Y_(h,k) = C_h rho_k^T for every (input block h, neutron density k)
//            that the pn table uses -- computed once and reused by every proton
//            operator, where the reference recomputes it per proton operator;
//   k_a    : out[P_l rows] += sum_(a,P_r) rho_a[P_l,P_r] (sum_k w_ak Y_(h,k)[P_r rows])
//            (mixing of the Y intermediates fused into the operand load).
//
// Templated on the contraction type: double (the FP64 form) or float (the FP32
// form, FP64 vectors converted at the boundary).
#include <algorithm>
#include <cstdio>
#include "nsx_internal.h"

namespace nsx {

// ---------------------------------------------------------------------------
// k_like: 64x64 output tile per CTA, 256 threads, 4x4 outputs per thread.
template <typename T>
__global__ void __launch_bounds__(256) k_like(const LTile *__restrict__ tiles, const T *__restrict__ x,
                                              T *__restrict__ out, const T *__restrict__ HA,
                                              const T *__restrict__ HB) {
  const LTile t = tiles[blockIdx.x];
  const T *C = x + t.c;
  const T *Ha = HA + t.ha;
  const T *Hb = HB + t.hb;
  __shared__ T As[16][64 + 1];
  __shared__ T Bs[16][64 + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // cols tx*4.., rows ty*4..
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  const int da = t.da, db = t.db;
  // pass 0: Ha[r0.., k] * C[k, c0..], K = da ; pass 1: C[r0.., k] * Hb[k, c0..], K = db
  for (int pass = 0; pass < 2; ++pass) {
    const T *L = pass == 0 ? Ha : C;
    const T *R = pass == 0 ? C : Hb;
    const int ldl = da;
    const int ldr = pass == 0 ? da : db;
    const int K = pass == 0 ? da : db;
    for (int k0 = 0; k0 < K; k0 += 16) {
      for (int e = threadIdx.x; e < 16 * 64; e += 256) {
        int r = e % 64, k = e / 64;
        int gr = t.r0 + r, gk = k0 + k;
        As[k][r] = (gr < da && gk < K) ? L[gr + (int64_t)ldl * gk] : T(0);
        int c = e / 16, kk = e % 16;
        int gc = t.c0 + c, gkk = k0 + kk;
        Bs[kk][c] = (gc < db && gkk < K) ? R[gkk + (int64_t)ldr * gc] : T(0);
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[k][ty * 4 + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx * 4 + j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int r = t.r0 + ty * 4 + i, c = t.c0 + tx * 4 + j;
      if (r < da && c < db) out[t.c + r + (int64_t)da * c] = acc[i][j];
    }
}

// ---------------------------------------------------------------------------
// k_y: one CTA per (Y matrix, 128-row tile); thread = row.  For each neutron
// density sub-block (Q_l, Q_r): Y[row, Q_l cols] = C[row, Q_r cols] rho^T.
template <typename T>
__global__ void __launch_bounds__(128) k_y(const YGroup *__restrict__ groups, const YBlk *__restrict__ blks,
                                           const T *__restrict__ x, const T *__restrict__ rho,
                                           T *__restrict__ Y, int max_nr, int max_nl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *rs = reinterpret_cast<T *>(smem_raw);          // [max_nl*max_nr]
  T *cs = rs + (size_t)max_nl * max_nr;             // [max_nr][128]
  const YGroup g = groups[blockIdx.x];
  const int row = g.row0 + threadIdx.x;
  const bool active = row < g.m;
  const T *C = x + g.c_base;
  T *Yg = Y + g.y_base;
  for (int bi = g.b_begin; bi < g.b_end; ++bi) {
    const YBlk b = blks[bi];
    const int n = b.nl * b.nr;
    for (int e = threadIdx.x; e < n; e += 128) rs[e] = rho[b.rho + e];
    if (active)
      for (int k = 0; k < b.nr; ++k) cs[k * 128 + threadIdx.x] = C[row + (int64_t)g.m * (b.ccol + k)];
    __syncthreads();
    if (active) {
      for (int l = 0; l < b.nl; ++l) {
        T acc = T(0);
        for (int k = 0; k < b.nr; ++k) acc = fma(cs[k * 128 + threadIdx.x], rs[l + b.nl * k], acc);
        Yg[row + (int64_t)g.m * (b.ycol + l)] = acc;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_a: one CTA per output tile (block, P_l, <=64 columns); 256 threads own the
// nl x ncols outputs (idx = tid + 256 q).  Per contribution: Z = sum w Y rows
// (mixing) in shared memory, then acc += rho_a Z.
constexpr int AQ = 16;  // outputs per thread: supports nl <= 64 with 64 columns
struct KaLayout {  // byte offsets of the k_a shared-memory arrays (16-byte aligned)
  size_t rs, zs, ws, ys, ls, total;
  __host__ __device__ static size_t al(size_t v) { return (v + 15) & ~size_t(15); }
  __host__ __device__ KaLayout(size_t es, int nl, int nr, int nm) {
    rs = 0;
    zs = al(rs + es * (size_t)nl * nr);
    ws = al(zs + es * (size_t)nr * 64);
    ys = al(ws + es * (size_t)nm);
    ls = al(ys + 8 * (size_t)nm);
    total = al(ls + 4 * (size_t)nm);
  }
};
template <typename T>
__global__ void __launch_bounds__(256) k_a(const ATile *__restrict__ tiles, const AContrib *__restrict__ contribs,
                                           const AMix *__restrict__ mixes, const T *__restrict__ wts,
                                           const T *__restrict__ rho, const T *__restrict__ Y, T *__restrict__ out,
                                           int max_nr, int max_nl, int max_mix) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  KaLayout L(sizeof(T), max_nl, max_nr, max_mix);
  T *rs = reinterpret_cast<T *>(smem_raw + L.rs);        // [max_nl*max_nr]
  T *zs = reinterpret_cast<T *>(smem_raw + L.zs);        // [max_nr][64]
  T *ws = reinterpret_cast<T *>(smem_raw + L.ws);        // [max_mix]
  int64_t *ys = reinterpret_cast<int64_t *>(smem_raw + L.ys);  // [max_mix]
  int *ls = reinterpret_cast<int *>(smem_raw + L.ls);    // [max_mix]
  const ATile t = tiles[blockIdx.x];
  const int nl = t.nl, ncols = t.ncols;
  T acc[AQ];
#pragma unroll
  for (int q = 0; q < AQ; ++q) acc[q] = T(0);
  for (int ci = t.c_begin; ci < t.c_end; ++ci) {
    const AContrib c = contribs[ci];
    const int nr = c.nr;
    const int nm = c.m_end - c.m_begin;
    for (int e = threadIdx.x; e < nl * nr; e += 256) rs[e] = rho[c.rho + e];
    for (int e = threadIdx.x; e < nm; e += 256) {
      const AMix m = mixes[c.m_begin + e];
      ws[e] = wts[m.wi];
      ys[e] = m.y;
      ls[e] = m.ld;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nr * ncols; e += 256) {
      const int k = e % nr, j = e / nr;
      T z = T(0);
      for (int m = 0; m < nm; ++m) z = fma(ws[m], Y[ys[m] + k + (int64_t)ls[m] * (t.col0 + j)], z);
      zs[k * 64 + j] = z;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < AQ; ++q) {
      const int idx = threadIdx.x + 256 * q;
      const int i = idx % nl, j = idx / nl;
      if (j < ncols) {
        T a = acc[q];
        for (int k = 0; k < nr; ++k) a = fma(rs[i + nl * k], zs[k * 64 + j], a);
        acc[q] = a;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < AQ; ++q) {
    const int idx = threadIdx.x + 256 * q;
    const int i = idx % nl, j = idx / nl;
    if (j < ncols) {
      T *o = out + t.out + i + (int64_t)t.ld * j;
      *o += acc[q];
    }
  }
}

__global__ void k_d2f(const double *__restrict__ a, float *__restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}
__global__ void k_f2d(const float *__restrict__ a, double *__restrict__ b, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (double)a[i];
}

// ---------------------------------------------------------------------------
template <typename T>
static T *dev_copy(const std::vector<double> &v) {
  T *p = nullptr;
  size_t n = std::max<size_t>(v.size(), 1);
  NSX_CUDA(cudaMalloc(&p, n * sizeof(T)));
  if (!v.empty()) {
    std::vector<T> tmp(v.begin(), v.end());
    NSX_CUDA(cudaMemcpy(p, tmp.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
  return p;
}
template <typename S>
static S *dev_copy_pod(const std::vector<S> &v) {
  S *p = nullptr;
  size_t n = std::max<size_t>(v.size(), 1);
  NSX_CUDA(cudaMalloc(&p, n * sizeof(S)));
  if (!v.empty()) NSX_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(S), cudaMemcpyHostToDevice));
  return p;
}

static size_t ky_smem(const nsx_handle *h, size_t es) {
  return es * ((size_t)h->max_ynl * h->max_ynr + (size_t)h->max_ynr * 128);
}
static size_t ka_smem(const nsx_handle *h, size_t es) {
  return KaLayout(es, h->max_anl, h->max_anr, h->max_mix).total;
}

void upload(nsx_handle *h) {
  NSX_CUDA(cudaSetDevice(h->device));
  if (h->max_anl > AQ * 256 / 64) fail(NSX_E_ARG, "proton partition with more than 64 J-states: not supported by k_a");
  auto &d = h->d;
  d.rhoA = dev_copy<double>(h->A.vals);
  d.rhoB = dev_copy<double>(h->B.vals);
  d.hA = dev_copy<double>(h->A.hdense);
  d.hB = dev_copy<double>(h->B.hdense);
  d.w = dev_copy<double>(h->weights);
  d.ygroups = dev_copy_pod(h->ygroups);
  d.yblks = dev_copy_pod(h->yblks);
  d.atiles = dev_copy_pod(h->atiles);
  d.acontribs = dev_copy_pod(h->acontribs);
  d.amixes = dev_copy_pod(h->amixes);
  d.ltiles = dev_copy_pod(h->ltiles);
  NSX_CUDA(cudaMalloc(&d.xin, h->no_state * sizeof(double)));
  NSX_CUDA(cudaMalloc(&d.xout, h->no_state * sizeof(double)));
  NSX_CUDA(cudaEventCreate(&h->ev0));
  NSX_CUDA(cudaEventCreate(&h->ev1));
  for (size_t es : {sizeof(double), sizeof(float)}) {
    if (ky_smem(h, es) > 227 * 1024 || ka_smem(h, es) > 227 * 1024)
      fail(NSX_E_ARG, "density sub-blocks too large for the shared-memory staging of k_y / k_a");
  }
  NSX_CUDA(cudaFuncSetAttribute(k_y<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ky_smem(h, 8)));
  NSX_CUDA(cudaFuncSetAttribute(k_a<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ka_smem(h, 8)));
  NSX_CUDA(cudaFuncSetAttribute(k_y<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ky_smem(h, 4)));
  NSX_CUDA(cudaFuncSetAttribute(k_a<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ka_smem(h, 4)));
}

void ensure_precision(nsx_handle *h, int precision) {
  auto &d = h->d;
  size_t ny = std::max<int64_t>(h->y_elems, 1);
  if (precision == NSX_FP64) {
    if (!d.y64) {
      NSX_CUDA(cudaMalloc(&d.y64, ny * sizeof(double)));
      NSX_CUDA(cudaMemset(d.y64, 0, ny * sizeof(double)));  // unreachable column slabs stay zero
    }
  } else if (precision == NSX_FP32) {
    if (!d.y32) {
      NSX_CUDA(cudaMalloc(&d.y32, ny * sizeof(float)));
      NSX_CUDA(cudaMemset(d.y32, 0, ny * sizeof(float)));
      d.rhoA32 = dev_copy<float>(h->A.vals);
      d.rhoB32 = dev_copy<float>(h->B.vals);
      d.hA32 = dev_copy<float>(h->A.hdense);
      d.hB32 = dev_copy<float>(h->B.hdense);
      d.w32 = dev_copy<float>(h->weights);
      NSX_CUDA(cudaMalloc(&d.x32, h->no_state * sizeof(float)));
      NSX_CUDA(cudaMalloc(&d.o32, h->no_state * sizeof(float)));
    }
  } else {
    fail(NSX_E_ARG, "unknown precision");
  }
}

// Brackets one stage launch with events when per-stage timing is enabled.
struct StageScope {
  nsx_handle *h;
  int stage;
  cudaStream_t s;
  cudaEvent_t a = nullptr, b = nullptr;
  StageScope(nsx_handle *h_, int st, cudaStream_t s_) : h(h_), stage(st), s(s_) {
    h->launches++;
    h->stage_launches[stage]++;
    if (h->timing) {
      NSX_CUDA(cudaEventCreate(&a));
      NSX_CUDA(cudaEventCreate(&b));
      NSX_CUDA(cudaEventRecord(a, s));
    }
  }
  ~StageScope() {
    if (h->timing) {
      cudaEventRecord(b, s);
      h->stage_events.push_back({stage, {a, b}});
    }
  }
};

void flush_stage_events(nsx_handle *h) {
  for (auto &e : h->stage_events) {
    float ms = 0;
    NSX_CUDA(cudaEventSynchronize(e.second.second));
    NSX_CUDA(cudaEventElapsedTime(&ms, e.second.first, e.second.second));
    h->stage_ms[e.first] += ms;
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  h->stage_events.clear();
}

// Algorithmic traffic (each operand read once, each result written once) and
// flops of one launch of each stage.
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[4], double flops[4]) {
  const double es = precision == NSX_FP64 ? 8.0 : 4.0;
  const double n = (double)h->no_state;
  double rhoA = (double)h->A.vals.size(), rhoB = (double)h->B.vals.size();
  double hd = (double)(h->A.hdense.size() + h->B.hdense.size());
  bytes[0] = es * (2.0 * n + hd);                               // C in, out written, dense H
  bytes[1] = es * (n + rhoB + (double)h->y_elems);              // C in, rho_B, Y written
  bytes[2] = es * ((double)h->y_elems + rhoA + 2.0 * n) + 4.0 * (double)h->weights.size();  // Y, rho_A, out r/w
  bytes[3] = precision == NSX_FP64 ? 0.0 : n * (8.0 + 4.0);     // one conversion launch
  flops[0] = h->flops_like;
  flops[1] = h->flops_y;
  flops[2] = h->flops_mix + h->flops_a;
  flops[3] = 0.0;
}

template <typename T>
static void run_stages(nsx_handle *h, const T *x, T *out, const T *rhoA, const T *rhoB, const T *hA, const T *hB,
                       const T *w, T *Y, cudaStream_t s) {
  auto &d = h->d;
  if (!h->ltiles.empty()) {
    StageScope sc(h, 0, s);
    k_like<T><<<(unsigned)h->ltiles.size(), 256, 0, s>>>(d.ltiles, x, out, hA, hB);
  }
  if (!h->ygroups.empty()) {
    StageScope sc(h, 1, s);
    k_y<T><<<(unsigned)h->ygroups.size(), 128, ky_smem(h, sizeof(T)), s>>>(d.ygroups, d.yblks, x, rhoB, Y,
                                                                             h->max_ynr, h->max_ynl);
  }
  if (!h->atiles.empty()) {
    StageScope sc(h, 2, s);
    k_a<T><<<(unsigned)h->atiles.size(), 256, ka_smem(h, sizeof(T)), s>>>(
        d.atiles, d.acontribs, d.amixes, w, rhoA, Y, out, h->max_anr, h->max_anl, h->max_mix);
  }
  NSX_CUDA(cudaGetLastError());
}

void matvec_device(nsx_handle *h, const double *x, double *y, int precision, cudaStream_t s) {
  ensure_precision(h, precision);
  auto &d = h->d;
  h->matvecs++;
  h->last_precision = precision;
  if (precision == NSX_FP64) {
    run_stages<double>(h, x, y, d.rhoA, d.rhoB, d.hA, d.hB, d.w, d.y64, s);
  } else {
    int64_t n = h->no_state;
    unsigned g = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    {
      StageScope sc(h, 3, s);
      k_d2f<<<g, 256, 0, s>>>(x, d.x32, n);
    }
    run_stages<float>(h, d.x32, d.o32, d.rhoA32, d.rhoB32, d.hA32, d.hB32, d.w32, d.y32, s);
    {
      StageScope sc(h, 3, s);
      k_f2d<<<g, 256, 0, s>>>(d.o32, y, n);
    }
    NSX_CUDA(cudaGetLastError());
  }
}

// The FP64 stages with a caller-provided Y buffer (used by the fixed-scratch entry point).
void matvec_fp64_with_scratch(nsx_handle *h, const double *x, double *y, double *Y, cudaStream_t s) {
  auto &d = h->d;
  h->matvecs++;
  h->last_precision = NSX_FP64;
  run_stages<double>(h, x, y, d.rhoA, d.rhoB, d.hA, d.hB, d.w, Y, s);
}

void release(nsx_handle *h) {
  auto &d = h->d;
  void *ptrs[] = {d.rhoA, d.rhoB, d.hA, d.hB, d.w, d.rhoA32, d.rhoB32, d.hA32, d.hB32, d.w32, d.ygroups, d.yblks,
                  d.atiles, d.acontribs, d.amixes, d.ltiles, d.y64, d.y32, d.x32, d.o32, d.xin, d.xout};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d = DeviceBuffers();
  for (auto &e : h->stage_events) {
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  h->stage_events.clear();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  h->ev0 = h->ev1 = nullptr;
}

}  // namespace nsx
