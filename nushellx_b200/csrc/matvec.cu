// H.v on the GPU for the pn-factorised J-scheme Hamiltonian.
//
// The reference computes the product as multiplyx (pn), multiplya (pp) and
// multiplyb (nn) in src/NuLnz/NuCoreX.f90:76-226 with axpy loops over density
// sub-blocks (src/NuCommonX/NuCommonX.f90:745-919, 1009-1104).  Here it is
// two stream-ordered kernels; every output element is owned by one CTA (no
// global atomics, no per-thread copies of the vector):
//
//   k_like : out_b  = H_pp(Ja) C_b + C_b H_nn(Jb)              (dense tiled GEMM)
//   k_pn   : persistent; a CTA owns the output columns of one neutron partition
//            Q_l (a chunk of CH states) of one block and, for every (J_ar, lam)
//            group of the pn table,
//            in batches of at most 64 (FP32) / 32 (FP64) proton rows:
//              stage 1: Y_(h,b)[batch rows, chunk] = C_h[rows, Q_r cols] rho_b[chunk, Q_r]^T
//                       straight into shared memory (Y never leaves the SM);
//              stage 2: per proton partition P_r (32/CH rows per warp item, one
//                       element per lane) the sources are mixed in registers,
//                       Z_a = sum w_(a,s) Y_s, and out[P_l rows] += rho_a[P_l, P_r] Z_a
//                       is accumulated in shared memory.
//            Each Y_(h,b) element is computed once (the reference recomputes the
//            neutron-side product for every proton operator).
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
// k_pn: see the file comment.  512 threads (16 warps), one CTA per SM.
//   shared Y batch layout: ybuf[p][row - batch row0][c] with odd row stride CH + 1
//   stage-2 lane map: column c = lane % CH, row lane / CH (32 / CH rows per item)
constexpr int PN_WARPS = 16;
struct PnLayout {  // byte offsets of the k_pn shared-memory arrays (16-byte aligned)
  size_t out, z, w, src, y, total;
  __host__ __device__ static size_t al(size_t v) { return (v + 15) & ~size_t(15); }
  __host__ __device__ static int ldo(int dal) { return dal | 1; }  // odd: conflict-free column stride
  __host__ __device__ PnLayout(size_t es, int max_dal, int ch, int batch_rows) {
    out = 0;
    z = al(out + es * (size_t)ldo(max_dal) * ch);
    w = al(z + es * (size_t)PN_WARPS * MAXA * 32);
    src = al(w + es * (size_t)MAXA * MAXS);
    y = al(src + sizeof(int) * 2 * (size_t)MAXS);
    total = al(y + es * (size_t)MAXS * batch_rows * (ch + 1));
  }
};

// Stage-2 mixing of one lane's element: z_a = sum_p W[a][p] y_p for the item's
// operators, y_p read once into registers (NP = 16 or 32 sources, zero-padded).
template <typename T, int NP>
__device__ __forceinline__ void pn_mix(const T *Yc, int pstride, int np, const uint32_t *cov, int lc, bool ok,
                                       const T *ws, int my_wrow, int na, T *zrow) {
  T y[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) y[p] = (ok && p < np && ((cov[p] >> lc) & 1u)) ? Yc[p * pstride] : T(0);
  for (int ai = 0; ai < na; ++ai) {
    const T *wr = ws + __shfl_sync(0xffffffffu, my_wrow, ai) * MAXS;
    T zz = T(0);
#pragma unroll
    for (int p = 0; p < NP; ++p) zz = fma(wr[p], y[p], zz);
    zrow[ai * 32] = zz;
  }
}

template <typename T, int CH>
__global__ void __launch_bounds__(512, 1)
    k_pn(const PnTask *__restrict__ tasks, int ntasks, const TGroup *__restrict__ tgroups,
         const Group *__restrict__ groups, const TSrc *__restrict__ tsrcs, const Piece *__restrict__ pieces,
         const PrWork *__restrict__ prwork, const Batch *__restrict__ batches, const AOp *__restrict__ aops,
         const T *__restrict__ W, const T *__restrict__ x, const T *__restrict__ rhoA, const T *__restrict__ rhoB,
         T *__restrict__ out, int *__restrict__ counter, int max_dal, int batch_rows,
         unsigned long long *__restrict__ cycles) {
  constexpr int IR = 32 / CH;              // rows per work item: one (row, column) element per lane
  constexpr int CHP = CH + 1;              // padded row stride of the Y batch (odd)
  extern __shared__ __align__(16) unsigned char smem[];
  const PnLayout L(sizeof(T), max_dal, CH, batch_rows);
  T *out_s = reinterpret_cast<T *>(smem + L.out);   // [CH][ldo] : out_s[row + ldo*c]
  T *zs = reinterpret_cast<T *>(smem + L.z);        // [warp][MAXA][32 lanes]
  T *ws = reinterpret_cast<T *>(smem + L.w);        // [MAXA][MAXS] weights of the present sources (0-padded)
  int *sidx_s = reinterpret_cast<int *>(smem + L.src);            // [MAXS]
  uint32_t *cov_s = reinterpret_cast<uint32_t *>(sidx_s + MAXS);  // [MAXS]
  T *ybuf = reinterpret_cast<T *>(smem + L.y);      // [p][batch row][CHP]
  const int pstride = batch_rows * CHP;
  __shared__ int s_task;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int lc = lane % CH, lrow = lane / CH;
  unsigned long long cyc[4] = {0, 0, 0, 0};
  long long t0 = clock64();
  auto mark = [&](int k) {
    if (cycles && threadIdx.x == 0) {
      long long t1 = clock64();
      cyc[k] += (unsigned long long)(t1 - t0);
      t0 = t1;
    }
  };
  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(counter, 1);
    __syncthreads();
    const int ti = s_task;
    __syncthreads();
    if (ti >= ntasks) break;
    const PnTask t = tasks[ti];
    const int dal = t.d_al, nq = t.nq, ldo = PnLayout::ldo(dal);
    for (int e = threadIdx.x; e < ldo * CH; e += blockDim.x) out_s[e] = T(0);
    for (int gi = t.g_begin; gi < t.g_end; ++gi) {
      const TGroup tg = tgroups[gi];
      const Group G = groups[tg.grp];
      const int np = tg.src_end - tg.src_begin;
      const int dar = G.d_ar;
      for (int e = threadIdx.x; e < MAXS; e += blockDim.x) {
        if (e < np) {
          const TSrc src = tsrcs[tg.src_begin + e];
          sidx_s[e] = src.sidx;
          cov_s[e] = src.cover;
        } else {
          sidx_s[e] = 0;
          cov_s[e] = 0u;
        }
      }
      __syncthreads();
      for (int e = threadIdx.x; e < G.na * MAXS; e += blockDim.x) {
        const int a = e / MAXS, p = e - a * MAXS;
        ws[e] = p < np ? W[G.w_off + a * G.nsrc + sidx_s[p]] : T(0);
      }
      mark(1);
      for (int bi = G.bt_begin; bi < G.bt_end; ++bi) {
        const Batch bt = batches[bi];
        // ---- stage 1: Y_p[row][c] for the batch rows, into shared memory ----
        for (int e = threadIdx.x; e < np * bt.nrows; e += blockDim.x) {
          const int p = e / bt.nrows, rr = e - p * bt.nrows;
          const int r = bt.row0 + rr;
          const TSrc src = tsrcs[tg.src_begin + p];
          T *Yr = ybuf + p * pstride + rr * CHP;
          for (int pi = src.piece_begin; pi < src.piece_end; ++pi) {
            const Piece pc = pieces[pi];
            const T *C = x + pc.c + r;
            for (int j0 = 0; j0 < pc.w; j0 += 4) {
              T acc[4] = {T(0), T(0), T(0), T(0)};
              const T *R = rhoB + pc.rho + j0;
              for (int k0 = 0; k0 < pc.nr; k0 += 8) {
                T ck[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) ck[k] = (k0 + k < pc.nr) ? C[(int64_t)dar * (k0 + k)] : T(0);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                  if (k0 + k < pc.nr) {
                    const T *Rk = R + (int64_t)pc.ld * (k0 + k);
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                      if (j0 + q < pc.w) acc[q] = fma(ck[k], __ldg(Rk + q), acc[q]);
                  }
                }
              }
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (j0 + q < pc.w) Yr[pc.cs + j0 + q] = acc[q];
            }
          }
        }
        __syncthreads();
        mark(0);
        // ---- stage 2: warp items (P_r, <= IR rows); lane = (row lrow, column lc) ----
        for (int it = bt.it_begin + warp; it < bt.it_end; it += PN_WARPS) {
          const PrWork pw = prwork[it];
          const int na = pw.a_end - pw.a_begin;
          AOp my_op = {0, 0, 0, 0, 0};
          if (lane < na) my_op = aops[pw.a_begin + lane];
          T *z = zs + (size_t)warp * (MAXA * 32);
          const bool ok = lrow < pw.nr;
          const T *Yc = ybuf + (pw.row0 - bt.row0 + (ok ? lrow : 0)) * CHP + lc;
          if (np <= 16)
            pn_mix<T, 16>(Yc, pstride, np, cov_s, lc, ok, ws, my_op.wrow, na, z + lane);
          else
            pn_mix<T, 32>(Yc, pstride, np, cov_s, lc, ok, ws, my_op.wrow, na, z + lane);
          __syncwarp();
          for (int ai = 0; ai < na; ++ai) {
            const int64_t a_rho = __shfl_sync(0xffffffffu, my_op.rho, ai);
            const int a_ld = __shfl_sync(0xffffffffu, my_op.ld, ai);
            const int a_row0 = __shfl_sync(0xffffffffu, my_op.out_row0, ai);
            const int a_nl = __shfl_sync(0xffffffffu, my_op.nl, ai);
            const T *zr = z + ai * 32 + lc;  // z of (row r, column lc) sits at lane r*CH + lc
            if (lc < nq) {
              for (int l = lrow; l < a_nl; l += IR) {
                const T *ra = rhoA + a_rho + l;
                T rv[IR];
#pragma unroll
                for (int r = 0; r < IR; ++r) rv[r] = r < pw.nr ? __ldg(ra + (int64_t)a_ld * r) : T(0);
                T v = T(0);
#pragma unroll
                for (int r = 0; r < IR; ++r)
                  if (r < pw.nr) v = fma(rv[r], zr[r * CH], v);
                atomicAdd(out_s + (a_row0 + l) + ldo * lc, v);
              }
            }
          }
          __syncwarp();
        }
        __syncthreads();  // ybuf is rewritten by the next batch; ws/sidx/cov by the next group
        mark(2);
      }
    }
    for (int e = threadIdx.x; e < dal * nq; e += blockDim.x) {
      const int r = e % dal, c = e / dal;
      out[t.out + r + (int64_t)dal * c] += out_s[r + ldo * c];
    }
    __syncthreads();
    mark(3);
  }
  if (cycles && threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) atomicAdd(cycles + k, cyc[k]);
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

static size_t pn_smem(const PnPlan &P, size_t es) { return PnLayout(es, P.max_dal, P.CH, P.batch_rows).total; }

template <typename T>
static void upload_pn(nsx_handle *h, const PnPlan &P, PnDevice &D) {
  D.groups = dev_copy_pod(P.groups);
  D.tgroups = dev_copy_pod(P.tgroups);
  D.tsrcs = dev_copy_pod(P.tsrcs);
  D.pieces = dev_copy_pod(P.pieces);
  D.prwork = dev_copy_pod(P.prwork);
  D.batches = dev_copy_pod(P.batches);
  D.aops = dev_copy_pod(P.aops);
  D.tasks = dev_copy_pod(P.tasks);
  D.weights = dev_copy<T>(P.weights);
  int sms = 0;
  NSX_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  D.grid = std::max(1, std::min<int>(sms, (int)P.tasks.size()));
  NSX_CUDA(cudaMalloc(&D.counter, sizeof(int)));
  NSX_CUDA(cudaMalloc(&D.cycles, 4 * sizeof(unsigned long long)));
  NSX_CUDA(cudaMemset(D.cycles, 0, 4 * sizeof(unsigned long long)));
  D.smem = pn_smem(P, sizeof(T));
  if (D.smem > 227 * 1024) fail(NSX_E_ARG, "k_pn shared-memory layout exceeds 227 KB (output block too tall)");
}

void upload(nsx_handle *h) {
  NSX_CUDA(cudaSetDevice(h->device));
  auto &d = h->d;
  for (const PnPlan *P : {&h->pn64, &h->pn32}) {
    for (const Group &g : P->groups)
      if (g.na > MAXA || g.nsrc > MAXS) fail(NSX_E_ARG, "pn group exceeds the k_pn operator/source limits");
  }
  d.rhoA = dev_copy<double>(h->A.vals);
  d.rhoB = dev_copy<double>(h->B.vals);
  d.hA = dev_copy<double>(h->A.hdense);
  d.hB = dev_copy<double>(h->B.hdense);
  d.ltiles = dev_copy_pod(h->ltiles);
  upload_pn<double>(h, h->pn64, d.pn64);
  NSX_CUDA(cudaMalloc(&d.xin, h->no_state * sizeof(double)));
  NSX_CUDA(cudaMalloc(&d.xout, h->no_state * sizeof(double)));
  NSX_CUDA(cudaEventCreate(&h->ev0));
  NSX_CUDA(cudaEventCreate(&h->ev1));
  NSX_CUDA(cudaFuncSetAttribute(k_pn<double, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.pn64.smem));
}

void ensure_precision(nsx_handle *h, int precision) {
  auto &d = h->d;
  if (precision == NSX_FP64) return;
  if (precision != NSX_FP32) fail(NSX_E_ARG, "unknown precision");
  if (d.x32) return;
  d.rhoA32 = dev_copy<float>(h->A.vals);
  d.rhoB32 = dev_copy<float>(h->B.vals);
  d.hA32 = dev_copy<float>(h->A.hdense);
  d.hB32 = dev_copy<float>(h->B.hdense);
  upload_pn<float>(h, h->pn32, d.pn32);
  NSX_CUDA(cudaFuncSetAttribute(k_pn<float, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)d.pn32.smem));
  NSX_CUDA(cudaMalloc(&d.x32, h->no_state * sizeof(float)));
  NSX_CUDA(cudaMalloc(&d.o32, h->no_state * sizeof(float)));
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
// flops of one launch of each stage.  k_pn keeps its Y operands on chip/L2, so
// its algorithmic bytes are the input vector, both density sets and the output.
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[4], double flops[4]) {
  const double es = precision == NSX_FP64 ? 8.0 : 4.0;
  const double n = (double)h->no_state;
  double rhoA = (double)h->A.vals.size(), rhoB = (double)h->B.vals.size();
  double hd = (double)(h->A.hdense.size() + h->B.hdense.size());
  const PnPlan &P = precision == NSX_FP64 ? h->pn64 : h->pn32;
  bytes[0] = es * (2.0 * n + hd);
  bytes[1] = es * (3.0 * n + rhoA + rhoB + (double)P.weights.size());
  bytes[2] = 0.0;
  bytes[3] = precision == NSX_FP64 ? 0.0 : n * (8.0 + 4.0);
  flops[0] = h->flops_like;
  flops[1] = h->flops_y + h->flops_mix + h->flops_a;
  flops[2] = 0.0;
  flops[3] = 0.0;
}

template <typename T, int CH>
static void run_stages(nsx_handle *h, const T *x, T *out, const T *rhoA, const T *rhoB, const T *hA, const T *hB,
                       const PnPlan &P, const PnDevice &D, cudaStream_t s) {
  auto &d = h->d;
  if (!h->ltiles.empty()) {
    StageScope sc(h, 0, s);
    k_like<T><<<(unsigned)h->ltiles.size(), 256, 0, s>>>(d.ltiles, x, out, hA, hB);
  }
  if (!P.tasks.empty()) {
    NSX_CUDA(cudaMemsetAsync(D.counter, 0, sizeof(int), s));
    StageScope sc(h, 1, s);
    k_pn<T, CH><<<D.grid, 512, D.smem, s>>>(D.tasks, (int)P.tasks.size(), D.tgroups, D.groups, D.tsrcs, D.pieces,
                                            D.prwork, D.batches, D.aops, (const T *)D.weights, x, rhoA, rhoB, out,
                                            D.counter, P.max_dal, P.batch_rows, h->timing ? D.cycles : nullptr);
  }
  NSX_CUDA(cudaGetLastError());
}

void matvec_device(nsx_handle *h, const double *x, double *y, int precision, cudaStream_t s) {
  ensure_precision(h, precision);
  auto &d = h->d;
  h->matvecs++;
  h->last_precision = precision;
  if (precision == NSX_FP64) {
    run_stages<double, 8>(h, x, y, d.rhoA, d.rhoB, d.hA, d.hB, h->pn64, d.pn64, s);
  } else {
    int64_t n = h->no_state;
    unsigned g = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    {
      StageScope sc(h, 3, s);
      k_d2f<<<g, 256, 0, s>>>(x, d.x32, n);
    }
    run_stages<float, 16>(h, d.x32, d.o32, d.rhoA32, d.rhoB32, d.hA32, d.hB32, h->pn32, d.pn32, s);
    {
      StageScope sc(h, 3, s);
      k_f2d<<<g, 256, 0, s>>>(d.o32, y, n);
    }
    NSX_CUDA(cudaGetLastError());
  }
}

static void free_pn(PnDevice &D) {
  void *ptrs[] = {D.groups, D.tgroups, D.tsrcs, D.pieces, D.prwork, D.batches, D.aops, D.tasks, D.weights,
                  D.counter, D.cycles};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  D = PnDevice();
}

void release(nsx_handle *h) {
  auto &d = h->d;
  void *ptrs[] = {d.rhoA, d.rhoB, d.hA, d.hB, d.rhoA32, d.rhoB32, d.hA32, d.hB32, d.ltiles,
                  d.x32, d.o32, d.xin, d.xout};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  free_pn(d.pn64);
  free_pn(d.pn32);
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
