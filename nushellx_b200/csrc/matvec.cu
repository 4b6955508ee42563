// H.v on the GPU for the pn-factorised J-scheme Hamiltonian.
//
// The reference computes the product as multiplyx (pn), multiplya (pp) and
// multiplyb (nn) in src/NuLnz/NuCoreX.f90:76-226 with axpy loops over density
// sub-blocks (src/NuCommonX/NuCommonX.f90:745-919, 1009-1104).  Here it is
// four stream-ordered kernels, with no per-thread copies of the vector:
//
//   k_like : out_b = H_pp(Ja) C_b + C_b H_nn(Jb)                  (dense tiled GEMM)
//   k_y    : Y_(h,k) = C_h rho_k^T for every (input block h, neutron density k)
//            the pn table uses -- once, where the reference recomputes it for
//            every proton operator; row-major d_ar x d_bl.  FP32 pieces on the
//            tensor cores (mma.sync TF32 with the 3xTF32 split), FP64 SIMT
//   k_z    : Z_a[P_r rows] = sum_s w_(a,s) Y_s[P_r rows] for the proton operators
//            of each (output block, J_ar, lam) group, written as rows of the
//            stacked operand Zbar of the output slab (block, P_l) a leads to
//   k_a    : out[P_l rows] += Abar Zbar, Abar = the slab's proton density blocks
//            side by side: one long-K product per output slab, streamed through
//            a cp.async shared-memory pipeline; slabs longer than 512 stacked rows
//            are split and their partial sums added atomically
//
// Each intermediate (Y, Zbar) is written once and read once, in row streams.
// Templated on the contraction type: double (the FP64 form) or float (the FP32
// form, FP64 vectors converted at the boundary).
#include <type_traits>
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
// k_y: one CTA per (Y matrix, 256-row tile); FP64: thread = rows t and t + 128;
// FP32: warp w = rows 64w .. 64w + 63 on the tensor cores (ky_piece_tc below).
// The tile's part of Y (256 consecutive rows of a row-major matrix) is produced
// in column windows of at most 128 bytes (32 FP32 / 16 FP64 columns).  A window
// holds whole neutron density sub-blocks (Q_l, Q_r); a sub-block wider than the
// window is cut at multiples of 8 outputs.  For each piece and each group of 8
// outputs the thread accumulates
//   Y[row, Q_l cols] = C[row, Q_r cols] rho^T
// over all nr coefficients in registers (C loads coalesced across the warp,
// density values as warp-uniform 16-byte loads: 16 FMAs per 2 C values and 8
// coefficients) and stores the result once into a padded shared-memory tile.  The
// window is then written out as coalesced row segments, columns no sub-block
// reaches as zeros, and cleared.  Every element of Y is written, so Y needs no
// clearing between products.  A warp whose second (or both) 32-row slots lie past
// the end of the matrix takes the one-row path (or only joins the barriers).
template <typename T> struct KyWin;
template <> struct KyWin<float> { static constexpr int W = 32; };
template <> struct KyWin<double> { static constexpr int W = 16; };

__device__ __forceinline__ void ky_load8(const float *p, float v[8]) {
  const float4 a = __ldg(reinterpret_cast<const float4 *>(p));
  const float4 b = __ldg(reinterpret_cast<const float4 *>(p) + 1);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
}
__device__ __forceinline__ void ky_load8(const double *p, double v[8]) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p) + i);
    v[2 * i] = a.x;
    v[2 * i + 1] = a.y;
  }
}

// Outputs l in [plo, phi) of one sub-block (plo a multiple of 8) for R rows of the
// thread: c0 points at C[row, Q_r col 0] of the first row; rows are 128 apart in C
// and 128 tile rows apart in t (t points at the tile column of output 0).
template <typename T, int R>
__device__ __forceinline__ void ky_piece(const T *__restrict__ c0, bool ok0, bool ok1, int64_t m,
                                         const T *__restrict__ rb, int ldr, int nr, int plo, int phi, T *t,
                                         int tstride) {
  for (int g = plo; g < phi; g += 8) {
    T a[R][8];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int q = 0; q < 8; ++q) a[r][q] = T(0);
    const T *cp = c0;
    const T *rp = rb + g;
#pragma unroll 2
    for (int k = 0; k < nr; ++k) {
      T c[R];
      c[0] = ok0 ? cp[0] : T(0);
      if (R == 2) c[R - 1] = ok1 ? cp[128] : T(0);
      T v[8];
      ky_load8(rp, v);
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int r = 0; r < R; ++r) a[r][q] = fma(c[r], v[q], a[r][q]);
      cp += m;
      rp += ldr;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (g + q < phi) {
#pragma unroll
        for (int r = 0; r < R; ++r) t[r * tstride + g + q] = a[r][q];
      }
  }
}

// FP32 pieces on the tensor cores: mma.sync m16n8k8 TF32 with the 3xTF32 split
// (x = big + small, both TF32; big*big + big*small + small*big accumulated in FP32),
// which keeps FP32 accuracy.  Fragment layouts (PTX ISA, m16n8k8 .tf32), with
// g = lane / 4 and q = lane % 4:  A (16 x 8, row-major) a0 = (g, q), a1 = (g+8, q),
// a2 = (g, q+4), a3 = (g+8, q+4);  B (8 x 8, column-major) b0 = (k q, n g),
// b1 = (k q+4, n g);  D (16 x 8) d0 = (g, 2q), d1 = (g, 2q+1), d2 = (g+8, 2q),
// d3 = (g+8, 2q+1).
__device__ __forceinline__ uint32_t ky_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void ky_split(float x, uint32_t &big, uint32_t &small) {
  big = ky_tf32(x);
  small = ky_tf32(x - __uint_as_float(big));
}
__device__ __forceinline__ void ky_mma(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
               "{%0,%1,%2,%3};\n"
               : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
               : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Rows [wr0, wr0 + 32) of the tile (two m16 tiles) for outputs l in [plo, phi)
// (plo a multiple of 8, NT = ceil((phi - plo) / 8) n8 tiles) of one sub-block:
// C points at C_h[row0 of the tile, Q_r col 0]; tcol at the tile column of output 0.
template <int NT>
__device__ __forceinline__ void ky_piece_tc(const float *__restrict__ C, int64_t m, int rows, int wr0, int nr,
                                            const float *__restrict__ rb, int ldr, int plo, int phi, float *tcol,
                                            int ld) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  float acc[2][NT][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int i = 0; i < 4; ++i) acc[mt][nt][i] = 0.f;
  const float *cr[2][2];
  bool rok[2][2];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = wr0 + 16 * mt + g + 8 * h;
      rok[mt][h] = r < rows;
      cr[mt][h] = C + r;
    }
  for (int k0 = 0; k0 < nr; k0 += 8) {
    const int ka = k0 + q, kb = k0 + q + 4;
    const bool kaok = ka < nr, kbok = kb < nr;
    uint32_t abig[2][4], asml[2][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const float v0 = (rok[mt][0] && kaok) ? cr[mt][0][m * ka] : 0.f;
      const float v1 = (rok[mt][1] && kaok) ? cr[mt][1][m * ka] : 0.f;
      const float v2 = (rok[mt][0] && kbok) ? cr[mt][0][m * kb] : 0.f;
      const float v3 = (rok[mt][1] && kbok) ? cr[mt][1][m * kb] : 0.f;
      ky_split(v0, abig[mt][0], asml[mt][0]);
      ky_split(v1, abig[mt][1], asml[mt][1]);
      ky_split(v2, abig[mt][2], asml[mt][2]);
      ky_split(v3, abig[mt][3], asml[mt][3]);
    }
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int l = plo + 8 * nt + g;
      const float w0 = kaok ? __ldg(rb + l + (int64_t)ldr * ka) : 0.f;
      const float w1 = kbok ? __ldg(rb + l + (int64_t)ldr * kb) : 0.f;
      uint32_t b0, b0s, b1, b1s;
      ky_split(w0, b0, b0s);
      ky_split(w1, b1, b1s);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        ky_mma(acc[mt][nt], asml[mt], b0, b1);
        ky_mma(acc[mt][nt], abig[mt], b0s, b1s);
        ky_mma(acc[mt][nt], abig[mt], b0, b1);
      }
    }
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int l = plo + 8 * nt + 2 * q;
      float *t0 = tcol + (wr0 + 16 * mt + g) * ld;
      float *t1 = t0 + 8 * ld;
      if (l < phi) {
        t0[l] = acc[mt][nt][0];
        t1[l] = acc[mt][nt][2];
      }
      if (l + 1 < phi) {
        t0[l + 1] = acc[mt][nt][1];
        t1[l + 1] = acc[mt][nt][3];
      }
    }
}

__device__ __forceinline__ void ky_piece_tc_any(const float *C, int64_t m, int rows, int wr0, int nr,
                                                const float *rb, int ldr, int plo, int phi, float *tcol, int ld) {
  switch ((phi - plo + 7) >> 3) {
    case 1: ky_piece_tc<1>(C, m, rows, wr0, nr, rb, ldr, plo, phi, tcol, ld); break;
    case 2: ky_piece_tc<2>(C, m, rows, wr0, nr, rb, ldr, plo, phi, tcol, ld); break;
    case 3: ky_piece_tc<3>(C, m, rows, wr0, nr, rb, ldr, plo, phi, tcol, ld); break;
    default: ky_piece_tc<4>(C, m, rows, wr0, nr, rb, ldr, plo, phi, tcol, ld); break;
  }
}

constexpr int KY_SIMT_MAX = 8;    // FP32 k_y: largest piece (outputs, coefficients) taken as SIMT FMAs

template <typename T>
__global__ void __launch_bounds__(128) k_y(const YGroup *__restrict__ groups, const YBlk *__restrict__ blks,
                                           const T *__restrict__ x, const T *__restrict__ rho, T *__restrict__ Y) {
  constexpr int W = KyWin<T>::W;
  constexpr int LD = W + 1;
  __shared__ T tile[KY_TILE_ROWS * LD];
  const YGroup g = groups[blockIdx.x];
  const int tid = threadIdx.x;
  const int rows = min(KY_TILE_ROWS, g.m - g.row0);
  const int wrow = tid & ~31;                 // first tile row of the warp's first slot
  const int mode = (wrow + 128 < rows) ? 2 : (wrow < rows ? 1 : 0);
  const bool ok0 = tid < rows, ok1 = tid + 128 < rows;
  const int64_t m = g.m;
  const T *C = x + g.c_base + g.row0 + tid;
  for (int e = tid; e < KY_TILE_ROWS * LD; e += 128) tile[e] = T(0);
  __syncthreads();
  T *Yt = Y + g.y_base + (int64_t)g.row0 * g.ldy;
  const int fc = tid % W;                     // flush: column of this thread, rows fr, fr + 128/W, ...
  int bi = g.b_begin, lst = 0;                // next sub-block and its first output not yet produced
  int ws = 0;
  while (ws < g.ldy) {
    int we = min(ws + W, g.ldy);
    int nbi = g.b_end, nlst = 0;
    for (int j = bi, l0 = lst; j < g.b_end; ++j, l0 = 0) {
      const YBlk b = blks[j];
      const int bs = b.ycol + l0;
      if (bs >= we) { nbi = j; nlst = l0; break; }
      int hi = b.nl;
      if (b.ycol + b.nl > we) {
        if (l0 == 0 && b.ycol > ws) { we = b.ycol; nbi = j; nlst = 0; break; }  // next window starts here
        hi = l0 + (we - bs);                                                     // cut: a multiple of 8
        nbi = j;
        nlst = hi;
      }
      // FP32: pieces of more than KY_SIMT_MAX outputs or coefficients on the tensor cores; small
      // ones (padded to m16n8k8 tiles they would waste most of the MMA work) as SIMT FMAs
      if (std::is_same<T, float>::value && (hi - l0 > KY_SIMT_MAX || b.nr > KY_SIMT_MAX)) {
        if constexpr (std::is_same<T, float>::value) {
          // tensor cores: warp w owns tile rows [64w, 64w + 64) in two halves of 32
          const float *Cb = x + g.c_base + g.row0 + m * b.ccol;
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int wr0 = 64 * (tid >> 5) + 32 * half;
            if (wr0 < rows) ky_piece_tc_any(Cb, m, rows, wr0, b.nr, rho + b.rho, b.ldr, l0, hi, tile + (b.ycol - ws), LD);
          }
        }
      } else {
        T *t = tile + tid * LD + (b.ycol - ws);
        const T *c0 = C + m * b.ccol;
        if (mode == 2) ky_piece<T, 2>(c0, ok0, ok1, m, rho + b.rho, b.ldr, b.nr, l0, hi, t, 128 * LD);
        else if (mode == 1) ky_piece<T, 1>(c0, ok0, ok1, m, rho + b.rho, b.ldr, b.nr, l0, hi, t, 128 * LD);
      }
      if (hi < b.nl) break;
    }
    __syncthreads();
    const int wn = we - ws;
    T *yp = Yt + ws + fc;
    for (int r = tid / W; r < rows; r += 128 / W) {
      T *tp = tile + r * LD + fc;
      if (fc < wn) __stcs(yp + (int64_t)r * g.ldy, *tp);   // streaming: keep C and rho_B in L2
      *tp = T(0);
    }
    __syncthreads();
    ws = we;
    bi = nbi;
    lst = nlst;
  }
}

// ---------------------------------------------------------------------------
// k_z: one CTA per (group, P_r, 128-column tile); thread = column.  For each row
// of P_r the group's sources are read once into registers (NS of them at most: 16,
// or ZMAXS when the plan has a larger group) and every operator's mixed row is
// written to its Zbar slab.
// TC: the FP32 tensor-core form, Zbar tiles in the MMA's swizzled layout (a row of 128 tile
// columns is 4 contiguous 128-byte lines, so a warp's store is still one full line).
template <typename T, int NS, bool TC>
__device__ __forceinline__ void kz_store(T *__restrict__ Zb, const int64_t *zdst, const int *zk, const ZUnit &u, int a,
                                         int rr, int c, int col, T z) {
  // streaming stores: Zbar is read once, by the proton side, long after
  if constexpr (TC) __stcs(Zb + zdst[a] + umma::ztile_index(zk[a] + rr, c), z);
  else __stcs(Zb + zdst[a] + (int64_t)rr * u.ldz + col, z);
}

// Rows are taken two at a time (with 16 sources): both rows' loads are in flight together and
// every weight read from shared memory serves two FMAs.
template <typename T, int NS, bool TC>
__device__ __forceinline__ void kz_body(const ZUnit &u, const T (*ws)[ZMAXS], const int64_t *ysrc, const int64_t *zdst,
                                        const int *zk, int ns, int na, const T *__restrict__ Y, T *__restrict__ Zb) {
  const int c = threadIdx.x;
  if (c >= u.ncols) return;
  const int col = u.c0 + c;
  constexpr int RB = NS <= 16 ? 2 : 1;
  for (int rr = 0; rr < u.nr; rr += RB) {
    const bool two = RB == 2 && rr + 1 < u.nr;
    const int64_t roff = (int64_t)(u.row0 + rr) * u.d_bl + col;
    T y[RB][NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      y[0][s] = s < ns ? Y[ysrc[s] + roff] : T(0);
      if constexpr (RB == 2) y[1][s] = (s < ns && two) ? Y[ysrc[s] + roff + u.d_bl] : T(0);
    }
    for (int a = 0; a < na; ++a) {
      T z0 = T(0), z1 = T(0);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const T wv = ws[a][s];
        z0 = fma(wv, y[0][s], z0);
        if constexpr (RB == 2) z1 = fma(wv, y[RB - 1][s], z1);
      }
      kz_store<T, NS, TC>(Zb, zdst, zk, u, a, rr, c, col, z0);
      if (two) kz_store<T, NS, TC>(Zb, zdst, zk, u, a, rr + 1, c, col, z1);
    }
  }
}

template <typename T, int NS, bool TC>
__global__ void __launch_bounds__(128) k_z(const ZUnit *__restrict__ units, const int32_t *__restrict__ cta_units,
                                           const ZGroup *__restrict__ groups, const ZSrc *__restrict__ srcs,
                                           const ZOp *__restrict__ ops, const ZOpTC *__restrict__ ops_tc,
                                           const T *__restrict__ W, const T *__restrict__ Y, T *__restrict__ Zb) {
  __shared__ T ws[ZMAXA][ZMAXS];
  __shared__ int64_t ysrc[ZMAXS];
  __shared__ int64_t zdst[ZMAXA], zbase[ZMAXA];
  __shared__ int zk[ZMAXA], zkg[ZMAXA];
  // the CTA's units: consecutive column tiles of one (group, P_r) with the same operators
  const int ub = cta_units[blockIdx.x], ue = cta_units[blockIdx.x + 1];
  const ZUnit u0 = units[ub];
  const ZGroup G = groups[u0.grp];
  const int na = u0.op_end - u0.op_begin;
  for (int e = threadIdx.x; e < na * ZMAXS; e += blockDim.x) {
    const int a = e / ZMAXS, s = e - a * ZMAXS;
    ws[a][s] = s < G.ns ? W[G.w_off + ops[u0.op_begin + a].wrow * G.ns + s] : T(0);
  }
  for (int e = threadIdx.x; e < na; e += blockDim.x) {
    if constexpr (TC) {
      const ZOpTC o = ops_tc[u0.op_begin + e];
      zbase[e] = o.base;
      zkg[e] = o.kgroups;
      zk[e] = o.kofs;
    } else {
      zdst[e] = ops[u0.op_begin + e].z;
      zk[e] = 0;
    }
  }
  for (int e = threadIdx.x; e < ZMAXS; e += blockDim.x) ysrc[e] = e < G.ns ? srcs[G.s_begin + e].y : 0;
  for (int ui = ub; ui < ue; ++ui) {
    const ZUnit u = ui == ub ? u0 : units[ui];
    __syncthreads();   // set-up done; the previous unit's destinations no longer read
    if constexpr (TC) {   // the unit's column tile of each operator's Zbar tiles
      for (int e = threadIdx.x; e < na; e += blockDim.x) zdst[e] = zbase[e] + (int64_t)(u.c0 / 128) * zkg[e] * 1024;
      __syncthreads();
    }
    kz_body<T, NS, TC>(u, ws, ysrc, zdst, zk, G.ns, na, Y, Zb);
  }
}

// ---------------------------------------------------------------------------
// k_yz (FP32 form): the neutron-side products fused into the mixing stage, so that Y never
// goes to HBM.  One CTA per k_z unit (group, P_r, 128-column tile), thread = column.  For
// each source s = (h, b) of the group the thread forms
//     Y_s[row, col] = sum_k C_h[row, Q_r col k] rho_b[col - (Q_l col 0), k]
// for KYZ_RB rows of P_r at a time in registers (the density sub-block (Q_l, Q_r) holding the
// column comes from a per-CTA column table; C values are shared by the columns of one
// sub-block and the densities by all rows, so both stay in L1), then writes every proton
// operator's mixed row sum_s w_(a,s) Y_s to its Zbar tile in the tensor-core layout.  A
// column no sub-block of a source reaches contributes zero for that source.
constexpr int KYZ_NS = 16;   // sources per group of the fused stage (larger groups: k_y + k_z)
constexpr int KYZ_RB = 4;    // rows per register block

__global__ void __launch_bounds__(128) k_yz(const ZUnit *__restrict__ units, const ZGroup *__restrict__ groups,
                                            const ZSrc *__restrict__ srcs, const ZOp *__restrict__ ops,
                                            const ZOpTC *__restrict__ ops_tc, const YBlk *__restrict__ blks,
                                            const float *__restrict__ W, const float *__restrict__ x,
                                            const float *__restrict__ rho, float *__restrict__ Zb) {
  __shared__ float ws[ZMAXA][KYZ_NS];
  __shared__ int64_t zdst[ZMAXA];
  __shared__ int zk[ZMAXA];
  __shared__ int16_t colblk[KYZ_NS][128];
  __shared__ ZSrc ss[KYZ_NS];
  const ZUnit u = units[blockIdx.x];
  const ZGroup G = groups[u.grp];
  const int na = u.op_end - u.op_begin, ns = G.ns;
  const int tid = threadIdx.x;
  for (int e = tid; e < na * KYZ_NS; e += blockDim.x) {
    const int a = e / KYZ_NS, sidx = e - a * KYZ_NS;
    ws[a][sidx] = sidx < ns ? W[G.w_off + ops[u.op_begin + a].wrow * ns + sidx] : 0.f;
  }
  for (int e = tid; e < na; e += blockDim.x) {
    const ZOpTC o = ops_tc[u.op_begin + e];
    zdst[e] = o.base + (int64_t)(u.c0 / 128) * o.kgroups * 1024;
    zk[e] = o.kofs;
  }
  for (int e = tid; e < KYZ_NS * 128; e += blockDim.x) (&colblk[0][0])[e] = -1;
  for (int e = tid; e < ns; e += blockDim.x) ss[e] = srcs[G.s_begin + e];
  __syncthreads();
  {  // column -> sub-block tables, 8 threads per source
    const int sidx = tid >> 3, q = tid & 7;
    if (sidx < ns) {
      const ZSrc S = ss[sidx];
      for (int bi = S.b_begin + q; bi < S.b_end; bi += 8) {
        const YBlk b = blks[bi];
        const int lo = max(b.ycol, u.c0), hi = min(b.ycol + b.nl, u.c0 + u.ncols);
        for (int c = lo; c < hi; ++c) colblk[sidx][c - u.c0] = (int16_t)(bi - S.b_begin);
      }
    }
  }
  __syncthreads();
  const int c = tid;
  if (c >= u.ncols) return;
  const int col = u.c0 + c;
  for (int rr0 = 0; rr0 < u.nr; rr0 += KYZ_RB) {
    const int nrb = min(KYZ_RB, u.nr - rr0);
    float y[KYZ_NS][KYZ_RB];
#pragma unroll
    for (int sidx = 0; sidx < KYZ_NS; ++sidx) {
#pragma unroll
      for (int rb = 0; rb < KYZ_RB; ++rb) y[sidx][rb] = 0.f;
      if (sidx < ns) {
        const int bi = colblk[sidx][c];
        if (bi >= 0) {
          const ZSrc &S = ss[sidx];
          const YBlk b = blks[S.b_begin + bi];
          const int64_t m = S.m;
          const float *cp = x + S.c_base + u.row0 + rr0 + m * b.ccol;
          const float *rp = rho + b.rho + (col - b.ycol);
          for (int k = 0; k < b.nr; ++k) {
            const float rv = __ldg(rp + (int64_t)b.ldr * k);
#pragma unroll
            for (int rb = 0; rb < KYZ_RB; ++rb)
              if (rb < nrb) y[sidx][rb] = fmaf(__ldg(cp + rb + m * k), rv, y[sidx][rb]);
          }
        }
      }
    }
    for (int a = 0; a < na; ++a) {
#pragma unroll
      for (int rb = 0; rb < KYZ_RB; ++rb) {
        if (rb < nrb) {
          float z = 0.f;
#pragma unroll
          for (int sidx = 0; sidx < KYZ_NS; ++sidx) z = fmaf(ws[a][sidx], y[sidx][rb], z);
          Zb[zdst[a] + umma::ztile_index(zk[a] + rr0 + rb, c)] = z;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_a: one CTA of 128 threads per (output slab P_l, 128-column tile, K range).
// The tile's Zbar rows (128 columns each, 16-byte aligned rows) and the matching
// Abar rows (nlp entries each) stream through a 3-stage shared-memory pipeline of
// asynchronous 16-byte copies, KS stacked rows per stage.  Within a stage the 4
// warps split the rows; lane q owns columns 4q .. 4q+3 and accumulates a group of
// RG output rows for them in registers (one 16-byte Zbar load and RG/4 broadcast
// 16-byte Abar loads per stacked row, 4*RG FMAs).  Slabs with more than RG rows
// take several passes.  At the end of a pass the warps' partial sums are added
// through shared memory and the tile adds its result to the output with atomic
// adds (K ranges of one slab are separate tiles; the like-particle stage wrote
// the output first).
// Tile shape (compile-time; the defaults are the fastest of a sweep on B200 at fp 6p+6n,
// 2-4 stages x 8-64 rows x row groups of 8/16 x 1 or 4 groups per pass): stacked rows per
// stage KS, output rows per register group RG, row groups sharing one pass over the K range
// GPP (1: the 4 warps split the stacked rows; 4: the warps take different row groups, so a
// slab with many rows does not re-read its Zbar tile from HBM), and the pipeline depth.
// Measured: FP32 0.76 ms (KS 32, RG 16, GPP 1), FP64 1.59 ms (KS 16, RG 8, GPP 4).
#ifndef KA_KS32
#define KA_KS32 32
#endif
#ifndef KA_RG32
#define KA_RG32 16
#endif
#ifndef KA_GPP32
#define KA_GPP32 1
#endif
#ifndef KA_KS64
#define KA_KS64 16
#endif
#ifndef KA_RG64
#define KA_RG64 8
#endif
#ifndef KA_GPP64
#define KA_GPP64 4
#endif
#ifndef KA_NSTAGE
#define KA_NSTAGE 2
#endif
#ifndef KA_MINB    // resident CTAs per SM the register budget is sized for (shared memory allows 4)
#define KA_MINB 4
#endif
template <typename T> struct KaCfg;
template <> struct KaCfg<float> { static constexpr int KS = KA_KS32, RG = KA_RG32, GPP = KA_GPP32; };
template <> struct KaCfg<double> { static constexpr int KS = KA_KS64, RG = KA_RG64, GPP = KA_GPP64; };
static_assert(KA_GPP32 >= 1 && KA_GPP32 <= 4 && KA_GPP64 >= 1 && KA_GPP64 <= 4, "1 to 4 row groups per pass");
constexpr int KA_STAGES = KA_NSTAGE;
constexpr int KA_MAXNL = 64;
static_assert(KA_RG32 % 4 == 0 && KA_RG64 % 4 == 0, "row groups of whole 4-row vectors");

__device__ __forceinline__ void ka_cp16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void ka_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void ka_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__device__ __forceinline__ void ka_ld4(const float *p, float v[4]) {
  const float4 q = *reinterpret_cast<const float4 *>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ka_ld4(const double *p, double v[4]) {
  const double2 a = *reinterpret_cast<const double2 *>(p);
  const double2 b = *reinterpret_cast<const double2 *>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

template <typename T>
struct KaSmem {
  static constexpr int KS = KaCfg<T>::KS, RG = KaCfg<T>::RG;
  static constexpr size_t pipe = sizeof(T) * (size_t)KA_STAGES * KS * (KA_TILE_COLS + KA_MAXNL);
  static constexpr size_t red = sizeof(T) * (size_t)4 * RG * KA_TILE_COLS;
  static constexpr size_t bytes = pipe > red ? pipe : red;
};

template <typename T>
__global__ void __launch_bounds__(128, KA_MINB) k_a(const ATile *__restrict__ tiles, const T *__restrict__ Abar,
                                           const T *__restrict__ Zb, T *__restrict__ out) {
  constexpr int KS = KaCfg<T>::KS, RG = KaCfg<T>::RG, TC = KA_TILE_COLS;
  constexpr int CPR = TC * (int)sizeof(T) / 16;                  // 16-byte chunks per Zbar row
  extern __shared__ __align__(16) unsigned char raw[];            // KaSmem<T>::bytes
  T *zs = reinterpret_cast<T *>(raw);                             // [KA_STAGES][KS][TC]
  T *as = zs + (size_t)KA_STAGES * KS * TC;                       // [KA_STAGES][KS * nlp]
  T *red = reinterpret_cast<T *>(raw);                            // [4][RG][TC] after a pass
  const ATile t = tiles[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nl = t.nl, nlp = t.nlp;
  const int ncp = (t.ncols * (int)sizeof(T) + 15) / 16;         // chunks per row that hold tile columns
  const int nchunk = (t.k_end - t.k_begin + KS - 1) / KS;
  const T *Zt = Zb + t.zbar;
  const T *At = Abar + t.abar;

  auto load = [&](int c, int b) {
    const int k0 = t.k_begin + c * KS;
    const int kc = min(KS, t.k_end - k0);
    T *zb = zs + (size_t)b * KS * TC;
    for (int e = tid; e < kc * CPR; e += 128) {
      const int r = e / CPR, q = e - r * CPR;
      if (q < ncp) ka_cp16(zb + r * TC + q * (16 / (int)sizeof(T)), Zt + (int64_t)(k0 + r) * t.ldz + q * (16 / (int)sizeof(T)));
    }
    T *ab = as + (size_t)b * KS * KA_MAXNL;
    const int na = kc * nlp * (int)sizeof(T) / 16;
    const T *asrc = At + (int64_t)k0 * nlp;
    for (int e = tid; e < na; e += 128) ka_cp16(ab + e * (16 / (int)sizeof(T)), asrc + e * (16 / (int)sizeof(T)));
  };

  // Row groups of RG output rows: up to GPP per pass over the K range, spread over the
  // warps (1 group: 4 warps split K; 2: 2 warps each; 3-4: one warp each), so that each
  // Zbar tile crosses HBM once per GPP row groups.
  const int ngr = (nl + RG - 1) / RG;
  constexpr int GPP = KaCfg<T>::GPP;
  for (int gp0 = 0; gp0 < ngr; gp0 += GPP) {
    const int npg = GPP == 1 ? 1 : min(GPP, ngr - gp0);          // a constant when GPP == 1
    const int wpg = npg == 1 ? 4 : (npg == 2 ? 2 : 1);
    const int gi = warp / wpg, ks = warp - gi * wpg;
    const bool active = gi < npg;
    const int l0 = (gp0 + (active ? gi : 0)) * RG;
    const int ng = active ? min(RG, nlp - l0) / 4 : 0;            // groups of 4 rows with Abar entries
    T acc[RG][4];
#pragma unroll
    for (int i = 0; i < RG; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[i][c] = T(0);
#pragma unroll
    for (int s = 0; s < KA_STAGES - 1; ++s) {
      if (s < nchunk) load(s, s);
      ka_commit();
    }
    for (int c = 0; c < nchunk; ++c) {
      if (c + KA_STAGES - 1 < nchunk) load(c + KA_STAGES - 1, (c + KA_STAGES - 1) % KA_STAGES);
      ka_commit();
      ka_wait<KA_STAGES - 1>();
      __syncthreads();
      const int b = c % KA_STAGES;
      const int kc = min(KS, t.k_end - (t.k_begin + c * KS));
      const T *zb = zs + (size_t)b * KS * TC + 4 * lane;
      const T *ab = as + (size_t)b * KS * KA_MAXNL + l0;
      if (active) {
        // the stacked rows of this warp: ks, ks + wpg, ... (the stride as a constant)
        auto rows = [&](auto stride) {
          constexpr int WS = decltype(stride)::value;
          for (int r = ks; r < kc; r += WS) {
            T z[4];
            ka_ld4(zb + r * TC, z);
            const T *ar = ab + r * nlp;
#pragma unroll
            for (int g = 0; g < RG / 4; ++g) {
              if (g < ng) {
                T a[4];
                ka_ld4(ar + 4 * g, a);
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                  for (int cc = 0; cc < 4; ++cc) acc[4 * g + i][cc] = fma(a[i], z[cc], acc[4 * g + i][cc]);
              }
            }
          }
        };
        if (wpg == 4) rows(std::integral_constant<int, 4>());
        else if (wpg == 2) rows(std::integral_constant<int, 2>());
        else rows(std::integral_constant<int, 1>());
      }
      __syncthreads();
    }
    ka_wait<0>();
    // add the K-slot warps' partial sums of each row group; the result goes to the output
#pragma unroll
    for (int i = 0; i < RG; ++i)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) red[((size_t)warp * RG + i) * TC + 4 * lane + cc] = acc[i][cc];
    __syncthreads();
    if (tid < t.ncols) {
      for (int gg = 0; gg < npg; ++gg) {
        const int lg = (gp0 + gg) * RG;
        for (int i = 0; i < RG && lg + i < nl; ++i) {
          T v = T(0);
          for (int w = 0; w < wpg; ++w) v += red[((size_t)(gg * wpg + w) * RG + i) * TC + tid];
          atomicAdd(out + t.out + (lg + i) + (int64_t)t.ld * tid, v);
        }
      }
    }
    __syncthreads();
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


template <typename T>
static void dev_refill(T *p, const std::vector<double> &v) {
  if (v.empty() || !p) return;
  std::vector<T> tmp(v.begin(), v.end());
  NSX_CUDA(cudaMemcpy(p, tmp.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}

// The segments' values scattered into the dense like-particle H (FP64, and FP32 once that form
// is set up), both triangles: one CTA per segment (NuOrth's layout, matrix(dimptr, dimpt):
// value[kr + nr * kl] = H[(np, kl), (npr, kr)]).
__global__ void k_fill_h(const HSeg *__restrict__ segs, const double *__restrict__ vals, double *__restrict__ hA,
                         double *__restrict__ hB, float *__restrict__ hA32, float *__restrict__ hB32) {
  const HSeg g = segs[blockIdx.x];
  double *H = g.species ? hB : hA;
  float *H32 = g.species ? hB32 : hA32;
  const int64_t n = (int64_t)g.nl * g.nr;
  const bool diag = g.ro == g.co;   // a diagonal segment: entry (kl, kr) with kl >= kr sets both
  for (int64_t e = threadIdx.x; e < n; e += blockDim.x) {
    const int kl = (int)(e / g.nr), kr = (int)(e - (int64_t)kl * g.nr);
    if (diag && kl < kr) continue;   // (the host fill's order: the later, lower-triangle write wins)
    const double v = vals[g.v + e];
    const int64_t i1 = g.h + (g.ro + kl) + (int64_t)g.d * (g.co + kr), i2 = g.h + (g.co + kr) + (int64_t)g.d * (g.ro + kl);
    H[i1] = v;
    H[i2] = v;
    if (H32) {
      H32[i1] = (float)v;
      H32[i2] = (float)v;
    }
  }
}

// Copies the interaction-dependent operands into the device buffers the handle already holds, in
// every precision that has been set up: the mixing weights, and the like-particle segments'
// values, which k_fill_h scatters into the dense H.  The copies and the scatter complete before
// return, so products issued afterwards on any stream see the new values.
void upload_interaction(nsx_handle *h, const double *a_seg_vals, const double *b_seg_vals) {
  NSX_CUDA(cudaDeviceSynchronize());  // no product of the old interaction may still read them
  auto &d = h->d;
  dev_refill<double>(d.w, h->weights);
  if (d.w32) dev_refill<float>(d.w32, h->weights);
  const int64_t na = h->A.seg_off.empty() ? 0 : h->A.seg_off.back();
  const int64_t nb = h->B.seg_off.empty() ? 0 : h->B.seg_off.back();
  if (na) NSX_CUDA(cudaMemcpy(d.segvals, a_seg_vals, sizeof(double) * na, cudaMemcpyHostToDevice));
  if (nb) NSX_CUDA(cudaMemcpy(d.segvals + na, b_seg_vals, sizeof(double) * nb, cudaMemcpyHostToDevice));
  const int nseg = (int)(h->A.seg_J2.size() + h->B.seg_J2.size());
  if (nseg > 0) {
    k_fill_h<<<nseg, 256>>>(d.hsegs, d.segvals, d.hA, d.hB, d.hA32, d.hB32);
    h->launches++;
    NSX_CUDA(cudaGetLastError());
  }
  NSX_CUDA(cudaDeviceSynchronize());
}

cudaStream_t solve_stream(nsx_handle *h) {
  if (!h->stream) NSX_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  return h->stream;
}

void upload(nsx_handle *h) {
  if (h->max_anl > KA_MAXNL) fail(NSX_E_ARG, "proton partition with more than 64 J-states: not supported by k_a");
  auto &d = h->d;
  d.rhoB = dev_copy<double>(h->yrho);
  d.hA = dev_copy<double>(h->A.hdense);
  d.hB = dev_copy<double>(h->B.hdense);
  {  // the segment table of the like-particle H (for new interactions)
    std::vector<HSeg> segs;
    const SpeciesPlan *sp[2] = {&h->A, &h->B};
    int64_t vbase = 0;
    for (int sI = 0; sI < 2; ++sI) {
      const SpeciesPlan &S = *sp[sI];
      for (size_t g = 0; g < S.seg_J2.size(); ++g) {
        const int J2 = S.seg_J2[g], j = S.jidx(J2);
        const int np = S.seg_np[g] - 1, npr = S.seg_npr[g] - 1;
        HSeg e;
        e.h = S.hoff[j];
        e.v = vbase + S.seg_off[g];
        e.d = (int32_t)S.poff[j][S.nspart];
        e.ro = S.poff[j][np];
        e.co = S.poff[j][npr];
        e.nl = S.njt_of(np, J2);
        e.nr = S.njt_of(npr, J2);
        e.species = sI;
        segs.push_back(e);
      }
      vbase += S.seg_off.empty() ? 0 : S.seg_off.back();
    }
    d.hsegs = dev_copy_pod(segs);
    NSX_CUDA(cudaMalloc(&d.segvals, sizeof(double) * std::max<int64_t>(vbase, 1)));
  }
  d.w = dev_copy<double>(h->weights);
  d.abar = dev_copy<double>(h->abar);
  d.ygroups = dev_copy_pod(h->ygroups);
  d.yblks = dev_copy_pod(h->yblks);
  d.zgroups = dev_copy_pod(h->zgroups);
  d.zsrcs = dev_copy_pod(h->zsrcs);
  d.zunits = dev_copy_pod(h->zunits);
  d.zcta = dev_copy_pod(h->zcta);
  d.zops = dev_copy_pod(h->zops);
  d.atiles = dev_copy_pod(h->atiles);
  d.ltiles = dev_copy_pod(h->ltiles);
  NSX_CUDA(cudaMalloc(&d.xin, h->no_state * sizeof(double)));
  NSX_CUDA(cudaMalloc(&d.xout, h->no_state * sizeof(double)));
  NSX_CUDA(cudaEventCreate(&h->ev0));
  NSX_CUDA(cudaEventCreate(&h->ev1));
  // k_a's shared-memory cap: the same constant on every call (harmless to repeat)
  NSX_CUDA(cudaFuncSetAttribute(k_a<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaSmem<double>::bytes));
  NSX_CUDA(cudaFuncSetAttribute(k_a<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaSmem<float>::bytes));
  NSX_CUDA(cudaFuncSetAttribute(k_a_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaTcCfg<16>::SMEM));
  NSX_CUDA(cudaFuncSetAttribute(k_a_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaTcCfg<32>::SMEM));
  NSX_CUDA(cudaFuncSetAttribute(k_a_tc<48>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaTcCfg<48>::SMEM));
  NSX_CUDA(cudaFuncSetAttribute(k_a_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KaTcCfg<64>::SMEM));
  NSX_CUDA(cudaMalloc(&d.err, sizeof(int)));
  NSX_CUDA(cudaMemset(d.err, 0, sizeof(int)));
  // copies from pageable memory may return before their DMA lands; work on non-blocking
  // streams (the caller's, or the handle's solve stream) is not ordered after them
  NSX_CUDA(cudaDeviceSynchronize());
}

void ensure_precision(nsx_handle *h, int precision) {
  auto &d = h->d;
  size_t ny = std::max<int64_t>(h->y_elems, 1), nz = std::max<int64_t>(h->z_elems, 1);
  if (precision == NSX_FP64) {
    if (!d.y64) {
      NSX_CUDA(cudaMalloc(&d.y64, ny * sizeof(double)));
      NSX_CUDA(cudaMalloc(&d.z64, nz * sizeof(double)));
    }
  } else if (precision == NSX_FP32) {
    if (!d.x32) {   // the data every FP32 variant reads; each variant's own buffers: ensure_fp32_path
      (void)nz;
      d.rhoB32 = dev_copy<float>(h->yrho);
      // the FP32 dense H from the device's FP64 copy (the host copy is the plan's: a new
      // interaction updates the device copy only)
      const int64_t nA = (int64_t)h->A.hdense.size(), nB = (int64_t)h->B.hdense.size();
      NSX_CUDA(cudaMalloc(&d.hA32, sizeof(float) * std::max<int64_t>(nA, 1)));
      NSX_CUDA(cudaMalloc(&d.hB32, sizeof(float) * std::max<int64_t>(nB, 1)));
      if (nA) k_d2f<<<(unsigned)std::min<int64_t>((nA + 255) / 256, 148 * 16), 256>>>(d.hA, d.hA32, nA);
      if (nB) k_d2f<<<(unsigned)std::min<int64_t>((nB + 255) / 256, 148 * 16), 256>>>(d.hB, d.hB32, nB);
      NSX_CUDA(cudaGetLastError());
      d.w32 = dev_copy<float>(h->weights);
      NSX_CUDA(cudaMalloc(&d.x32, h->no_state * sizeof(float)));
      NSX_CUDA(cudaMalloc(&d.o32, h->no_state * sizeof(float)));
      NSX_CUDA(cudaDeviceSynchronize());  // as in upload()
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
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[NSX_STAGES], double flops[NSX_STAGES]) {
  const double es = precision == NSX_FP64 ? 8.0 : 4.0;
  const double n = (double)h->no_state;
  const double rhoB = (double)h->B.vals.size();
  double hd = (double)(h->A.hdense.size() + h->B.hdense.size());
  const double y = (double)h->y_elems, z = (double)h->z_elems;
  bytes[0] = es * (2.0 * n + hd);                         // C in, out written, dense H
  bytes[1] = es * (n + rhoB + y);                         // C in, rho_B, Y written
  bytes[2] = es * (y + z + (double)h->weights.size());    // Y in, Zbar written
  bytes[3] = es * (z + (double)h->abar.size() + 2.0 * n); // Zbar in, Abar, out read + written
  // the FP32 variant in use (before the first FP32 product: the fused one where it exists)
  const int path = precision != NSX_FP32 ? 0 : (h->fp32_path ? h->fp32_path : (h->max_zns <= KYZ_NS ? 1 : 2));
  const bool fused = path == NSX_FP32_FUSED;
  if (path == NSX_FP32_FUSED || path == NSX_FP32_TC) {   // tensor-core layout of Zbar, split Abar
    bytes[2] = es * (y + (double)h->z32_elems + (double)h->weights.size());
    bytes[3] = es * ((double)h->z32_elems + 2.0 * (double)h->abar_big.size() + 2.0 * n);
  }
  if (fused) {   // k_yz: C and rho_B in, Zbar written; Y never stored
    bytes[1] = 0.0;
    bytes[2] = es * (n + rhoB + (double)h->z32_elems + (double)h->weights.size());
  }
  bytes[4] = precision == NSX_FP64 ? 0.0 : n * (8.0 + 4.0);
  flops[0] = h->flops_like;
  flops[1] = fused ? 0.0 : h->flops_y;
  flops[2] = fused ? h->flops_y + h->flops_mix : h->flops_mix;
  flops[3] = h->flops_a;
  flops[4] = 0.0;
}

// The k_a_tc launches, one per N class, run concurrently: the class of 64-row partitions
// (few tiles with the longest stacked operands) and the other non-empty classes start on
// the handle's auxiliary streams, forked from and joined back into `s` with events, so that
// the long tiles overlap the many short ones instead of following them.  Returns the launches.
// The handle's auxiliary streams and their fork/join events (created on first use).
static void ensure_aux(nsx_handle *h) {
  if (h->fork_ev) return;
  NSX_CUDA(cudaEventCreateWithFlags(&h->fork_ev, cudaEventDisableTiming));
  NSX_CUDA(cudaEventCreateWithFlags(&h->like_fork, cudaEventDisableTiming));
  NSX_CUDA(cudaEventCreateWithFlags(&h->like_join, cudaEventDisableTiming));
  for (int i = 0; i < KTC_NCLASS - 1; ++i) {
    NSX_CUDA(cudaStreamCreateWithFlags(&h->aux[i], cudaStreamNonBlocking));
    NSX_CUDA(cudaEventCreateWithFlags(&h->join_ev[i], cudaEventDisableTiming));
  }
}

static int launch_ka_tc(nsx_handle *h, const float *Z, float *out, cudaStream_t s) {
  auto &d = h->d;
  int used[KTC_NCLASS], nu = 0;
  for (int c = KTC_NCLASS - 1; c >= 0; --c)   // widest class first
    if (h->atc_off[c + 1] > h->atc_off[c]) used[nu++] = c;
  if (nu == 0) return 0;
  if (nu > 1) {
    ensure_aux(h);
    NSX_CUDA(cudaEventRecord(h->fork_ev, s));
  }
  for (int i = 0; i < nu; ++i) {
    const int c = used[i];
    cudaStream_t st = i + 1 < nu ? h->aux[i] : s;   // the last (narrowest) class on s itself
    if (st != s) NSX_CUDA(cudaStreamWaitEvent(st, h->fork_ev, 0));
    const unsigned n = (unsigned)(h->atc_off[c + 1] - h->atc_off[c]);
    const ATileTC *tl = d.atiles_tc + h->atc_off[c];
    switch (c) {
      case 0: k_a_tc<16><<<n, 128, KaTcCfg<16>::SMEM, st>>>(tl, Z, d.abar_big, d.abar_small, out, d.err); break;
      case 1: k_a_tc<32><<<n, 128, KaTcCfg<32>::SMEM, st>>>(tl, Z, d.abar_big, d.abar_small, out, d.err); break;
      case 2: k_a_tc<48><<<n, 128, KaTcCfg<48>::SMEM, st>>>(tl, Z, d.abar_big, d.abar_small, out, d.err); break;
      default: k_a_tc<64><<<n, 128, KaTcCfg<64>::SMEM, st>>>(tl, Z, d.abar_big, d.abar_small, out, d.err); break;
    }
    if (st != s) {
      NSX_CUDA(cudaEventRecord(h->join_ev[i], st));
      NSX_CUDA(cudaStreamWaitEvent(s, h->join_ev[i], 0));
    }
  }
  NSX_CUDA(cudaGetLastError());
  return nu;
}

// One product's stages.  path: 0 for FP64; for FP32 the variant (NSX_FP32_FUSED / _TC / _SIMT).
// fork: the like-particle stage may run on an auxiliary stream (the fixed-scratch entry point
// keeps everything on the caller's stream and creates nothing).
template <typename T>
static void run_stages(nsx_handle *h, int path, const T *x, T *out, const T *rhoB, const T *hA, const T *hB,
                       const T *w, const T *abar, T *Y, T *Z, cudaStream_t s, bool fork = true) {
  auto &d = h->d;
  // The like-particle stage writes the output block and reads only x: it runs on an auxiliary
  // stream beside the neutron-side and mixing stages (which never touch the output) and is
  // joined back before the proton side adds to the output.  With per-stage timing on, the
  // stages run one after another, so that each stage's interval is its own.
  const bool pn = !h->zunits.empty();
  bool forked = false;
  if (!h->ltiles.empty()) {
    cudaStream_t ls = s;
    if (pn && fork && !h->timing) {
      ensure_aux(h);
      NSX_CUDA(cudaEventRecord(h->like_fork, s));
      NSX_CUDA(cudaStreamWaitEvent(h->aux[0], h->like_fork, 0));
      ls = h->aux[0];
      forked = true;
    }
    StageScope sc(h, 0, ls);
    k_like<T><<<(unsigned)h->ltiles.size(), 256, 0, ls>>>(d.ltiles, x, out, hA, hB);
  }
  if (forked) NSX_CUDA(cudaEventRecord(h->like_join, h->aux[0]));
  constexpr bool F32 = std::is_same<T, float>::value;
  const bool fused = F32 && path == NSX_FP32_FUSED;   // Y formed inside the mixing stage
  const bool tc = F32 && path != NSX_FP32_SIMT;        // proton side on the tensor cores
  if (fused) {
    if constexpr (F32) {
      if (!h->zunits.empty()) {
        StageScope sc(h, 2, s);
        k_yz<<<(unsigned)h->zunits.size(), 128, 0, s>>>(d.zunits, d.zgroups, d.zsrcs, d.zops, d.zops_tc, d.yblks, w, x,
                                                         rhoB, Z);
      }
    }
  } else {
    if (!h->ygroups.empty()) {
      StageScope sc(h, 1, s);
      k_y<T><<<(unsigned)h->ygroups.size(), 128, 0, s>>>(d.ygroups, d.yblks, x, rhoB, Y);
    }
    if (!h->zunits.empty()) {
      StageScope sc(h, 2, s);
      const unsigned nu = (unsigned)(h->zcta.size() - 1);
      // sources per group: registers for 16 unless the plan has a larger group
      if (tc) {
        if constexpr (F32) {
          if (h->max_zns <= 16) k_z<T, 16, true><<<nu, 128, 0, s>>>(d.zunits, d.zcta, d.zgroups, d.zsrcs, d.zops, d.zops_tc, w, Y, Z);
          else k_z<T, ZMAXS, true><<<nu, 128, 0, s>>>(d.zunits, d.zcta, d.zgroups, d.zsrcs, d.zops, d.zops_tc, w, Y, Z);
        }
      } else if (h->max_zns <= 16) {
        k_z<T, 16, false><<<nu, 128, 0, s>>>(d.zunits, d.zcta, d.zgroups, d.zsrcs, d.zops, d.zops_tc, w, Y, Z);
      } else {
        k_z<T, ZMAXS, false><<<nu, 128, 0, s>>>(d.zunits, d.zcta, d.zgroups, d.zsrcs, d.zops, d.zops_tc, w, Y, Z);
      }
    }
  }
  if (forked) NSX_CUDA(cudaStreamWaitEvent(s, h->like_join, 0));   // the output block is written
  if (tc) {
    if constexpr (F32) {
      if (h->atc_off[KTC_NCLASS] > 0) {
        StageScope sc(h, 3, s);   // one stage interval around the concurrent class launches
        const int nl = launch_ka_tc(h, Z, out, s);
        h->launches += nl - 1;
      }
    }
  } else if (!h->atiles.empty()) {
    StageScope sc(h, 3, s);
    k_a<T><<<(unsigned)h->atiles.size(), 128, KaSmem<T>::bytes, s>>>(d.atiles, abar, Z, out);
  }
  NSX_CUDA(cudaGetLastError());
}

static bool fp32_path_available(const nsx_handle *h, int path) {
  return path == NSX_FP32_TC || path == NSX_FP32_SIMT || (path == NSX_FP32_FUSED && h->max_zns <= KYZ_NS);
}

// The device buffers of one FP32 variant (allocated once; the tensor-core Zbar's padding rows
// and columns stay zero for good).
static void ensure_fp32_path(nsx_handle *h, int path) {
  auto &d = h->d;
  bool any = false;
  if (path != NSX_FP32_FUSED && !d.y32) {
    NSX_CUDA(cudaMalloc(&d.y32, std::max<int64_t>(h->y_elems, 1) * sizeof(float)));
    any = true;
  }
  if (path != NSX_FP32_SIMT && !d.z32) {
    const size_t nz32 = std::max<int64_t>(h->z32_elems, 1);
    NSX_CUDA(cudaMalloc(&d.z32, nz32 * sizeof(float)));
    NSX_CUDA(cudaMemset(d.z32, 0, nz32 * sizeof(float)));
    d.abar_big = dev_copy_pod(h->abar_big);
    d.abar_small = dev_copy_pod(h->abar_small);
    d.zops_tc = dev_copy_pod(h->zops_tc);
    d.atiles_tc = dev_copy_pod(h->atiles_tc);
    any = true;
  }
  if (path == NSX_FP32_SIMT && !d.z32r) {
    NSX_CUDA(cudaMalloc(&d.z32r, std::max<int64_t>(h->z_elems, 1) * sizeof(float)));
    d.abar32 = dev_copy<float>(h->abar);
    any = true;
  }
  if (any) NSX_CUDA(cudaDeviceSynchronize());   // copies from pageable memory have landed
}

// Frees what the chosen variant does not read.
static void release_fp32_unused(nsx_handle *h, int path) {
  auto &d = h->d;
  auto drop = [](auto *&p) {
    if (p) cudaFree(p);
    p = nullptr;
  };
  if (path == NSX_FP32_FUSED) drop(d.y32);
  if (path == NSX_FP32_SIMT) {
    drop(d.z32);
    drop(d.abar_big);
    drop(d.abar_small);
    drop(d.zops_tc);
    drop(d.atiles_tc);
  } else {
    drop(d.z32r);
    drop(d.abar32);
  }
}

static void run_fp32(nsx_handle *h, int path, cudaStream_t s) {
  auto &d = h->d;
  run_stages<float>(h, path, d.x32, d.o32, d.rhoB32, d.hA32, d.hB32, d.w32, d.abar32, d.y32,
                    path == NSX_FP32_SIMT ? d.z32r : d.z32, s);
}

// The variant of the handle's FP32 products: the requested one, or the fastest available one
// timed on the product at hand (second of two runs each, CUDA events on `s`; the counters and
// stage timings leave the trial runs out).
static void choose_fp32_path(nsx_handle *h, cudaStream_t s) {
  int best = h->fp32_request;
  if (best == NSX_FP32_AUTO) {
    const int64_t launches = h->launches;
    int64_t sl[NSX_STAGES];
    std::copy(h->stage_launches, h->stage_launches + NSX_STAGES, sl);
    const bool timing = h->timing;
    h->timing = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NSX_CUDA(cudaEventCreate(&e0));
    NSX_CUDA(cudaEventCreate(&e1));
    float tbest = 0.f;
    try {
      for (int p = NSX_FP32_FUSED; p <= NSX_FP32_SIMT; ++p) {
        if (!fp32_path_available(h, p)) continue;
        ensure_fp32_path(h, p);
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {
          NSX_CUDA(cudaEventRecord(e0, s));
          run_fp32(h, p, s);
          NSX_CUDA(cudaEventRecord(e1, s));
        }
        NSX_CUDA(cudaEventSynchronize(e1));
        NSX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (best == NSX_FP32_AUTO || ms < tbest) {
          best = p;
          tbest = ms;
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      h->timing = timing;
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->timing = timing;
    h->launches = launches;
    std::copy(sl, sl + NSX_STAGES, h->stage_launches);
  }
  ensure_fp32_path(h, best);
  release_fp32_unused(h, best);
  h->fp32_path = best;
}

void set_fp32_path(nsx_handle *h, int path) {
  if (path < NSX_FP32_AUTO || path > NSX_FP32_SIMT) fail(NSX_E_ARG, "unknown FP32 variant");
  if (path != NSX_FP32_AUTO && !fp32_path_available(h, path))
    fail(NSX_E_ARG, "the fused FP32 variant needs mixing groups of at most 16 sources");
  h->fp32_request = path;
  h->fp32_path = 0;   // chosen again at the next FP32 product
}

void matvec_device(nsx_handle *h, const double *x, double *y, int precision, cudaStream_t s) {
  ensure_precision(h, precision);
  auto &d = h->d;
  h->matvecs++;
  h->last_precision = precision;
  if (precision == NSX_FP64) {
    run_stages<double>(h, 0, x, y, d.rhoB, d.hA, d.hB, d.w, d.abar, d.y64, d.z64, s);
  } else {
    int64_t n = h->no_state;
    unsigned g = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
    {
      StageScope sc(h, 4, s);
      k_d2f<<<g, 256, 0, s>>>(x, d.x32, n);
    }
    if (h->fp32_path == 0) choose_fp32_path(h, s);
    run_fp32(h, h->fp32_path, s);
    if (h->row1 > h->row0) {   // the rows this handle computed (all of them unless it is a shard)
      StageScope sc(h, 4, s);
      k_f2d<<<g, 256, 0, s>>>(d.o32 + h->row0, y + h->row0, h->row1 - h->row0);
    }
    NSX_CUDA(cudaGetLastError());
  }
  // a shard's product: the other ranks' rows come from the exchange
  if (h->shard_world > 1 && h->exch && h->exch(h->exch_user, y, h->no_state, (void *)s) != 0)
    fail(NSX_E_CUDA, "the exchange of the shards' rows failed");
}

// The FP64 stages with a caller-provided scratch buffer: Y (y_elems) and Zbar (z_elems) from
// zbar_scratch_offset(h).  Used by the fixed-scratch entry point.
void matvec_fp64_with_scratch(nsx_handle *h, const double *x, double *y, double *scratch, cudaStream_t s) {
  auto &d = h->d;
  h->matvecs++;
  h->last_precision = NSX_FP64;
  run_stages<double>(h, 0, x, y, d.rhoB, d.hA, d.hB, d.w, d.abar, scratch, scratch + zbar_scratch_offset(h), s,
                     false);
}

// Fails with NSX_E_CUDA if a tensor-core kernel gave up a bounded wait since the last check
// (the word is cleared).  Synchronises the device.
void check_device_error(nsx_handle *h) {
  if (!h->d.err) return;
  int e = 0;
  NSX_CUDA(cudaMemcpy(&e, h->d.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    NSX_CUDA(cudaMemset(h->d.err, 0, sizeof(int)));
    fail(NSX_E_CUDA, "a tensor-core kernel gave up waiting for its operands (bounded wait); results are invalid");
  }
}

void release(nsx_handle *h) {
  release_lanczos(h);
  auto &d = h->d;
  void *ptrs[] = {d.rhoB, d.hA, d.hB, d.w, d.abar, d.rhoB32, d.hA32, d.hB32, d.w32, d.abar32,
                  d.abar_big, d.abar_small, d.zops_tc, d.atiles_tc, d.err,
                  d.ygroups, d.yblks, d.zgroups, d.zsrcs, d.zunits, d.zcta, d.zops, d.atiles, d.ltiles,
                  d.y64, d.z64, d.y32, d.z32, d.z32r, d.x32, d.o32, d.xin, d.xout, d.hsegs, d.segvals};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  d = DeviceBuffers();
  for (int i = 0; i < KTC_NCLASS - 1; ++i) {
    if (h->aux[i]) cudaStreamDestroy(h->aux[i]);
    if (h->join_ev[i]) cudaEventDestroy(h->join_ev[i]);
    h->aux[i] = nullptr;
    h->join_ev[i] = nullptr;
  }
  if (h->fork_ev) cudaEventDestroy(h->fork_ev);
  if (h->like_fork) cudaEventDestroy(h->like_fork);
  if (h->like_join) cudaEventDestroy(h->like_join);
  h->fork_ev = h->like_fork = h->like_join = nullptr;
  for (auto &e : h->stage_events) {
    cudaEventDestroy(e.second.first);
    cudaEventDestroy(e.second.second);
  }
  h->stage_events.clear();
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  h->ev0 = h->ev1 = nullptr;
  if (h->stream) cudaStreamDestroy(h->stream);
  h->stream = nullptr;
}

}  // namespace nsx
