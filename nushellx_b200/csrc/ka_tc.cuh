// k_a on the 5th-generation tensor cores: out[P_l rows, 128-column tile] += Abar * Zbar
// for one proton slab, as a tcgen05 GEMM with the output transposed so that the long
// dimension is M:
//
//     D (128 x N) = Zbar^T (128 x K) * Abar^T (K x N),    M = output columns of the tile,
//                                                           N = nl (rows of P_l) padded to 16,
//                                                           K = the slab's stacked rows.
//
// Operands: the Zbar tile (written by the mixing stage as plain rows of 128 floats,
// umma::ztile_index) and the slab's Abar (static,
// packed at plan time K-major as umma::b_kmajor_index, split into its TF32 big and small parts)
// stream through an S-stage shared-memory pipeline of bulk asynchronous copies, 16 or 32
// stacked rows per stage (KaTcCfg).  After a stage lands, thread m (= output column m = TMEM lane
// m) reads its Zbar values of the stage (conflict-free: a warp's 32 columns of one row are one
// 128-byte line), splits them into TF32 big and small parts in registers and stores them to
// its TMEM lane (the big columns, then the small).  One thread issues 3 MMAs per 8 stacked rows
// with A in tensor memory and B in shared memory (big*big + big*small + small*big: FP32
// accuracy with FP32 accumulation) and commits them to the stage's mbarrier, which frees the
// stage for the copy S chunks ahead.  So a stage costs one shared-memory read of Zbar (no split
// halves written back, no A reads by the MMAs).
//
// TMEM: two accumulators of NPAD columns from column 0, taken by alternate stages, then two A
// buffers (big and small halves of one stage) from ACOL, also alternating (the MMAs of stage c - 2, which read the
// buffer stage c overwrites, have completed: the drain of stage c - 2 waited for them).  Once a
// stage's MMAs have completed the 4 warps add its accumulator to FP32 registers.  (The tensor
// core's own accumulation over thousands of stacked rows loses bits at every step, an error
// that grows with K; summing 32-row partial products in registers keeps the product at FP32
// accuracy.)  The registers are added to the output block, which the like-particle stage wrote
// first.  Each output element of a slab tile belongs to one CTA: no atomics.
#pragma once
#include "umma.cuh"

namespace nsx {

struct ATileTC {
  int64_t zbar;     // float offset of the Zbar tile (kgroups * 1024 floats, umma::ztile_index)
  int64_t abar;     // float offset of the slab's Abar (kgroups * 8 * npad floats, umma::b_kmajor_index)
  int64_t out;      // element offset of out[P_l row 0, col0]
  int32_t kgroups;  // stacked rows / 8 (the slab's K padded to a multiple of 8)
  int32_t ld;       // d_al (leading dimension of the output block)
  int32_t nl;       // rows of P_l
  int32_t ncols;    // columns of the tile (<= 128)
  int32_t split;    // 1: one of several K pieces of the slab tile (partial sums added atomically)
  int32_t pad;
};
constexpr int KTC_PIECE_GROUPS = 128;   // 8-row groups per K piece of a long slab (32 stages)

constexpr int KTC_GROUPS = 4;   // 8-row groups per pipeline stage of N = 48 / 64 (plan statistics)

// Stage size, stages and TMEM per N class.  N <= 32 (most tiles) takes 16-row stages: 128 TMEM
// columns and 51 KB of shared memory let four CTAs share an SM (more independent stage chains
// per SM); N = 48 / 64 take 32-row stages, two CTAs per SM.
template <int NPAD>
struct KaTcCfg {
  static constexpr int KG = NPAD <= 32 ? 2 : 4;                   // 8-row groups per stage
  static constexpr int S = NPAD <= 32 ? 4 : 3;                    // pipeline stages
  static constexpr int MIN_CTAS = NPAD <= 32 ? 4 : 2;             // resident CTAs per SM
  static constexpr uint32_t A_BYTES = KG * umma::A_GROUP_BYTES;
  static constexpr uint32_t B_BYTES = KG * NPAD * 32;             // one of big / small
  static constexpr uint32_t STAGE = A_BYTES + 2 * B_BYTES;
  // + 1 KB alignment slack and a 2 KB tail that no copy writes.  An MMA step reads exactly its B
  // footprint: NPAD/8 core matrices (SBO 128 B apart) x 2 K halves (LBO NPAD*16 B) = the
  // NPAD*32-byte group it starts; the tail is margin beyond that.
  static constexpr size_t SMEM = (size_t)S * STAGE + 1024 + 2048;
  static constexpr uint32_t ABUF = 16 * KG;                       // TMEM columns of one A buffer (big, small)
  static constexpr uint32_t ACOL = (2 * NPAD + 31) / 32 * 32;     // first A column, after the accumulators
  static constexpr uint32_t TCOLS = ACOL + 2 * ABUF <= 128 ? 128 : 256;   // a power of 2
};

template <int NPAD>
__global__ void __launch_bounds__(128, KaTcCfg<NPAD>::MIN_CTAS) k_a_tc(const ATileTC *__restrict__ tiles,
                                                                       const float *__restrict__ Zb,
                                                                       const float *__restrict__ Bbig,
                                                                       const float *__restrict__ Bsml,
                                                                       float *__restrict__ out, int *__restrict__ err) {
  using Cfg = KaTcCfg<NPAD>;
  constexpr int S = Cfg::S;
  constexpr int KG = Cfg::KG;
  static_assert(Cfg::ACOL >= 2 * NPAD && Cfg::ACOL + 2 * Cfg::ABUF <= Cfg::TCOLS, "TMEM columns");
  static_assert(Cfg::SMEM * Cfg::MIN_CTAS + 1024 * Cfg::MIN_CTAS <= 228 * 1024, "shared memory per SM");
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full[S], done[S], fin;
  __shared__ uint32_t tslot;
  const ATileTC t = tiles[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = (t.kgroups + KG - 1) / KG;
  auto A_raw = [&](int s) { return sm + (size_t)s * Cfg::STAGE; };
  auto B_big = [&](int s) { return sm + (size_t)s * Cfg::STAGE + Cfg::A_BYTES; };
  auto B_sml = [&](int s) { return sm + (size_t)s * Cfg::STAGE + Cfg::A_BYTES + Cfg::B_BYTES; };

  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      umma::mbar_init(&full[s], 1);
      umma::mbar_init(&done[s], 1);
    }
    umma::mbar_init(&fin, 1);
    umma::mbar_fence_init();
  }
  if (warp == 0) umma::tmem_alloc(&tslot, Cfg::TCOLS);
  umma::tc_fence_before();
  __syncthreads();
  umma::tc_fence_after();
  const uint32_t tmem = tslot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;   // this warp's TMEM lanes

  int issued = 0;
  auto issue = [&](int c) {
    const int s = c % S;
    const int ng = min(KG, t.kgroups - c * KG);
    const uint32_t ab = (uint32_t)ng * umma::A_GROUP_BYTES, bb = (uint32_t)ng * NPAD * 32;
    umma::mbar_arrive_tx(&full[s], ab + 2 * bb);
    umma::bulk_g2s(A_raw(s), Zb + t.zbar + (int64_t)c * KG * 1024, ab, &full[s]);
    umma::bulk_g2s(B_big(s), Bbig + t.abar + (int64_t)c * KG * 8 * NPAD, bb, &full[s]);
    umma::bulk_g2s(B_sml(s), Bsml + t.abar + (int64_t)c * KG * 8 * NPAD, bb, &full[s]);
    ++issued;
  };
  if (tid == 0)
    for (int c = 0; c < S && c < nchunk; ++c) issue(c);

  constexpr uint32_t IDESC = umma::idesc_tf32(NPAD, false);
  const int m = warp * 32 + lane;   // output column within the tile = TMEM lane
  float acc[NPAD];
#pragma unroll
  for (int i = 0; i < NPAD; ++i) acc[i] = 0.f;
  auto drain = [&](int cc) -> bool {
    if (!umma::mbar_wait(&done[cc % S], (uint32_t)(cc / S) & 1u)) return false;
    umma::tc_fence_after();
#pragma unroll
    for (int q = 0; q < NPAD / 16; ++q) {
      float v[16];
      umma::tmem_ld16(tmem + lane_base + (uint32_t)((cc & 1) * NPAD + q * 16), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[q * 16 + i] += v[i];
    }
    umma::tc_fence_before();
    return true;
  };
  bool bad = false;
  int c = 0;
  bool ok = true;
  for (; c < nchunk; ++c) {
    const int s = c % S;
    const bool w = umma::mbar_wait(&full[s], (uint32_t)(c / S) & 1u);
    if (__syncthreads_or(!w || bad)) {
      ok = false;
      break;
    }
    const int ng = min(KG, t.kgroups - c * KG);
    const float *a = reinterpret_cast<const float *>(A_raw(s));
    const uint32_t abuf = tmem + lane_base + Cfg::ACOL + (uint32_t)((c & 1) * Cfg::ABUF);
#pragma unroll
    for (int h = 0; h < KG / 2; ++h) {   // stacked rows 16h .. 16h + 15 of the stage
      float big[16], sml[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const int kk = 16 * h + k;
        const float x = kk < 8 * ng ? a[umma::ztile_index(kk, m)] : 0.f;
        big[k] = umma::tf32_big(x);
        sml[k] = x - big[k];
      }
      umma::tmem_st16(abuf + 16 * h, big);
      umma::tmem_st16(abuf + 8 * KG + 16 * h, sml);
    }
    umma::tmem_wait_st();
    umma::tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      umma::tc_fence_after();
      const uint32_t br = umma::smem_u32(B_big(s)), bs = umma::smem_u32(B_sml(s));
      const uint32_t dacc = tmem + (uint32_t)((c & 1) * NPAD);
      const uint32_t a0 = tmem + Cfg::ACOL + (uint32_t)((c & 1) * Cfg::ABUF);
      for (int j = 0; j < ng; ++j) {
        const uint64_t bdb = umma::sdesc(br + j * NPAD * 32, NPAD * 16, 128, umma::LAYOUT_NONE);
        const uint64_t bds = umma::sdesc(bs + j * NPAD * 32, NPAD * 16, 128, umma::LAYOUT_NONE);
        umma::mma_tf32_ta(dacc, a0 + 8 * j, bdb, IDESC, j > 0 ? 1u : 0u);   // a fresh partial sum per stage
        umma::mma_tf32_ta(dacc, a0 + 8 * j, bds, IDESC, 1u);
        umma::mma_tf32_ta(dacc, a0 + 8 * KG + 8 * j, bdb, IDESC, 1u);
      }
      umma::mma_commit(&done[s]);
    }
    if (c >= 1) {
      if (!drain(c - 1)) bad = true;
      else if (tid == 0 && c - 1 + S < nchunk) issue(c - 1 + S);
    }
  }
  if (ok && nchunk > 0 && !bad) {
    if (!drain(nchunk - 1)) bad = true;
  }
  if (tid == 0) {
    umma::mma_commit(&fin);
    if (!umma::mbar_wait(&fin, 0)) bad = true;
  }
  if (__syncthreads_or(bad)) ok = false;
  if (ok) {
    if (m < t.ncols) {
      float *o = out + t.out + (int64_t)t.ld * m;
      if (t.split) {
#pragma unroll
        for (int i = 0; i < NPAD; ++i)
          if (i < t.nl) atomicAdd(o + i, acc[i]);
      } else {
#pragma unroll
        for (int i = 0; i < NPAD; ++i)
          if (i < t.nl) o[i] += acc[i];
      }
    }
  } else if (tid == 0) {
    atomicOr(err, 1);
    for (int cc = c; cc < issued; ++cc) umma::mbar_wait(&full[cc % S], (uint32_t)(cc / S) & 1u);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, Cfg::TCOLS);
}

}  // namespace nsx
