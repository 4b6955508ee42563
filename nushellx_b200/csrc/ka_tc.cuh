// k_a on the 5th-generation tensor cores: out[P_l rows, 128-column tile] += Abar * Zbar
// for one proton slab, as a tcgen05 GEMM with the output transposed so that the long
// dimension is M:
//
//     D (128 x N) = Zbar^T (128 x K) * Abar^T (K x N),    M = output columns of the tile,
//                                                           N = nl (rows of P_l) padded to 16,
//                                                           K = the slab's stacked rows.
//
// Operands: the Zbar tile (written by the mixing stage directly in the MN-major
// 128-byte / 32-byte-base swizzled layout, umma::a_sw128_index) and the slab's Abar (static, packed at
// plan time K-major as umma::b_kmajor_index, split into its TF32 big and small parts)
// stream through an S-stage shared-memory pipeline of bulk asynchronous copies, 32
// stacked rows per stage.  After a stage lands, the 4 warps split Zbar into big/small
// parts in shared memory; one thread issues 3 MMAs per 8 stacked rows (big*big +
// big*small + small*big: FP32 accuracy with FP32 accumulation in TMEM) and commits them
// to the stage's mbarrier, which frees the stage for the copy S chunks ahead.  Each stage
// accumulates into one of two TMEM accumulators (128 x N, lane = output column), taken in
// turn; once a stage's MMAs have completed the 4 warps add its accumulator to FP32 registers.
// (The tensor core's own accumulation over thousands of stacked rows loses bits at every
// step, an error that grows with K; summing 32-row partial products in registers keeps the
// product at FP32 accuracy.)  The registers are added to the output block, which the
// like-particle stage wrote first.  Each output element of a slab tile belongs to one CTA: no
// atomics.
#pragma once
#include "umma.cuh"

namespace nsx {

struct ATileTC {
  int64_t zbar;     // float offset of the Zbar tile (kgroups * 1024 floats, umma::a_sw128_index)
  int64_t abar;     // float offset of the slab's Abar (kgroups * 8 * npad floats, umma::b_kmajor_index)
  int64_t out;      // element offset of out[P_l row 0, col0]
  int32_t kgroups;  // stacked rows / 8 (the slab's K padded to a multiple of 8)
  int32_t ld;       // d_al (leading dimension of the output block)
  int32_t nl;       // rows of P_l
  int32_t ncols;    // columns of the tile (<= 128)
};

constexpr int KTC_GROUPS = 4;   // 8-row groups per pipeline stage (32 stacked rows)

template <int NPAD>
struct KaTcCfg {
  // pipeline stages; N = 16 (most tiles) takes 3 so that two CTAs share an SM
  static constexpr int S = NPAD <= 16 ? 3 : (NPAD <= 32 ? 4 : 3);
  static constexpr int MIN_CTAS = NPAD <= 16 ? 2 : 1;             // resident CTAs per SM
  static constexpr uint32_t A_BYTES = KTC_GROUPS * umma::A_GROUP_BYTES;  // 16 KB
  static constexpr uint32_t B_BYTES = KTC_GROUPS * NPAD * 32;     // one of big / small
  static constexpr uint32_t STAGE = 2 * A_BYTES + 2 * B_BYTES;
  // + 1 KB alignment slack and a 2 KB tail that no copy writes.  An MMA step reads exactly its
  // operand footprint: A = 4 atoms (LBO 512 B apart) x 2 row groups (SBO 2048 B) = the 4096-byte
  // group it starts, B = NPAD/8 core matrices (SBO 128 B) x 2 K halves (LBO NPAD*16 B) = its
  // NPAD*32-byte group; the tail is margin beyond that.
  static constexpr size_t SMEM = (size_t)S * STAGE + 1024 + 2048;
  static constexpr uint32_t TCOLS = NPAD <= 16 ? 32 : (NPAD <= 32 ? 64 : 128);   // 2 accumulators, power of 2
};

template <int NPAD>
__global__ void __launch_bounds__(128, KaTcCfg<NPAD>::MIN_CTAS) k_a_tc(const ATileTC *__restrict__ tiles, const float *__restrict__ Zb,
                                                 const float *__restrict__ Bbig, const float *__restrict__ Bsml,
                                                 float *__restrict__ out, int *__restrict__ err) {
  using Cfg = KaTcCfg<NPAD>;
  constexpr int S = Cfg::S;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t full[S], done[S], fin;
  __shared__ uint32_t tslot;
  const ATileTC t = tiles[blockIdx.x];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = (t.kgroups + KTC_GROUPS - 1) / KTC_GROUPS;
  auto A_raw = [&](int s) { return sm + (size_t)s * Cfg::STAGE; };
  auto A_sml = [&](int s) { return sm + (size_t)s * Cfg::STAGE + Cfg::A_BYTES; };
  auto B_big = [&](int s) { return sm + (size_t)s * Cfg::STAGE + 2 * Cfg::A_BYTES; };
  auto B_sml = [&](int s) { return sm + (size_t)s * Cfg::STAGE + 2 * Cfg::A_BYTES + Cfg::B_BYTES; };

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

  int issued = 0;   // chunks whose copies thread 0 has issued
  auto issue = [&](int c) {
    const int s = c % S;
    const int ng = min(KTC_GROUPS, t.kgroups - c * KTC_GROUPS);
    const uint32_t ab = (uint32_t)ng * umma::A_GROUP_BYTES, bb = (uint32_t)ng * NPAD * 32;
    umma::mbar_arrive_tx(&full[s], ab + 2 * bb);
    umma::bulk_g2s(A_raw(s), Zb + t.zbar + (int64_t)c * KTC_GROUPS * 1024, ab, &full[s]);
    umma::bulk_g2s(B_big(s), Bbig + t.abar + (int64_t)c * KTC_GROUPS * 8 * NPAD, bb, &full[s]);
    umma::bulk_g2s(B_sml(s), Bsml + t.abar + (int64_t)c * KTC_GROUPS * 8 * NPAD, bb, &full[s]);
    ++issued;
  };
  if (tid == 0)
    for (int c = 0; c < S && c < nchunk; ++c) issue(c);

  constexpr uint32_t IDESC = umma::idesc_tf32(NPAD, true);
  const int m = warp * 32 + lane;   // output column within the tile = TMEM lane
  float acc[NPAD];
#pragma unroll
  for (int i = 0; i < NPAD; ++i) acc[i] = 0.f;
  // adds chunk cc's accumulator (columns (cc & 1) * NPAD ..) to the registers, once its MMAs completed
  auto drain = [&](int cc) -> bool {
    if (!umma::mbar_wait(&done[cc % S], (uint32_t)(cc / S) & 1u)) return false;
    umma::tc_fence_after();
#pragma unroll
    for (int q = 0; q < NPAD / 16; ++q) {
      float v[16];
      umma::tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((cc & 1) * NPAD + q * 16), v);
#pragma unroll
      for (int i = 0; i < 16; ++i) acc[q * 16 + i] += v[i];
    }
    umma::tc_fence_before();
    return true;
  };
  bool bad = false;   // this thread's failed waits
  int c = 0;
  bool ok = true;
  for (; c < nchunk; ++c) {
    const int s = c % S;
    const bool w = umma::mbar_wait(&full[s], (uint32_t)(c / S) & 1u);
    if (__syncthreads_or(!w || bad)) {
      ok = false;
      break;
    }
    // split the landed Zbar rows into TF32 big (in place) and small parts
    const int ng = min(KTC_GROUPS, t.kgroups - c * KTC_GROUPS);
    float4 *a4 = reinterpret_cast<float4 *>(A_raw(s));
    float4 *s4 = reinterpret_cast<float4 *>(A_sml(s));
    for (int i = tid; i < ng * 256; i += 128) {
      const float4 x = a4[i];
      float4 b;
      b.x = umma::tf32_big(x.x);
      b.y = umma::tf32_big(x.y);
      b.z = umma::tf32_big(x.z);
      b.w = umma::tf32_big(x.w);
      a4[i] = b;
      s4[i] = make_float4(x.x - b.x, x.y - b.y, x.z - b.z, x.w - b.w);
    }
    umma::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      umma::tc_fence_after();
      const uint32_t ar = umma::smem_u32(A_raw(s)), as = umma::smem_u32(A_sml(s));
      const uint32_t br = umma::smem_u32(B_big(s)), bs = umma::smem_u32(B_sml(s));
      const uint32_t dacc = tmem + (uint32_t)((c & 1) * NPAD);
      for (int j = 0; j < ng; ++j) {
        const uint64_t adb = umma::sdesc(ar + j * umma::A_GROUP_BYTES, umma::A_ATOM_BYTES, umma::A_ROWS4_BYTES,
                                         umma::LAYOUT_SW128_BASE32B);
        const uint64_t ads = umma::sdesc(as + j * umma::A_GROUP_BYTES, umma::A_ATOM_BYTES, umma::A_ROWS4_BYTES,
                                         umma::LAYOUT_SW128_BASE32B);
        const uint64_t bdb = umma::sdesc(br + j * NPAD * 32, NPAD * 16, 128, umma::LAYOUT_NONE);
        const uint64_t bds = umma::sdesc(bs + j * NPAD * 32, NPAD * 16, 128, umma::LAYOUT_NONE);
        umma::mma_tf32(dacc, adb, bdb, IDESC, j > 0 ? 1u : 0u);   // a fresh partial sum per chunk
        umma::mma_tf32(dacc, adb, bds, IDESC, 1u);
        umma::mma_tf32(dacc, ads, bdb, IDESC, 1u);
      }
      umma::mma_commit(&done[s]);
    }
    // the previous chunk's partial sum: into the registers; its stage is then free for the
    // copy S chunks ahead, and its accumulator for the chunk after this one
    if (c >= 1) {
      if (!drain(c - 1)) bad = true;
      else if (tid == 0 && c - 1 + S < nchunk) issue(c - 1 + S);
    }
  }
  if (ok && nchunk > 0 && !bad) {
    if (!drain(nchunk - 1)) bad = true;
  }
  // completion of every MMA issued (or of none) before the accumulators are released
  if (tid == 0) {
    umma::mma_commit(&fin);
    if (!umma::mbar_wait(&fin, 0)) bad = true;
  }
  if (__syncthreads_or(bad)) ok = false;
  if (ok) {
    if (m < t.ncols) {
      float *o = out + t.out + (int64_t)t.ld * m;
#pragma unroll
      for (int i = 0; i < NPAD; ++i)
        if (i < t.nl) o[i] += acc[i];
    }
  } else if (tid == 0) {
    atomicOr(err, 1);
    // copies still in flight into this CTA's shared memory land before it exits
    for (int cc = c; cc < issued; ++cc) umma::mbar_wait(&full[cc % S], (uint32_t)(cc / S) & 1u);
  }
  umma::tc_fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, Cfg::TCOLS);
}

}  // namespace nsx
