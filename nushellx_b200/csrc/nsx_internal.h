// Internal structures of libnsx: host-side plan of one J-scheme pn problem and
// the device buffers the H.v kernels and the Lanczos driver work on.
#pragma once
#include <climits>
#include <cstdint>
#include <string>
#include <vector>
#include <unordered_map>
#include <cuda_runtime.h>
#include "nsx.h"
#include "ka_tc.cuh"

namespace nsx {

struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);
#define NSX_CUDA(x) ::nsx::check_cuda((x), #x)

// Makes `device` current for the lifetime of the guard and then restores the caller's current
// device, so that an entry point never leaves a multi-GPU host on another device than it chose.
// device < 0 (plan-only handles) leaves the current device alone.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int device) {
    if (device < 0) return;
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != device) check_cuda(cudaSetDevice(device), "cudaSetDevice");
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard &) = delete;
  DeviceGuard &operator=(const DeviceGuard &) = delete;
};

// One density sub-block: left partition pl, right partition pr, value offset.
struct RhoBlk {
  int pl, pr;
  int64_t voff;
};

struct SpeciesPlan {
  int nspart = 0, minJ2 = 0, maxJ2 = -2, nJ = 0;
  int shell_first = 1, nshell = 0;
  std::vector<int> njt;               // [nJ][nspart]
  std::vector<int> par;               // [nspart]
  std::vector<int16_t> occ;           // [nspart][nshell] shell occupations (empty: not given)
  std::vector<std::vector<int>> poff; // [nJ][nspart+1] partition row offsets inside d(J)
  // densities
  std::vector<uint64_t> keys;         // packed 8-byte keys
  std::unordered_map<uint64_t, int> key_index;
  std::vector<std::vector<RhoBlk>> kblocks;  // per key
  std::vector<double> vals;           // all density values (.trd order)
  // like-particle Hamiltonian, dense per J (d x d, column-major, symmetric), and the layout of
  // the .mat segments it was built from (kept so that new segment values can replace it)
  std::vector<int64_t> hoff;          // [nJ+1] offsets into hdense
  std::vector<double> hdense;
  std::vector<int> seg_J2, seg_np, seg_npr;
  std::vector<int64_t> seg_off;

  int jidx(int J2) const { return (J2 - minJ2) / 2; }
  bool has_J(int J2) const { return J2 >= minJ2 && J2 <= maxJ2 && ((J2 - minJ2) % 2 == 0); }
  int njt_of(int ip, int J2) const { return has_J(J2) ? njt[(size_t)jidx(J2) * nspart + ip] : 0; }
  int dim(int J2) const { return has_J(J2) ? poff[jidx(J2)][nspart] : 0; }
  int find_key(int J2l, int J2r, int sl, int sr, int lam) const;
};

uint64_t pack_key(int b0, int b1, int b2, int b3, int b4);

struct Block {
  int J2a, J2b, da, db;
  int64_t off;
};

// One term of a mixing weight: weights[w] += V(op) * rw, V the multipole value of operator
// op (its index in the problem's op list, renorm applied) and rw the Racah factor.
struct WTerm {
  int64_t w;
  int32_t op;
  double rw;
};

// ---- task lists of the H.v kernels -------------------------------------------
// Y stage: Y_(h,b) = C_h * rho_b^T (row-major d_ar x d_bl), one group per (Y matrix, row tile).
// The densities are re-laid out for it: every sub-block starts at a multiple of 8 elements and
// has its leading dimension rounded up to a multiple of 8 (zero padding), so that groups of 8
// outputs load their coefficients with aligned 16-byte vector loads in FP32 and FP64.
constexpr int KY_TILE_ROWS = 256;  // 128 threads x 2 rows
constexpr int KY_PAD = 8;
constexpr int KA_K_SPLIT = 512;   // stacked rows per k_a tile (longer slabs are split, partial sums added atomically)
struct YGroup {
  int64_t c_base;   // element offset of input block h
  int64_t y_base;   // element offset of the Y matrix
  int32_t m;        // d_ar (rows; leading dimension of C_h)
  int32_t row0;     // first row of the tile
  int32_t b_begin, b_end;  // range in yblks
  int32_t ldy;      // d_bl (row length of Y)
  int32_t pad;
};
struct YBlk {
  int64_t rho;      // offset of the nl x nr (column-major, leading dimension ldr) padded density sub-block
  int32_t ccol;     // first column of C_h (right partition Q_r)
  int32_t ycol;     // first column of Y (left partition Q_l); blocks of one Y matrix ascend in ycol
  int32_t nl, nr;
  int32_t ldr;      // nl rounded up to KY_PAD
  int32_t pad;
};
// Mixing stage k_z: Z_a[P_r rows] = sum_s w_(a,s) Y_s[P_r rows] for the proton operators a of a
// group (output block, J_ar, lam) acting on P_r; written into the stacked operand Zbar.
constexpr int ZMAXS = 32;   // sources (h, b) per group
constexpr int ZMAXA = 16;   // proton operators per group
struct ZGroup {
  int32_t s_begin, s_end;   // range in zsrcs
  int32_t ns;               // sources
  int32_t w_off;            // weights [operator][ns] row-major
};
struct ZSrc {
  int64_t y;                // offset of the source's Y matrix
  int64_t c_base;           // offset of the source's input block h (the fused stage forms Y itself)
  int32_t m;                // d_ar (leading dimension of C_h)
  int32_t b_begin, b_end;   // the Y matrix's density sub-blocks in yblks (ascending ycol)
  int32_t pad;
};
struct ZUnit {              // (group, P_r, column tile)
  int32_t grp;
  int32_t row0, nr;         // rows of P_r in the J_ar space
  int32_t c0, ncols;        // column tile
  int32_t d_bl;             // row length of Y
  int32_t op_begin, op_end; // range in zops
  int32_t ldz;              // row length of Zbar (d_bl rounded up to KZ_PAD)
  int32_t pad;
};
// Zbar rows are padded to a multiple of KZ_PAD elements and every slab starts at a multiple of
// KZ_PAD, so that each row of a 128-column tile starts on a 16-byte boundary (asynchronous
// 16-byte copies into shared memory in k_a, FP32 and FP64); Abar rows likewise (nl -> nlp).
constexpr int KZ_PAD = 4;
constexpr int KZ_UNITS_PER_CTA = 8;   // column tiles of one (group, P_r) per k_z CTA
struct ZOp {
  int64_t z;                // Zbar destination of the operator: element (row rr of P_r, col c) at z + rr*ldz + c
  int32_t wrow;             // weight row within the group
  int32_t pad;
};
// Proton side k_a: out[P_l rows, cols] += Abar (nl x K, column-major, leading dimension nlp) *
// Zbar (K x d_bl, row-major, leading dimension ldz).
constexpr int KA_TILE_COLS = 128;   // output columns per k_a tile (64 threads x 2 columns)
struct ATile {
  int64_t out;      // element offset of out[P_l row 0, col0]
  int32_t ld;       // d_al (leading dimension of the output block)
  int32_t nl;       // rows = nJT(P_l, J_al)
  int32_t col0, ncols;
  int32_t ldz;      // Zbar row length (d_bl rounded up to KZ_PAD)
  int32_t k_begin, k_end;  // range of stacked contribution rows handled by this tile
  int32_t nlp;      // Abar leading dimension (nl rounded up to KZ_PAD; padding rows are zero)
  int64_t zbar;     // offset of Zbar[0, col0]
  int64_t abar;     // offset of Abar[0, 0] of the slab
};
// FP32 form on the tensor cores (k_a_tc): the mixing stage writes each Zbar tile (slab,
// 128-column tile) in the MMA's MN-major swizzled layout; a ZOpTC gives the operator's slab
// (base of its tile 0, tiles kgroups * 1024 floats apart) and its first stacked row.
struct ZOpTC {
  int64_t base;     // float offset of the slab's Zbar tile 0
  int32_t kofs;     // first stacked row of the operator's rows
  int32_t kgroups;  // the slab's stacked rows / 8 (padded)
};
constexpr int KTC_NCLASS = 4;   // N padded to 16, 32, 48, 64 (nl of the proton partition)

// One like-particle segment of the .mat files in the dense per-J matrix it belongs to: value
// (kl, kr) of the segment is H[(ro + kl), (co + kr)] and its mirror of the d x d matrix at h.
struct HSeg {
  int64_t h;        // element offset of the J block in the species' dense H
  int64_t v;        // offset of the segment's values in the staging buffer
  int32_t d, ro, co, nl, nr;
  int32_t species;  // 0: a (protons), 1: b (neutrons)
};

// like-particle part: out_blk = Ha C + C Hb, 64x64 output tiles.
struct LTile {
  int64_t c;        // block offset
  int64_t ha, hb;   // offsets of the dense like-particle matrices
  int32_t da, db;
  int32_t r0, c0;
};

struct DeviceBuffers {
  // FP64 operator data
  // rhoB: the padded neutron densities of the Y stage (the proton densities live in abar)
  double *rhoB = nullptr, *hA = nullptr, *hB = nullptr, *w = nullptr;
  float *rhoB32 = nullptr, *hA32 = nullptr, *hB32 = nullptr, *w32 = nullptr;
  double *abar = nullptr;
  float *abar32 = nullptr;
  float *abar_big = nullptr, *abar_small = nullptr;   // k_a_tc operands (TF32 split)
  ZOpTC *zops_tc = nullptr;
  ATileTC *atiles_tc = nullptr;                       // all classes, class c from atc_off[c]
  int *err = nullptr;                                 // kernels' error word (bounded waits)
  YGroup *ygroups = nullptr;
  YBlk *yblks = nullptr;
  ZGroup *zgroups = nullptr;
  ZSrc *zsrcs = nullptr;
  ZUnit *zunits = nullptr;
  int32_t *zcta = nullptr;   // k_z: first unit of each CTA (consecutive column tiles of one (group, P_r))
  ZOp *zops = nullptr;
  ATile *atiles = nullptr;
  LTile *ltiles = nullptr;
  double *y64 = nullptr, *z64 = nullptr;  // Y and Zbar intermediates, FP64
  float *y32 = nullptr, *z32 = nullptr;   // Y and Zbar (tensor-core tile layout) intermediates, FP32
  float *z32r = nullptr;                  // Zbar in the row-major layout of the SIMT proton side, FP32
  float *x32 = nullptr, *o32 = nullptr;
  double *xin = nullptr, *xout = nullptr;  // host-API staging
  // like-particle segments (a new interaction's values are scattered into the dense H on the GPU)
  HSeg *hsegs = nullptr;                   // all segments of both species
  double *segvals = nullptr;               // their values (species a, then b)
};

}  // namespace nsx

struct nsx_handle {
  int device = 0;
  int J2 = 0, parity = 0;
  nsx::SpeciesPlan A, B;
  std::vector<nsx::Block> blocks;
  int64_t no_state = 0;
  std::vector<uint8_t> lcoef;
  double renorm = 1.0;
  // pn multipole interaction: key (sal, sar, sbl, sbr, lam) -> V * renorm, and -> index in the
  // op list of the problem the handle was created from
  std::unordered_map<uint64_t, double> vop;
  std::unordered_map<uint64_t, int> vop_index;
  int nop = 0;
  std::vector<nsx::WTerm> wterms;  // every weight as a sum of (V, Racah factor) terms, in summation order
  // plan
  std::vector<nsx::YGroup> ygroups;
  std::vector<nsx::YBlk> yblks;
  std::vector<nsx::ZGroup> zgroups;
  std::vector<nsx::ZSrc> zsrcs;
  std::vector<nsx::ZUnit> zunits;
  std::vector<int32_t> zcta;       // k_z CTAs: units [zcta[b], zcta[b+1])
  std::vector<nsx::ZOp> zops;
  std::vector<nsx::ATile> atiles;
  std::vector<double> abar;
  // FP32 tensor-core form of the proton side
  std::vector<nsx::ZOpTC> zops_tc;      // parallel to zops
  std::vector<nsx::ATileTC> atiles_tc;  // grouped by N class, longest first in each
  int64_t atc_off[nsx::KTC_NCLASS + 1] = {};
  std::vector<float> abar_big, abar_small;
  int64_t z32_elems = 0;
  std::vector<double> yrho;        // padded neutron densities read by the Y stage
  std::vector<double> weights;
  std::vector<nsx::LTile> ltiles;
  int64_t y_elems = 0, z_elems = 0;
  int max_ynl = 0, max_ynr = 0, max_anl = 0, max_ldy = 0, max_zns = 0;
  double flops_like = 0, flops_y = 0, flops_mix = 0, flops_a = 0;
  nsx::DeviceBuffers d;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaStream_t stream = nullptr;   // non-blocking stream of nsx_solve / nsx_batch_solve (created on first use)
  // statistics
  int64_t launches = 0, matvecs = 0;
  int64_t stage_launches[NSX_STAGES] = {};
  double stage_ms[NSX_STAGES] = {};
  bool timing = false;
  int last_precision = NSX_FP64;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> stage_events;
  void *lws = nullptr;   // the Lanczos solver's device workspace (lanczos.cu), kept between solves
  // FP32 variant (NSX_FP32_*): requested by nsx_set_fp32_path, and the one in use (0: not chosen)
  int fp32_request = 0, fp32_path = 0;
  // streams and events of the concurrent k_a_tc classes (created on first use)
  cudaStream_t aux[nsx::KTC_NCLASS - 1] = {};
  cudaEvent_t fork_ev = nullptr, join_ev[nsx::KTC_NCLASS - 1] = {};
  cudaEvent_t like_fork = nullptr, like_join = nullptr;   // the like-particle stage on aux[0]
  // output-block shard: the plan covers the output rows of blocks [own_b0, own_b1), rows
  // [row0, row1); shard_first[r] = first block of rank r (world + 1 entries)
  int shard_rank = 0, shard_world = 1;
  int own_b0 = 0, own_b1 = INT_MAX;
  int64_t row0 = 0, row1 = 0;
  std::vector<int> shard_first;
  std::vector<double> block_flops;   // per output block: flops of its rows' product (estimate of the split)
  nsx_exchange_fn exch = nullptr;
  void *exch_user = nullptr;
};

namespace nsx {
// Terms of a compressed pn interaction read from a .dop file (compress.cpp).
struct DopArrays {
  std::vector<int32_t> lam2, parity, eig;
  std::vector<double> e, u;
  std::vector<uint8_t> shells;
  nsx_dop view() {
    nsx_dop d;
    d.nterms = (int32_t)e.size();
    d.lam2 = lam2.data();
    d.parity = parity.data();
    d.eig = eig.data();
    d.e = e.data();
    d.shells = shells.data();
    d.u = u.data();
    return d;
  }
};
// Offset of Zbar in a caller-provided FP64 scratch buffer that holds Y then Zbar: Y's length
// rounded up to 32 elements, so that Zbar starts on a 256-byte boundary (k_a copies its rows
// with 16-byte asynchronous copies).
inline int64_t zbar_scratch_offset(const nsx_handle *h) { return (h->y_elems + 31) / 32 * 32; }
void build_plan(nsx_handle *h, const nsx_problem *p);
std::vector<int> split_blocks(const std::vector<double> &cost, int world);
void require_full_product(const nsx_handle *h);
void set_interaction(nsx_handle *h, const double *op_vals, int32_t nop, const double *a_seg_vals, int64_t a_nvals,
                     const double *b_seg_vals, int64_t b_nvals);
void upload(nsx_handle *h);
void upload_interaction(nsx_handle *h, const double *a_seg_vals, const double *b_seg_vals);
cudaStream_t solve_stream(nsx_handle *h);
void ensure_precision(nsx_handle *h, int precision);
void set_fp32_path(nsx_handle *h, int path);
void release(nsx_handle *h);
void matvec_device(nsx_handle *h, const double *x, double *y, int precision, cudaStream_t s);
void matvec_fp64_with_scratch(nsx_handle *h, const double *x, double *y, double *scratch, cudaStream_t s);
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[NSX_STAGES], double flops[NSX_STAGES]);
void flush_stage_events(nsx_handle *h);
void check_device_error(nsx_handle *h);
void write_state(const nsx_handle *h, const char *prefix, const nsx_state *st, const double *evals,
                 const double *evecs, int nev, const char *intfile, int T2);
void read_state(const nsx_handle *h, const char *prefix, nsx_state *st);
void expectation_matrix(nsx_handle *h, const double *vecs, int nvec, int precision, double *out);
void xpct_files(nsx_handle *h, const char *xvc_path, const char *out_prefix, int precision);
void release_lanczos(nsx_handle *h);
void write_results(const nsx_handle *h, const char *prefix, const double *evals, const double *evecs, int nev,
                   int iterations, const char *intfile, int T2);
double sixj(int a, int b, int c, int d, int e, int f);
double racah_w(int j1, int j2, int j3, int j4, int J, int K);
}  // namespace nsx
