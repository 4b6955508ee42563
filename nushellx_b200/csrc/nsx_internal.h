// Internal structures of libnsx: host-side plan of one J-scheme pn problem and
// the device buffers the H.v kernels and the Lanczos driver work on.
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <unordered_map>
#include <cuda_runtime.h>
#include "nsx.h"

namespace nsx {

struct Error {
  int code;
  std::string msg;
};
[[noreturn]] void fail(int code, const std::string &msg);
void check_cuda(cudaError_t e, const char *what);
#define NSX_CUDA(x) ::nsx::check_cuda((x), #x)

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
  std::vector<std::vector<int>> poff; // [nJ][nspart+1] partition row offsets inside d(J)
  // densities
  std::vector<uint64_t> keys;         // packed 8-byte keys
  std::unordered_map<uint64_t, int> key_index;
  std::vector<std::vector<RhoBlk>> kblocks;  // per key
  std::vector<double> vals;           // all density values (.trd order)
  // like-particle Hamiltonian, dense per J (d x d, column-major, symmetric)
  std::vector<int64_t> hoff;          // [nJ+1] offsets into hdense
  std::vector<double> hdense;

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

// ---- task lists of the H.v kernels -------------------------------------------
// Y stage: Y_(h,b) = C_h * rho_b^T, one group per (Y matrix, row tile).
struct YGroup {
  int64_t c_base;   // element offset of input block h
  int64_t y_base;   // element offset of the Y matrix (d_ar x d_bl, column-major)
  int32_t m;        // d_ar (rows, leading dimension of C_h and Y)
  int32_t row0;     // first row of the tile
  int32_t b_begin, b_end;  // range in yblks
};
struct YBlk {
  int64_t rho;      // offset of the nl x nr (column-major) density sub-block
  int32_t ccol;     // first column of C_h (right partition Q_r)
  int32_t ycol;     // first column of Y (left partition Q_l)
  int32_t nl, nr;
};
// A stage: output tile (block, left proton partition P_l, column range).
struct ATile {
  int64_t out;      // element offset of out[P_l row 0, col0] in the output vector
  int32_t ld;       // d_al (leading dimension of the output block)
  int32_t nl;       // rows of the tile = nJT(P_l, J_al)
  int32_t col0, ncols;
  int32_t c_begin, c_end;  // range in contribs
};
struct AContrib {
  int64_t rho;      // offset of the nl x nr proton density sub-block (column-major)
  int32_t nr;       // nJT(P_r, J_ar)
  int32_t m_begin, m_end;  // range in mixes
};
struct AMix {
  int64_t y;        // offset of Y_(h,b)[P_r row 0, col 0]
  int32_t ld;       // d_ar (leading dimension of that Y matrix)
  int32_t wi;       // index into the weight array
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
  double *rhoA = nullptr, *rhoB = nullptr, *hA = nullptr, *hB = nullptr, *w = nullptr;
  float *rhoA32 = nullptr, *rhoB32 = nullptr, *hA32 = nullptr, *hB32 = nullptr, *w32 = nullptr;
  YGroup *ygroups = nullptr;
  YBlk *yblks = nullptr;
  ATile *atiles = nullptr;
  AContrib *acontribs = nullptr;
  AMix *amixes = nullptr;
  LTile *ltiles = nullptr;
  double *y64 = nullptr;   // Y intermediates, FP64
  float *y32 = nullptr;    // Y intermediates, FP32
  float *x32 = nullptr, *o32 = nullptr;
  double *xin = nullptr, *xout = nullptr;  // host-API staging
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
  // pn multipole interaction: key (sal, sar, sbl, sbr, lam) -> V * renorm
  std::unordered_map<uint64_t, double> vop;
  // plan
  std::vector<nsx::YGroup> ygroups;
  std::vector<nsx::YBlk> yblks;
  std::vector<nsx::ATile> atiles;
  std::vector<nsx::AContrib> acontribs;
  std::vector<nsx::AMix> amixes;
  std::vector<double> weights;
  std::vector<nsx::LTile> ltiles;
  int64_t y_elems = 0;
  int max_ynl = 0, max_ynr = 0, max_anl = 0, max_anr = 0, max_mix = 0;
  double flops_like = 0, flops_y = 0, flops_mix = 0, flops_a = 0;
  nsx::DeviceBuffers d;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // statistics
  int64_t launches = 0, matvecs = 0;
  int64_t stage_launches[4] = {0, 0, 0, 0};
  double stage_ms[4] = {0, 0, 0, 0};
  bool timing = false;
  int last_precision = NSX_FP64;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> stage_events;
};

namespace nsx {
void build_plan(nsx_handle *h, const nsx_problem *p);
void upload(nsx_handle *h);
void ensure_precision(nsx_handle *h, int precision);
void release(nsx_handle *h);
void matvec_device(nsx_handle *h, const double *x, double *y, int precision, cudaStream_t s);
void matvec_fp64_with_scratch(nsx_handle *h, const double *x, double *y, double *Y, cudaStream_t s);
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[4], double flops[4]);
void flush_stage_events(nsx_handle *h);
double sixj(int a, int b, int c, int d, int e, int f);
double racah_w(int j1, int j2, int j3, int j4, int J, int K);
}  // namespace nsx
