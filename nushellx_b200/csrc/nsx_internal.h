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

// ---- pn table (drdbh) -----------------------------------------------------------
struct TabEnt {
  int bk, hb;       // neutron density key, input block
  double w;         // V_lam * renorm * Racah weight
};
struct TabRow {     // one (output block, J_ar, proton density key)
  int bl, jar, ak, lam;
  std::vector<TabEnt> e;
};

// ---- plan of the fused pn kernel k_pn ---------------------------------------------
constexpr int MAXA = 16;    // proton operators per work item
constexpr int MAXS = 32;    // sources (h, b) per group
struct Group {              // (output block, J_ar, lam): shared by the block's tasks
  int32_t d_ar;             // proton rows of the Y operands (d_a(J_ar))
  int32_t nsrc;             // sources of the group (<= MAXS)
  int32_t na;               // proton operators of the group (weight rows)
  int32_t w_off;            // weights [na][nsrc], row-major
  int32_t pr_begin, pr_end; // range in prwork
  int32_t bt_begin, bt_end; // range in batches (row batches of the group's items)
};
struct Batch {              // consecutive work items whose rows fit one shared-memory row batch
  int32_t it_begin, it_end; // range in prwork
  int32_t row0, nrows;      // proton rows [row0, row0 + nrows), nrows <= batch_rows
};
struct TGroup {             // a group as seen by one task: the sources present at Q_l
  int32_t grp;
  int32_t src_begin, src_end;
};
struct TSrc {               // a group source present in a task's column chunk
  int32_t piece_begin, piece_end;  // range in pieces
  uint32_t cover;           // chunk columns the pieces cover (bit c)
  int32_t sidx;             // source index within the group
};
struct Piece {              // Y_s[:, cs..cs+w) = C_h[:, Q_r cols] rho_b[rows.., Q_r]^T
  int64_t c;                // offset of C_h[0, first column of Q_r]
  int64_t rho;              // offset of rho_b(Q_l, Q_r) element (first row of the piece, col 0)
  int32_t ld;               // n(Q_l): leading dimension of the density block
  int32_t nr;               // n(Q_r)
  int32_t cs, w;            // chunk columns [cs, cs+w)
};
struct PrWork {             // <= item_rows rows of one proton right partition P_r
  int32_t row0, nr;
  int32_t a_begin, a_end;   // range in aops (<= MAXA)
};
struct AOp {                // proton density block rho_a(P_l, P_r), rows chunk of P_r
  int64_t rho;              // offset of element (0, chunk row 0); block nl x n(P_r) column-major
  int32_t ld, out_row0, nl, wrow;
};
struct PnTask {             // output block, CH consecutive neutron states (columns)
  int64_t out;              // offset of out[row 0, first column]
  int32_t d_al, nq;
  int32_t g_begin, g_end;   // range in tgroups
};
struct PnPlan {
  int CH = 8;
  int item_rows = 4;        // = 32 / CH: one row per lane in stage 2
  int batch_rows = 64;      // proton rows of Y held in shared memory at a time
  std::vector<Group> groups;
  std::vector<TGroup> tgroups;
  std::vector<TSrc> tsrcs;
  std::vector<Piece> pieces;
  std::vector<PrWork> prwork;
  std::vector<Batch> batches;
  std::vector<AOp> aops;
  std::vector<PnTask> tasks;
  std::vector<double> task_cost;
  std::vector<double> weights;
  int max_dar = 0, max_dal = 0, max_nsrc = 0, max_nl = 0;
};
struct PnDevice {           // device copy of one plan (typed operand data lives in DeviceBuffers)
  Group *groups = nullptr;
  TGroup *tgroups = nullptr;
  TSrc *tsrcs = nullptr;
  Piece *pieces = nullptr;
  PrWork *prwork = nullptr;
  Batch *batches = nullptr;
  AOp *aops = nullptr;
  PnTask *tasks = nullptr;
  void *weights = nullptr;  // T[]
  int *counter = nullptr;
  unsigned long long *cycles = nullptr;  // [4] sub-stage SM cycles (timing only)
  int grid = 0;
  size_t smem = 0;
};

// like-particle part: out_blk = Ha C + C Hb, 64x64 output tiles.
struct LTile {
  int64_t c;        // block offset
  int64_t ha, hb;   // offsets of the dense like-particle matrices
  int32_t da, db;
  int32_t r0, c0;
};

struct DeviceBuffers {
  double *rhoA = nullptr, *rhoB = nullptr, *hA = nullptr, *hB = nullptr;
  float *rhoA32 = nullptr, *rhoB32 = nullptr, *hA32 = nullptr, *hB32 = nullptr;
  LTile *ltiles = nullptr;
  PnDevice pn64, pn32;
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
  std::vector<nsx::LTile> ltiles;
  nsx::PnPlan pn64, pn32;   // CH = 8 (FP64) and CH = 16 (FP32)
  int64_t y_elems = 0;      // Y operand elements of one H.v (algorithmic)
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
void stage_bytes_flops(const nsx_handle *h, int precision, double bytes[4], double flops[4]);
void flush_stage_events(nsx_handle *h);
double sixj(int a, int b, int c, int d, int e, int f);
std::vector<TabRow> pn_table(const nsx_handle *h);
void build_pn_plan(const nsx_handle *h, const std::vector<TabRow> &table, int CH, int batch_rows, PnPlan &P);
double racah_w(int j1, int j2, int j3, int j4, int J, int K);
}  // namespace nsx
