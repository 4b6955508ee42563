// Host-side setup of one J-scheme pn problem (the B200 counterpart of the
// reference's Lnz_TRD + drdbh, src/NuLnz/NuCoreX.f90:807-1367 and 1428-1577):
// species tables, the block list and parity mask, the Racah-weighted pn
// interaction table, and the task lists of the three H.v stages.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <array>
#include <map>
#include <set>
#include "nsx_internal.h"

namespace nsx {

uint64_t pack_key(int b0, int b1, int b2, int b3, int b4) {
  return (uint64_t)(uint8_t)b0 | ((uint64_t)(uint8_t)b1 << 8) | ((uint64_t)(uint8_t)b2 << 16) |
         ((uint64_t)(uint8_t)b3 << 24) | ((uint64_t)(uint8_t)b4 << 32);
}

int SpeciesPlan::find_key(int J2l, int J2r, int sl, int sr, int lam) const {
  auto it = key_index.find(pack_key(J2l, J2r, sl, sr, lam));
  return it == key_index.end() ? -1 : it->second;
}

// ---- angular momentum (twice-values), Racah's closed forms -------------------
static double fact_half(int n2) {  // (n2/2)!
  static std::vector<double> tab;
  if (tab.empty()) {
    tab.resize(171);
    tab[0] = 1.0;
    for (int i = 1; i < 171; ++i) tab[i] = tab[i - 1] * i;
  }
  int n = n2 / 2;
  if (n < 0 || n > 170) fail(NSX_E_ARG, "angular momentum too large for the factorial table");
  return tab[n];
}
static bool tri(int a, int b, int c) { return std::abs(a - b) <= c && c <= a + b && ((a + b + c) % 2 == 0); }
static double delta(int a, int b, int c) {
  return fact_half(a + b - c) * fact_half(a - b + c) * fact_half(-a + b + c) / fact_half(a + b + c + 2);
}
// Wigner 6-j {a b c; d e f}, Racah formula (Edmonds 6.3.7).
double sixj(int a, int b, int c, int d, int e, int f) {
  if (!tri(a, b, c) || !tri(a, e, f) || !tri(d, b, f) || !tri(d, e, c)) return 0.0;
  double pre = std::sqrt(delta(a, b, c) * delta(a, e, f) * delta(d, b, f) * delta(d, e, c));
  int tlo = std::max(std::max(a + b + c, a + e + f), std::max(d + b + f, d + e + c));
  int thi = std::min(std::min(a + b + d + e, b + c + e + f), a + c + d + f);
  double s = 0.0;
  for (int t = tlo; t <= thi; t += 2) {
    double num = ((t / 2) % 2 ? -1.0 : 1.0) * fact_half(t + 2);
    double den = fact_half(t - a - b - c) * fact_half(t - a - e - f) * fact_half(t - d - b - f) *
                 fact_half(t - d - e - c) * fact_half(a + b + d + e - t) * fact_half(b + c + e + f - t) *
                 fact_half(a + c + d + f - t);
    s += num / den;
  }
  return pre * s;
}
// W(j1 j2 j3 j4; J K) = (-1)^((j1+j2+j3+j4)/2) {j1 j2 J; j4 j3 K}  (src/NuCommon/NuCommon.f90:3255-3265)
double racah_w(int j1, int j2, int j3, int j4, int J, int K) {
  double ph = (((j1 + j2 + j3 + j4) / 2) % 2) ? -1.0 : 1.0;
  return ph * sixj(j1, j2, J, j4, j3, K);
}
// (-1)^((Jal+Jbr-J-lam)/2) W(Jal Jbl Jar Jbr; J lam) sqrt(lam+1)  (src/NuLnz/NuCoreX.f90:1114-1126)
static double racah_weight(int Jal, int Jbl, int Jar, int Jbr, int J, int lam) {
  double w = racah_w(Jal, Jbl, Jar, Jbr, J, lam);
  if (w == 0.0) return 0.0;
  int e = (Jal + Jbr - J - lam) / 2;
  double ph = (e % 2) ? -1.0 : 1.0;
  return ph * w * std::sqrt((double)lam + 1.0);
}

// ---- species ------------------------------------------------------------------
static void fill_hdense(SpeciesPlan &S, const double *seg_vals);

static void load_species(SpeciesPlan &S, const nsx_species &s, const char *name) {
  if (s.nspart <= 0 || s.maxJ2 < s.minJ2 || ((s.maxJ2 - s.minJ2) % 2) != 0)
    fail(NSX_E_ARG, std::string("species ") + name + ": bad partition count or J range");
  S.nspart = s.nspart;
  S.minJ2 = s.minJ2;
  S.maxJ2 = s.maxJ2;
  S.nJ = (s.maxJ2 - s.minJ2) / 2 + 1;
  S.shell_first = s.shell_first;
  S.nshell = s.nshell;
  S.njt.assign(s.njt, s.njt + (size_t)S.nJ * S.nspart);
  S.par.assign(s.parity, s.parity + S.nspart);
  if (s.occ) S.occ.assign(s.occ, s.occ + (size_t)S.nspart * std::max(S.nshell, 0));
  else S.occ.clear();
  for (int v : S.njt)
    if (v < 0) fail(NSX_E_ARG, std::string("species ") + name + ": negative nJT");
  S.poff.assign(S.nJ, std::vector<int>(S.nspart + 1, 0));
  for (int j = 0; j < S.nJ; ++j)
    for (int p = 0; p < S.nspart; ++p) S.poff[j][p + 1] = S.poff[j][p] + S.njt[(size_t)j * S.nspart + p];
  // densities: walk the masks in .trd order (src/NuCommonX/NuCommonX.f90:609-636 next_ij)
  S.keys.resize(s.nkeys);
  S.kblocks.assign(s.nkeys, {});
  int64_t nvals = s.nkeys ? s.val_off[s.nkeys] : 0;
  S.vals.assign(s.vals, s.vals + nvals);
  for (int k = 0; k < s.nkeys; ++k) {
    const uint8_t *kb = s.keys + 8 * (size_t)k;
    uint64_t key = pack_key(kb[0], kb[1], kb[2], kb[3], kb[4]);
    S.keys[k] = key;
    S.key_index[key] = k;
    int J2l = kb[0], J2r = kb[1];
    int64_t v = s.val_off[k];
    for (int r = 0; r < S.nspart; ++r) {
      const uint32_t *m = s.masks + ((size_t)k * S.nspart + r) * s.words;
      for (int l = 0; l < S.nspart; ++l) {
        if (!((m[l / 32] >> (l % 32)) & 1u)) continue;
        int nl = S.njt_of(l, J2l), nr = S.njt_of(r, J2r);
        if (nl == 0 || nr == 0) fail(NSX_E_ARG, std::string("species ") + name + ": density block on an empty partition");
        S.kblocks[k].push_back({l, r, v});
        v += (int64_t)nl * nr;
      }
    }
    if (v != s.val_off[k + 1]) fail(NSX_E_ARG, std::string("species ") + name + ": density key size disagrees with its masks");
  }
  // like-particle Hamiltonian: dense per J from the symmetric segments
  S.hoff.assign(S.nJ + 1, 0);
  for (int j = 0; j < S.nJ; ++j) {
    int64_t d = S.poff[j][S.nspart];
    S.hoff[j + 1] = S.hoff[j] + d * d;
  }
  S.seg_J2.assign(s.seg_J2, s.seg_J2 + s.nseg);
  S.seg_np.assign(s.seg_np, s.seg_np + s.nseg);
  S.seg_npr.assign(s.seg_npr, s.seg_npr + s.nseg);
  S.seg_off.assign(s.seg_off, s.seg_off + s.nseg + 1);
  for (int g = 0; g < s.nseg; ++g) {
    int J2 = S.seg_J2[g];
    if (!S.has_J(J2)) fail(NSX_E_ARG, std::string("species ") + name + ": segment J out of range");
    int np = S.seg_np[g] - 1, npr = S.seg_npr[g] - 1;
    if (np < 0 || npr < 0 || np >= S.nspart || npr >= S.nspart || npr < np)
      fail(NSX_E_ARG, std::string("species ") + name + ": bad segment partitions");
    int nl = S.njt_of(np, J2), nr = S.njt_of(npr, J2);
    if ((int64_t)nl * nr != S.seg_off[g + 1] - S.seg_off[g])
      fail(NSX_E_ARG, std::string("species ") + name + ": segment size mismatch");
  }
  fill_hdense(S, s.seg_vals);
}

// Dense like-particle H per J from segment values laid out as recorded by load_species.
static void fill_hdense(SpeciesPlan &S, const double *seg_vals) {
  S.hdense.assign(S.hoff[S.nJ], 0.0);
  for (size_t g = 0; g < S.seg_J2.size(); ++g) {
    int J2 = S.seg_J2[g];
    int j = S.jidx(J2);
    int np = S.seg_np[g] - 1, npr = S.seg_npr[g] - 1;
    int nl = S.njt_of(np, J2), nr = S.njt_of(npr, J2);
    int64_t d = S.poff[j][S.nspart];
    double *H = S.hdense.data() + S.hoff[j];
    const double *M = seg_vals + S.seg_off[g];
    int ro = S.poff[j][np], co = S.poff[j][npr];
    // matrix(dimptr, dimpt): value[kr + nr*kl] = H[(np,kl), (npr,kr)]
    for (int kl = 0; kl < nl; ++kl)
      for (int kr = 0; kr < nr; ++kr) {
        double v = M[kr + (int64_t)nr * kl];
        H[(ro + kl) + d * (co + kr)] = v;
        H[(co + kr) + d * (ro + kl)] = v;
      }
  }
}

void set_interaction(nsx_handle *h, const double *op_vals, int32_t nop, const double *a_seg_vals, int64_t a_nvals,
                     const double *b_seg_vals, int64_t b_nvals) {
  if (nop != h->nop) fail(NSX_E_ARG, "op_vals holds " + std::to_string(nop) + " values; the handle was created with " +
                                         std::to_string(h->nop) + " operators");
  if (nop > 0 && !op_vals) fail(NSX_E_ARG, "null op_vals");
  const int64_t na = h->A.seg_off.empty() ? 0 : h->A.seg_off.back();
  const int64_t nb = h->B.seg_off.empty() ? 0 : h->B.seg_off.back();
  if (a_nvals != na || b_nvals != nb)
    fail(NSX_E_ARG, "segment value counts " + std::to_string(a_nvals) + ", " + std::to_string(b_nvals) +
                        " differ from the handle's " + std::to_string(na) + ", " + std::to_string(nb));
  if ((na > 0 && !a_seg_vals) || (nb > 0 && !b_seg_vals)) fail(NSX_E_ARG, "null segment values");
  std::vector<double> v(nop);
  for (int i = 0; i < nop; ++i) {
    double x = op_vals[i];
    if (!std::isfinite(x)) fail(NSX_E_ARG, "op_vals holds a value that is not finite");
    if (std::fabs(x) < 1e-10) x = 0.0;
    v[i] = x * h->renorm;
  }
  for (auto &kv : h->vop_index) h->vop[kv.first] = v[kv.second];
  std::fill(h->weights.begin(), h->weights.end(), 0.0);
  for (const WTerm &t : h->wterms) h->weights[t.w] += v[t.op] * t.rw;
  // a device handle fills its dense like-particle H from the segment values on the GPU
  // (upload_interaction); the host copy is the plan's and stays as built
  if (h->device < 0) {
    fill_hdense(h->A, a_seg_vals);
    fill_hdense(h->B, b_seg_vals);
  }
}

void build_plan(nsx_handle *h, const nsx_problem *p) {
  h->J2 = p->J2;
  h->parity = p->parity;
  h->renorm = p->renorm;
  load_species(h->A, p->a, "a");
  load_species(h->B, p->b, "b");
  SpeciesPlan &A = h->A, &B = h->B;
  // pn multipole interaction (src/NuLnz/NuCoreX.f90:1133-1142: tiny values zeroed, times renorm)
  h->nop = p->nop;
  for (int i = 0; i < p->nop; ++i) {
    const uint8_t *kb = p->op_keys + 8 * (size_t)i;
    double v = p->op_vals[i];
    if (std::fabs(v) < 1e-10) v = 0.0;
    const uint64_t key = pack_key(kb[0], kb[1], kb[2], kb[3], kb[4]);
    h->vop[key] = v * p->renorm;
    h->vop_index[key] = i;
  }
  // block list (src/NuLnz/NuCoreX.f90:926-988): ascending (2Ja, 2Jb)
  const int J2 = p->J2;
  h->blocks.clear();
  for (int ja = A.minJ2; ja <= A.maxJ2; ja += 2) {
    int lo = std::max(std::abs(ja - J2), B.minJ2);
    int hi = std::min(ja + J2, B.maxJ2);
    lo += (lo - B.minJ2) % 2;
    for (int jb = lo; jb <= hi; jb += 2) h->blocks.push_back({ja, jb, A.dim(ja), B.dim(jb), 0});
  }
  int64_t off = 0;
  for (auto &b : h->blocks) {
    b.off = off;
    off += (int64_t)b.da * b.db;
  }
  h->no_state = off;
  if (off == 0) fail(NSX_E_ARG, "empty J-scheme space");
  // output-block shard: this handle plans the rows of blocks [own_b0, own_b1) only
  const int nbl = (int)h->blocks.size();
  const int ob0 = std::min(std::max(h->own_b0, 0), nbl), ob1 = std::min(std::max(h->own_b1, ob0), nbl);
  auto owned = [&](int bl) { return bl >= ob0 && bl < ob1; };
  h->row0 = ob0 < nbl ? h->blocks[ob0].off : off;
  h->row1 = ob1 < nbl ? h->blocks[ob1].off : off;
  // the flops of every block's rows come from the plan of the whole product (a shard's plan
  // keeps those of the whole plan it was split from)
  const bool whole = ob0 == 0 && ob1 == nbl;
  if (whole) h->block_flops.assign(nbl, 0.0);
  std::map<std::pair<int, int>, int> bidx;
  for (size_t i = 0; i < h->blocks.size(); ++i) bidx[{h->blocks[i].J2a, h->blocks[i].J2b}] = (int)i;
  // parity mask lcoef (src/NuLnz/NuCoreX.f90:996-1030)
  h->lcoef.assign(off, 0);
  for (auto &b : h->blocks) {
    int64_t n = b.off;
    for (int pb = 0; pb < B.nspart; ++pb)
      for (int kb = 0; kb < B.njt_of(pb, b.J2b); ++kb)
        for (int pa = 0; pa < A.nspart; ++pa)
          for (int ka = 0; ka < A.njt_of(pa, b.J2a); ++ka, ++n)
            h->lcoef[n] = (p->parity == 0 || A.par[pa] * B.par[pb] == p->parity) ? 1 : 0;
  }
  // key indices: a-keys by (Jl, Jr); b-keys by (Jl, Jr, lam)
  std::map<std::pair<int, int>, std::vector<int>> akeys;
  std::map<std::tuple<int, int, int>, std::vector<int>> bkeys;
  for (int k = 0; k < (int)A.keys.size(); ++k) {
    uint64_t key = A.keys[k];
    akeys[{(int)(key & 255), (int)((key >> 8) & 255)}].push_back(k);
  }
  for (int k = 0; k < (int)B.keys.size(); ++k) {
    uint64_t key = B.keys[k];
    bkeys[{(int)(key & 255), (int)((key >> 8) & 255), (int)((key >> 32) & 255)}].push_back(k);
  }
  // like-particle tiles and flops (segment count, src/NuCommonX/NuCommonX.f90:1009-1104)
  h->ltiles.clear();
  h->flops_like = 0;
  for (int bl = ob0; bl < ob1; ++bl) {
    const Block &b = h->blocks[bl];
    if (b.da == 0 || b.db == 0) continue;
    for (int r0 = 0; r0 < b.da; r0 += 64)
      for (int c0 = 0; c0 < b.db; c0 += 64)
        h->ltiles.push_back({b.off, A.hoff[A.jidx(b.J2a)], B.hoff[B.jidx(b.J2b)], b.da, b.db, r0, c0});
  }
  for (int g = 0; g < p->a.nseg; ++g) {
    int J2s = p->a.seg_J2[g];
    double nn = (double)(p->a.seg_off[g + 1] - p->a.seg_off[g]) * (p->a.seg_np[g] == p->a.seg_npr[g] ? 1 : 2);
    for (int bl = 0; bl < nbl; ++bl)
      if (h->blocks[bl].J2a == J2s) {
        if (whole) h->block_flops[bl] += 2.0 * nn * h->blocks[bl].db;
        if (owned(bl)) h->flops_like += 2.0 * nn * h->blocks[bl].db;
      }
  }
  for (int g = 0; g < p->b.nseg; ++g) {
    int J2s = p->b.seg_J2[g];
    double nn = (double)(p->b.seg_off[g + 1] - p->b.seg_off[g]) * (p->b.seg_np[g] == p->b.seg_npr[g] ? 1 : 2);
    for (int bl = 0; bl < nbl; ++bl)
      if (h->blocks[bl].J2b == J2s) {
        if (whole) h->block_flops[bl] += 2.0 * nn * h->blocks[bl].da;
        if (owned(bl)) h->flops_like += 2.0 * nn * h->blocks[bl].da;
      }
  }

  // ---- pn table (drdbh, src/NuLnz/NuCoreX.f90:1428-1577) ----------------------
  // Rows: (output block, J_ar, proton density key a) with entries (neutron key b, input block h, weight).
  struct Entry { int bk, hb; double w; int op; double rw; };
  struct Row { int bl, jar, ak, lam; std::vector<Entry> e; };
  std::vector<Row> table;
  for (size_t bl = 0; bl < h->blocks.size(); ++bl) {
    const Block &ob = h->blocks[bl];
    if (ob.da == 0 || ob.db == 0) continue;
    for (int jar = A.minJ2; jar <= A.maxJ2; jar += 2) {
      auto ait = akeys.find({ob.J2a, jar});
      if (ait == akeys.end()) continue;
      for (int ak : ait->second) {
        if (A.kblocks[ak].empty()) continue;
        uint64_t akey = A.keys[ak];
        int sal = (akey >> 16) & 255, sar = (akey >> 24) & 255, lam = (akey >> 32) & 255;
        Row row{(int)bl, jar, ak, lam, {}};
        int jbrn = std::max(std::abs(ob.J2b - lam), std::abs(jar - J2));
        int jbrx = std::min(std::min(ob.J2b + lam, jar + J2), B.maxJ2);
        for (int jbr = jbrn; jbr <= jbrx; jbr += 2) {
          if (!B.has_J(jbr)) continue;
          auto hit = bidx.find({jar, jbr});
          if (hit == bidx.end()) continue;
          const Block &ib = h->blocks[hit->second];
          if (ib.da == 0 || ib.db == 0) continue;
          double rw = racah_weight(ob.J2a, ob.J2b, jar, jbr, J2, lam);
          if (rw == 0.0) continue;
          auto bit = bkeys.find({ob.J2b, jbr, lam});
          if (bit == bkeys.end()) continue;
          for (int bk : bit->second) {
            uint64_t bkey = B.keys[bk];
            int sbl = (bkey >> 16) & 255, sbr = (bkey >> 24) & 255;
            // operators of the problem's list are kept even where V is zero, so that a new
            // interaction (nsx_set_interaction) finds a slot for every one of them
            const uint64_t okey = pack_key(sal, sar, sbl, sbr, lam);
            auto vit = h->vop.find(okey);
            if (vit == h->vop.end()) continue;
            if (B.kblocks[bk].empty()) continue;
            row.e.push_back({bk, hit->second, vit->second * rw, h->vop_index[okey], rw});
          }
        }
        if (!row.e.empty()) table.push_back(std::move(row));
      }
    }
  }
  // ---- Y operands: one row-major d_ar x d_bl matrix per (input block h, neutron key b, layer) ----
  // A layer of a neutron density holds at most one sub-block per left partition (the Y stage
  // gives each output column one sub-block).  The densities of the reference's files have one
  // layer; combined operators (the compressed interaction) sum several densities and get one
  // layer per sub-block of a left partition, each a source of its own with the same weight.
  std::vector<std::vector<int>> blayer(B.keys.size());
  std::vector<int> nlayer(B.keys.size(), 1);
  for (size_t bk = 0; bk < B.keys.size(); ++bk) {
    std::map<int, int> seen;   // left partition -> sub-blocks so far
    for (const RhoBlk &rb : B.kblocks[bk]) {
      const int L = seen[rb.pl]++;
      blayer[bk].push_back(L);
      nlayer[bk] = std::max(nlayer[bk], L + 1);
    }
  }
  // Y flops of every output block's rows (for the shard split; the mixing and proton-side flops
  // are added where the plan forms them), then the table keeps the owned blocks' rows only:
  // every task list below follows from it.  A Y matrix counts for every block that reads it (a
  // shard that owns two such blocks forms it once).
  if (whole) {
    std::vector<std::vector<double>> lnnz(B.keys.size());
    for (size_t bk = 0; bk < B.keys.size(); ++bk) {
      lnnz[bk].assign(nlayer[bk], 0.0);
      const int J2bl = (int)(B.keys[bk] & 255), J2br = (int)((B.keys[bk] >> 8) & 255);
      for (size_t bi = 0; bi < B.kblocks[bk].size(); ++bi) {
        const RhoBlk &rb = B.kblocks[bk][bi];
        lnnz[bk][blayer[bk][bi]] += (double)B.njt_of(rb.pl, J2bl) * B.njt_of(rb.pr, J2br);
      }
    }
    std::set<std::array<int, 4>> yseen;   // (output block, input block, neutron key, layer)
    for (const Row &r : table)
      for (const Entry &e : r.e)
        for (int L = 0; L < nlayer[e.bk]; ++L)
          if (yseen.insert({r.bl, e.hb, e.bk, L}).second)
            h->block_flops[r.bl] += 2.0 * h->blocks[e.hb].da * lnnz[e.bk][L];
  }
  table.erase(std::remove_if(table.begin(), table.end(), [&](const Row &r) { return !owned(r.bl); }), table.end());
  std::map<std::tuple<int, int, int>, int> ymat;
  std::vector<std::tuple<int, int, int>> ymats;
  std::vector<int64_t> yoff;
  int64_t ytot = 0;
  auto get_ymat = [&](int hb, int bk, int L) {
    auto it = ymat.find({hb, bk, L});
    if (it != ymat.end()) return it->second;
    int id = (int)ymats.size();
    ymat[{hb, bk, L}] = id;
    ymats.push_back({hb, bk, L});
    yoff.push_back(ytot);
    ytot += (int64_t)h->blocks[hb].da * B.dim((int)(B.keys[bk] & 255));
    return id;
  };
  for (const Row &r : table)
    for (const Entry &e : r.e)
      for (int L = 0; L < nlayer[e.bk]; ++L) get_ymat(e.hb, e.bk, L);
  h->ygroups.clear();
  h->yblks.clear();
  h->yrho.clear();
  h->flops_y = 0;
  std::unordered_map<int64_t, int64_t> yrho_at;  // .trd value offset -> padded offset
  std::vector<int32_t> ymat_b0(ymats.size()), ymat_b1(ymats.size());
  for (size_t y = 0; y < ymats.size(); ++y) {
    const int hb = std::get<0>(ymats[y]), bk = std::get<1>(ymats[y]), layer = std::get<2>(ymats[y]);
    const Block &ib = h->blocks[hb];
    int J2bl = (int)(B.keys[bk] & 255), J2br = (int)((B.keys[bk] >> 8) & 255);
    int b0 = (int)h->yblks.size();
    double nnz = 0;
    for (size_t bi = 0; bi < B.kblocks[bk].size(); ++bi) {
      if (blayer[bk][bi] != layer) continue;
      const RhoBlk &rb = B.kblocks[bk][bi];
      YBlk yb;
      yb.ccol = B.poff[B.jidx(J2br)][rb.pr];
      yb.ycol = B.poff[B.jidx(J2bl)][rb.pl];
      yb.nl = B.njt_of(rb.pl, J2bl);
      yb.nr = B.njt_of(rb.pr, J2br);
      yb.ldr = (yb.nl + KY_PAD - 1) / KY_PAD * KY_PAD;
      yb.pad = 0;
      auto it = yrho_at.find(rb.voff);
      if (it == yrho_at.end()) {
        int64_t at = (int64_t)h->yrho.size();
        h->yrho.resize(at + (size_t)yb.ldr * yb.nr, 0.0);
        for (int k = 0; k < yb.nr; ++k)
          for (int l = 0; l < yb.nl; ++l) h->yrho[at + (size_t)yb.ldr * k + l] = B.vals[rb.voff + (size_t)yb.nl * k + l];
        it = yrho_at.emplace(rb.voff, at).first;
      }
      yb.rho = it->second;
      nnz += (double)yb.nl * yb.nr;
      h->yblks.push_back(yb);
    }
    int b1 = (int)h->yblks.size();
    std::sort(h->yblks.begin() + b0, h->yblks.end(), [](const YBlk &u, const YBlk &v) { return u.ycol < v.ycol; });
    for (int i = b0 + 1; i < b1; ++i)
      if (h->yblks[i].ycol < h->yblks[i - 1].ycol + h->yblks[i - 1].nl)
        fail(NSX_E_ARG, "neutron density sub-blocks of one operator overlap in their left partition");
    h->flops_y += 2.0 * ib.da * nnz;
    ymat_b0[y] = b0;
    ymat_b1[y] = b1;
    for (int r0 = 0; r0 < ib.da; r0 += KY_TILE_ROWS)
      h->ygroups.push_back({ib.off, yoff[y], ib.da, r0, b0, b1, B.dim(J2bl), 0});
  }
  // ---- stacked proton side: per output (block, P_l) the contributions (a, P_r) in a fixed
  // order; Abar = their density blocks side by side (nl x K column-major), Zbar = K x d_bl
  // row-major mixed operands written by k_z and consumed by k_a ----
  h->weights.clear();
  h->wterms.clear();
  h->zgroups.clear();
  h->zsrcs.clear();
  h->zunits.clear();
  h->zops.clear();
  h->atiles.clear();
  h->abar.clear();
  h->flops_mix = h->flops_a = 0;
  std::map<std::pair<int, int>, int> slab;  // (block, P_l) -> slab index
  std::vector<std::pair<int, int>> slabs;
  std::vector<int> slabK;
  std::vector<std::vector<std::pair<int, int64_t>>> slab_blocks;  // (nr, rho offset) in K order
  auto get_slab = [&](int bl, int pl) {
    auto it = slab.find({bl, pl});
    if (it != slab.end()) return it->second;
    int id = (int)slabs.size();
    slab[{bl, pl}] = id;
    slabs.push_back({bl, pl});
    slabK.push_back(0);
    slab_blocks.push_back({});
    return id;
  };
  // groups: (block, J_ar, lam) -> table rows
  std::map<std::tuple<int, int, int>, std::vector<int>> groups;
  for (size_t i = 0; i < table.size(); ++i) groups[{table[i].bl, table[i].jar, table[i].lam}].push_back((int)i);
  struct PendingOp { int slab, kofs, wrow; };
  struct Pending { int gid, row0, nr; std::vector<PendingOp> ops; };
  std::vector<Pending> pending;  // one per (group, right proton partition P_r)
  for (auto &gk : groups) {
    const int bl = std::get<0>(gk.first), jar = std::get<1>(gk.first);
    const Block &ob = h->blocks[bl];
    const std::vector<int> &rows = gk.second;
    std::map<std::tuple<int, int, int>, int> sidx;
    std::vector<std::tuple<int, int, int>> srcs;
    for (int r : rows)
      for (const Entry &e : table[r].e)
        for (int L = 0; L < nlayer[e.bk]; ++L)
          if (!sidx.count({e.hb, e.bk, L})) {
            sidx[{e.hb, e.bk, L}] = (int)srcs.size();
            srcs.push_back({e.hb, e.bk, L});
          }
    // sub-groups of at most ZMAXS sources; each has its own stacked rows (the proton density
    // block is repeated in Abar), so no two k_z units write the same Zbar row
    for (size_t s0 = 0; s0 < srcs.size(); s0 += ZMAXS) {
      const size_t s1 = std::min(srcs.size(), s0 + (size_t)ZMAXS);
      ZGroup G;
      G.s_begin = (int)h->zsrcs.size();
      for (size_t si = s0; si < s1; ++si) {
        const int ym = get_ymat(std::get<0>(srcs[si]), std::get<1>(srcs[si]), std::get<2>(srcs[si]));
        const Block &ib = h->blocks[std::get<0>(srcs[si])];
        h->zsrcs.push_back({yoff[ym], ib.off, ib.da, ymat_b0[ym], ymat_b1[ym], 0});
      }
      G.s_end = (int)h->zsrcs.size();
      G.ns = (int)(s1 - s0);
      G.w_off = (int)h->weights.size();
      std::vector<char> active(rows.size(), 0);  // operators with a source in this sub-group
      for (size_t ai = 0; ai < rows.size(); ++ai) {
        std::vector<double> wr(G.ns, 0.0);
        for (const Entry &e : table[rows[ai]].e)
          for (int L = 0; L < nlayer[e.bk]; ++L) {
            int si = sidx[{e.hb, e.bk, L}];
            if (si >= (int)s0 && si < (int)s1) {
              wr[si - s0] += e.w;
              h->wterms.push_back({(int64_t)G.w_off + (int64_t)ai * G.ns + (si - (int)s0), e.op, e.rw});
              active[ai] = 1;
            }
          }
        h->weights.insert(h->weights.end(), wr.begin(), wr.end());
      }
      const int gid = (int)h->zgroups.size();
      h->zgroups.push_back(G);
      // operators per right proton partition
      std::map<int, std::vector<PendingOp>> by_pr;
      for (size_t ai = 0; ai < rows.size(); ++ai) {
        if (!active[ai]) continue;
        const Row &r = table[rows[ai]];
        for (const RhoBlk &rb : A.kblocks[r.ak]) {
          int nl = A.njt_of(rb.pl, ob.J2a), nr = A.njt_of(rb.pr, jar);
          int sl = get_slab(bl, rb.pl);
          PendingOp op{sl, slabK[sl], (int)ai};
          slabK[sl] += nr;
          slab_blocks[sl].push_back({nr, rb.voff});
          by_pr[rb.pr].push_back(op);
          h->flops_a += 2.0 * nl * nr * ob.db;
          h->flops_mix += 2.0 * nr * ob.db * G.ns;
          if (whole) h->block_flops[bl] += 2.0 * nl * nr * ob.db + 2.0 * nr * ob.db * G.ns;
        }
      }
      for (auto &pp : by_pr)
        for (size_t o0 = 0; o0 < pp.second.size(); o0 += ZMAXA) {
          std::vector<PendingOp> part(pp.second.begin() + o0,
                                      pp.second.begin() + std::min(pp.second.size(), o0 + (size_t)ZMAXA));
          pending.push_back({gid, A.poff[A.jidx(jar)][pp.first], A.njt_of(pp.first, jar), part});
        }
    }
  }
  // Zbar slabs and Abar
  auto padz = [](int64_t n) { return (n + KZ_PAD - 1) / KZ_PAD * KZ_PAD; };
  std::vector<int64_t> zoff(slabs.size());
  int64_t ztot = 0;
  for (size_t sl = 0; sl < slabs.size(); ++sl) {
    zoff[sl] = ztot;
    ztot += (int64_t)slabK[sl] * padz(h->blocks[slabs[sl].first].db);
  }
  // FP32 tensor-core layout: per slab, ceil(d_bl / 128) tiles of kgroups * 1024 floats
  std::vector<int64_t> ztc(slabs.size());
  std::vector<int32_t> kgr(slabs.size());
  int64_t ztc_tot = 0;
  for (size_t sl = 0; sl < slabs.size(); ++sl) {
    kgr[sl] = (slabK[sl] + 7) / 8;
    ztc[sl] = ztc_tot;
    const int db = h->blocks[slabs[sl].first].db;
    ztc_tot += (int64_t)((db + 127) / 128) * kgr[sl] * 1024;
  }
  h->z32_elems = ztc_tot;
  h->zops_tc.clear();
  // k_z units: (group, P_r, 128-column tile)
  const int ZT = 128;
  for (auto &pd : pending) {
    const int bl = slabs[pd.ops[0].slab].first;
    const Block &ob = h->blocks[bl];
    int op0 = (int)h->zops.size();
    const int ldz = (int)padz(ob.db);
    for (const PendingOp &o : pd.ops) {
      h->zops.push_back({zoff[o.slab] + (int64_t)o.kofs * ldz, o.wrow, 0});
      h->zops_tc.push_back({ztc[o.slab], o.kofs, kgr[o.slab]});
    }
    int op1 = (int)h->zops.size();
    for (int c0 = 0; c0 < ob.db; c0 += ZT) {
      ZUnit u;
      u.grp = pd.gid;
      u.row0 = pd.row0;
      u.nr = pd.nr;
      u.c0 = c0;
      u.ncols = std::min(ZT, ob.db - c0);
      u.d_bl = ob.db;
      u.op_begin = op0;
      u.op_end = op1;
      u.ldz = ldz;
      u.pad = 0;
      h->zunits.push_back(u);
    }
  }
  // k_z CTAs: runs of consecutive units of one (group, P_r) (its column tiles), at most
  // KZ_UNITS_PER_CTA each, share the CTA's set-up (weights, destinations, sources)
  h->zcta.clear();
  for (size_t i = 0; i < h->zunits.size(); ++i) {
    const ZUnit &u = h->zunits[i];
    const bool start = h->zcta.empty() || (int)i - h->zcta.back() >= KZ_UNITS_PER_CTA || u.grp != h->zunits[i - 1].grp ||
                       u.row0 != h->zunits[i - 1].row0 || u.op_begin != h->zunits[i - 1].op_begin;
    if (start) h->zcta.push_back((int32_t)i);
  }
  h->zcta.push_back((int32_t)h->zunits.size());
  // k_a tiles: (slab, KA_TILE_COLS-column tile)
  const int TW = KA_TILE_COLS;
  for (size_t sl = 0; sl < slabs.size(); ++sl) {
    const int bl = slabs[sl].first, pl = slabs[sl].second;
    const Block &ob = h->blocks[bl];
    const int nl = A.njt_of(pl, ob.J2a), nlp = (int)padz(nl);
    h->abar.resize(padz((int64_t)h->abar.size()), 0.0);
    const int64_t a0 = (int64_t)h->abar.size();
    for (auto &bv : slab_blocks[sl]) {   // bv = (nr, offset of the nl x nr density block)
      const int64_t at = (int64_t)h->abar.size();
      h->abar.resize(at + (int64_t)nlp * bv.first, 0.0);
      for (int k = 0; k < bv.first; ++k)
        for (int l = 0; l < nl; ++l) h->abar[at + (int64_t)nlp * k + l] = A.vals[bv.second + (int64_t)nl * k + l];
    }
    for (int c0 = 0; c0 < ob.db; c0 += TW)
      for (int kb = 0; kb < slabK[sl]; kb += KA_K_SPLIT) {
        ATile t;
        t.out = ob.off + A.poff[A.jidx(ob.J2a)][pl] + (int64_t)c0 * ob.da;
        t.ld = ob.da;
        t.nl = A.njt_of(pl, ob.J2a);
        t.col0 = c0;
        t.ncols = std::min(TW, ob.db - c0);
        t.ldz = (int)padz(ob.db);
        t.k_begin = kb;
        t.k_end = std::min(slabK[sl], kb + KA_K_SPLIT);
        t.nlp = nlp;
        t.zbar = zoff[sl] + c0;
        t.abar = a0;
        h->atiles.push_back(t);
      }
  }
  // longest tiles first
  std::stable_sort(h->atiles.begin(), h->atiles.end(), [](const ATile &x, const ATile &y) {
    return (int64_t)(x.k_end - x.k_begin) * x.nl > (int64_t)(y.k_end - y.k_begin) * y.nl;
  });
  // FP32 tensor-core tiles: Abar^T packed K-major per slab (TF32 big and small parts), one
  // tile per (slab, 128-column tile), grouped by N = nl padded to 16 and longest first
  h->abar_big.clear();
  h->abar_small.clear();
  std::vector<std::vector<ATileTC>> tcls(KTC_NCLASS);
  for (size_t sl = 0; sl < slabs.size(); ++sl) {
    const int bl = slabs[sl].first, pl = slabs[sl].second;
    const Block &ob = h->blocks[bl];
    const int nl = A.njt_of(pl, ob.J2a);
    if (nl > 16 * KTC_NCLASS) continue;   // refused in upload (k_a's limit)
    const int npad = (nl + 15) / 16 * 16;
    const int kg = kgr[sl];
    if (kg == 0) continue;
    const int64_t at = (int64_t)h->abar_big.size();
    h->abar_big.resize(at + (int64_t)kg * 8 * npad, 0.f);
    h->abar_small.resize(at + (int64_t)kg * 8 * npad, 0.f);
    int k = 0;
    for (auto &bv : slab_blocks[sl])   // (nr, offset of the nl x nr density block)
      for (int kk = 0; kk < bv.first; ++kk, ++k)
        for (int l = 0; l < nl; ++l) {
          const float x = (float)A.vals[bv.second + (int64_t)nl * kk + l];
          const float b = umma::tf32_big(x);
          const int64_t e = at + umma::b_kmajor_index(l, k, npad);
          h->abar_big[e] = b;
          h->abar_small[e] = x - b;
        }
    // a slab longer than 1.5 pieces is cut into K pieces of KTC_PIECE_GROUPS groups, one CTA
    // each, so that no single chain of pipeline stages sets the launch's time
    const int npieces = kg > KTC_PIECE_GROUPS * 3 / 2 ? (kg + KTC_PIECE_GROUPS - 1) / KTC_PIECE_GROUPS : 1;
    for (int t = 0; t * 128 < ob.db; ++t)
      for (int pc = 0; pc < npieces; ++pc) {
        const int g0 = pc * KTC_PIECE_GROUPS, g1 = npieces == 1 ? kg : std::min(kg, g0 + KTC_PIECE_GROUPS);
        ATileTC u;
        u.zbar = ztc[sl] + (int64_t)t * kg * 1024 + (int64_t)g0 * 1024;
        u.abar = at + (int64_t)g0 * 8 * npad;
        u.out = ob.off + A.poff[A.jidx(ob.J2a)][pl] + (int64_t)t * 128 * ob.da;
        u.kgroups = g1 - g0;
        u.ld = ob.da;
        u.nl = nl;
        u.ncols = std::min(128, ob.db - t * 128);
        u.split = npieces > 1 ? 1 : 0;
        u.pad = 0;
        tcls[npad / 16 - 1].push_back(u);
      }
  }
  h->atiles_tc.clear();
  for (int c = 0; c < KTC_NCLASS; ++c) {
    std::stable_sort(tcls[c].begin(), tcls[c].end(),
                     [](const ATileTC &x, const ATileTC &y) { return x.kgroups > y.kgroups; });
    h->atc_off[c] = (int64_t)h->atiles_tc.size();
    h->atiles_tc.insert(h->atiles_tc.end(), tcls[c].begin(), tcls[c].end());
  }
  h->atc_off[KTC_NCLASS] = (int64_t)h->atiles_tc.size();
  h->z_elems = ztot;
  h->y_elems = ytot;
  h->max_ynl = h->max_ynr = h->max_anl = h->max_ldy = 0;
  for (auto &g : h->ygroups) h->max_ldy = std::max(h->max_ldy, g.ldy);
  for (auto &y : h->yblks) {
    h->max_ynl = std::max(h->max_ynl, y.nl);
    h->max_ynr = std::max(h->max_ynr, y.nr);
  }
  for (auto &t : h->atiles) h->max_anl = std::max(h->max_anl, t.nl);
  h->max_zns = 0;
  for (auto &g : h->zgroups) h->max_zns = std::max(h->max_zns, g.ns);
}

// Contiguous split of the output blocks into `world` ranges that minimises the largest range's
// flops (exact, by dynamic programming over the prefix sums).  first[r] = first block of rank r,
// first[world] = the block count; ranks past the last block get empty ranges.
std::vector<int> split_blocks(const std::vector<double> &cost, int world) {
  const int n = (int)cost.size();
  std::vector<double> S(n + 1, 0.0);
  for (int i = 0; i < n; ++i) S[i + 1] = S[i] + cost[i];
  const double INF = 1e300;
  // best[k][i]: the smallest largest range when the first i blocks go to k ranks; cut[k][i] the
  // start of the k-th range in that split
  std::vector<std::vector<double>> best(world + 1, std::vector<double>(n + 1, INF));
  std::vector<std::vector<int>> cut(world + 1, std::vector<int>(n + 1, 0));
  best[0][0] = 0.0;
  for (int k = 1; k <= world; ++k)
    for (int i = 0; i <= n; ++i)
      for (int j = 0; j <= i; ++j) {
        if (best[k - 1][j] >= INF) continue;
        const double v = std::max(best[k - 1][j], S[i] - S[j]);
        if (v < best[k][i]) {   // strict: the earliest cut among equal splits
          best[k][i] = v;
          cut[k][i] = j;
        }
      }
  std::vector<int> first(world + 1, n);
  int i = n;
  for (int k = world; k >= 1; --k) {
    first[k] = i;
    i = cut[k][i];
  }
  first[0] = 0;
  return first;
}

}  // namespace nsx
