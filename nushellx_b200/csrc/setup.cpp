// Host-side setup of one J-scheme pn problem (the B200 counterpart of the
// reference's Lnz_TRD + drdbh, src/NuLnz/NuCoreX.f90:807-1367 and 1428-1577):
// species tables, the block list and parity mask, the Racah-weighted pn
// interaction table, and the task lists of the three H.v stages.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
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
  S.hdense.assign(S.hoff[S.nJ], 0.0);
  for (int g = 0; g < s.nseg; ++g) {
    int J2 = s.seg_J2[g];
    if (!S.has_J(J2)) fail(NSX_E_ARG, std::string("species ") + name + ": segment J out of range");
    int j = S.jidx(J2);
    int np = s.seg_np[g] - 1, npr = s.seg_npr[g] - 1;
    if (np < 0 || npr < 0 || np >= S.nspart || npr >= S.nspart || npr < np)
      fail(NSX_E_ARG, std::string("species ") + name + ": bad segment partitions");
    int nl = S.njt_of(np, J2), nr = S.njt_of(npr, J2);
    if ((int64_t)nl * nr != s.seg_off[g + 1] - s.seg_off[g]) fail(NSX_E_ARG, std::string("species ") + name + ": segment size mismatch");
    int64_t d = S.poff[j][S.nspart];
    double *H = S.hdense.data() + S.hoff[j];
    const double *M = s.seg_vals + s.seg_off[g];
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

void build_plan(nsx_handle *h, const nsx_problem *p) {
  h->J2 = p->J2;
  h->parity = p->parity;
  h->renorm = p->renorm;
  load_species(h->A, p->a, "a");
  load_species(h->B, p->b, "b");
  SpeciesPlan &A = h->A, &B = h->B;
  // pn multipole interaction (src/NuLnz/NuCoreX.f90:1133-1142: tiny values zeroed, times renorm)
  for (int i = 0; i < p->nop; ++i) {
    const uint8_t *kb = p->op_keys + 8 * (size_t)i;
    double v = p->op_vals[i];
    if (std::fabs(v) < 1e-10) v = 0.0;
    h->vop[pack_key(kb[0], kb[1], kb[2], kb[3], kb[4])] = v * p->renorm;
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
  // like-particle tiles and flops (segment count, src/NuCommonX/NuCommonX.f90:1009-1104)
  h->ltiles.clear();
  h->flops_like = 0;
  for (auto &b : h->blocks) {
    if (b.da == 0 || b.db == 0) continue;
    for (int r0 = 0; r0 < b.da; r0 += 64)
      for (int c0 = 0; c0 < b.db; c0 += 64)
        h->ltiles.push_back({b.off, A.hoff[A.jidx(b.J2a)], B.hoff[B.jidx(b.J2b)], b.da, b.db, r0, c0});
  }
  for (int g = 0; g < p->a.nseg; ++g) {
    int J2s = p->a.seg_J2[g];
    double nn = (double)(p->a.seg_off[g + 1] - p->a.seg_off[g]) * (p->a.seg_np[g] == p->a.seg_npr[g] ? 1 : 2);
    for (auto &b : h->blocks)
      if (b.J2a == J2s) h->flops_like += 2.0 * nn * b.db;
  }
  for (int g = 0; g < p->b.nseg; ++g) {
    int J2s = p->b.seg_J2[g];
    double nn = (double)(p->b.seg_off[g + 1] - p->b.seg_off[g]) * (p->b.seg_np[g] == p->b.seg_npr[g] ? 1 : 2);
    for (auto &b : h->blocks)
      if (b.J2b == J2s) h->flops_like += 2.0 * nn * b.da;
  }
  // pn table and its algorithmic cost (reuse-aware: each Y_(h,b) once, mixing, proton side)
  std::vector<TabRow> table = pn_table(h);
  h->flops_y = h->flops_mix = h->flops_a = 0;
  h->y_elems = 0;
  std::map<std::pair<int, int>, int> seen;
  for (const TabRow &r : table) {
    const Block &ob = h->blocks[r.bl];
    for (const TabEnt &e : r.e) {
      if (!seen.count({e.hb, e.bk})) {
        seen[{e.hb, e.bk}] = 1;
        double nnz = 0, cols = 0;
        int J2bl = (int)(B.keys[e.bk] & 255), J2br = (int)((B.keys[e.bk] >> 8) & 255);
        for (const RhoBlk &rb : B.kblocks[e.bk]) {
          nnz += (double)B.njt_of(rb.pl, J2bl) * B.njt_of(rb.pr, J2br);
          cols += B.njt_of(rb.pl, J2bl);
        }
        h->flops_y += 2.0 * h->blocks[e.hb].da * nnz;
        h->y_elems += (int64_t)h->blocks[e.hb].da * (int64_t)cols;
      }
    }
    for (const RhoBlk &rb : A.kblocks[r.ak]) {
      double nl = A.njt_of(rb.pl, ob.J2a), nr = A.njt_of(rb.pr, r.jar);
      h->flops_a += 2.0 * nl * nr * ob.db;
      h->flops_mix += 2.0 * nr * ob.db * r.e.size();
    }
  }
  build_pn_plan(h, table, 8, 32, h->pn64);   // FP64: 8 columns per task, 32-row batches
  build_pn_plan(h, table, 16, 64, h->pn32);  // FP32: 16 columns per task, 64-row batches
}

double racah_weight_ext(int Jal, int Jbl, int Jar, int Jbr, int J, int lam) {
  return racah_weight(Jal, Jbl, Jar, Jbr, J, lam);
}

}  // namespace nsx
