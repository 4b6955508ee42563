// Plan of the fused pn kernel (k_pn): the Racah-weighted pn table of the
// reference's drdbh (src/NuLnz/NuCoreX.f90:1428-1577), regrouped for a GPU
// that owns output columns.
//
// Output block (Ja_l, Jb_l) is cut into tasks = CH consecutive neutron states
// (output columns, possibly spanning several partitions Q_l).  Everything a task needs is local to it:
//   Y_(h,b)[:, chunk] = C_h[:, Q_r(b) cols] rho_b[chunk, Q_r]^T    (Y columns are output columns)
//   Z_a[P_r rows]     = sum_(h,b) w_(a,(h,b)) Y_(h,b)[P_r rows]    (mixing)
//   out[P_l rows]    += rho_a[P_l, P_r] Z_a[P_r rows]
// The table rows of one output block with the same (J_ar, lam) form a group:
// its sources (h, b) and proton operators a share one dense weight matrix.
#include <algorithm>
#include <cmath>
#include <map>
#include <tuple>
#include "nsx_internal.h"

namespace nsx {

double racah_weight_ext(int Jal, int Jbl, int Jar, int Jbr, int J, int lam);

std::vector<TabRow> pn_table(const nsx_handle *h) {
  const SpeciesPlan &A = h->A, &B = h->B;
  const int J2 = h->J2;
  std::map<std::pair<int, int>, int> bidx;
  for (size_t i = 0; i < h->blocks.size(); ++i) bidx[{h->blocks[i].J2a, h->blocks[i].J2b}] = (int)i;
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
  std::vector<TabRow> rows;
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
        TabRow row{(int)bl, jar, ak, lam, {}};
        int jbrn = std::max(std::abs(ob.J2b - lam), std::abs(jar - J2));
        int jbrx = std::min(std::min(ob.J2b + lam, jar + J2), B.maxJ2);
        for (int jbr = jbrn; jbr <= jbrx; jbr += 2) {
          if (!B.has_J(jbr)) continue;
          auto hit = bidx.find({jar, jbr});
          if (hit == bidx.end()) continue;
          const Block &ib = h->blocks[hit->second];
          if (ib.da == 0 || ib.db == 0) continue;
          double rw = racah_weight_ext(ob.J2a, ob.J2b, jar, jbr, J2, lam);
          if (rw == 0.0) continue;
          auto bit = bkeys.find({ob.J2b, jbr, lam});
          if (bit == bkeys.end()) continue;
          for (int bk : bit->second) {
            if (B.kblocks[bk].empty()) continue;
            uint64_t bkey = B.keys[bk];
            int sbl = (bkey >> 16) & 255, sbr = (bkey >> 24) & 255;
            auto vit = h->vop.find(pack_key(sal, sar, sbl, sbr, lam));
            if (vit == h->vop.end() || vit->second == 0.0) continue;
            row.e.push_back({bk, hit->second, vit->second * rw});
          }
        }
        if (!row.e.empty()) rows.push_back(std::move(row));
      }
    }
  }
  return rows;
}

void build_pn_plan(const nsx_handle *h, const std::vector<TabRow> &table, int CH, int batch_rows, PnPlan &P) {
  const SpeciesPlan &A = h->A, &B = h->B;
  P = PnPlan();
  P.CH = CH;
  P.batch_rows = batch_rows;
  P.item_rows = 32 / CH;
  const int IR = P.item_rows;
  // per b-key: left partition -> (right partition, value offset)
  std::vector<std::vector<std::pair<int, int64_t>>> bl_lookup(B.keys.size());
  for (size_t k = 0; k < B.keys.size(); ++k) {
    bl_lookup[k].assign(B.nspart, {-1, 0});
    for (const RhoBlk &rb : B.kblocks[k]) bl_lookup[k][rb.pl] = {rb.pr, rb.voff};
  }
  // groups per output block: (J_ar, lam) -> table rows
  std::map<int, std::map<std::pair<int, int>, std::vector<int>>> by_block;
  for (size_t i = 0; i < table.size(); ++i) by_block[table[i].bl][{table[i].jar, table[i].lam}].push_back((int)i);
  for (auto &bk : by_block) {
    const int bl = bk.first;
    const Block &ob = h->blocks[bl];
    std::vector<int> gids;             // group indices of this block
    std::vector<std::vector<std::pair<int, int>>> gsrc;
    for (auto &gk : bk.second) {
      const int jar = gk.first.first;
      const std::vector<int> &rows = gk.second;
      // sources of the group
      std::map<std::pair<int, int>, int> sidx;
      std::vector<std::pair<int, int>> srcs;
      for (int r : rows)
        for (const TabEnt &e : table[r].e)
          if (!sidx.count({e.hb, e.bk})) {
            sidx[{e.hb, e.bk}] = (int)srcs.size();
            srcs.push_back({e.hb, e.bk});
          }
      // split into sub-groups of at most 32 sources (each keeps all proton operators)
      for (size_t s0 = 0; s0 < srcs.size(); s0 += 32) {
        size_t s1 = std::min(srcs.size(), s0 + 32);
        Group G;
        G.d_ar = A.dim(jar);
        G.nsrc = (int)(s1 - s0);
        G.na = (int)rows.size();
        G.w_off = (int)P.weights.size();
        // weights [na][nsrc]
        for (size_t ai = 0; ai < rows.size(); ++ai) {
          std::vector<double> wr(G.nsrc, 0.0);
          for (const TabEnt &e : table[rows[ai]].e) {
            int s = sidx[{e.hb, e.bk}];
            if (s >= (int)s0 && s < (int)s1) wr[s - s0] += e.w;
          }
          P.weights.insert(P.weights.end(), wr.begin(), wr.end());
        }
        // right proton partitions: operators acting on each, rows in chunks of item_rows
        G.pr_begin = (int)P.prwork.size();
        for (int pr = 0; pr < A.nspart; ++pr) {
          int nr = A.njt_of(pr, jar);
          if (nr == 0) continue;
          std::vector<std::pair<int, const RhoBlk *>> ops;  // (a index in group, block)
          for (size_t ai = 0; ai < rows.size(); ++ai)
            for (const RhoBlk &rb : A.kblocks[table[rows[ai]].ak])
              if (rb.pr == pr) ops.push_back({(int)ai, &rb});
          if (ops.empty()) continue;
          for (int r0 = 0; r0 < nr; r0 += IR) {
            for (size_t o0 = 0; o0 < ops.size(); o0 += MAXA) {
              PrWork w;
              w.row0 = A.poff[A.jidx(jar)][pr] + r0;
              w.nr = std::min(IR, nr - r0);
              w.a_begin = (int)P.aops.size();
              for (size_t o = o0; o < std::min(ops.size(), o0 + MAXA); ++o) {
                const RhoBlk *rb = ops[o].second;
                int nl = A.njt_of(rb->pl, ob.J2a);
                AOp a;
                a.rho = rb->voff + (int64_t)nl * r0;
                a.ld = nl;
                a.out_row0 = A.poff[A.jidx(ob.J2a)][rb->pl];
                a.nl = nl;
                a.wrow = ops[o].first;
                P.aops.push_back(a);
                P.max_nl = std::max(P.max_nl, nl);
              }
              w.a_end = (int)P.aops.size();
              P.prwork.push_back(w);
            }
          }
        }
        G.pr_end = (int)P.prwork.size();
        // row batches: maximal runs of items whose rows fit batch_rows (items are in row order)
        G.bt_begin = (int)P.batches.size();
        for (int it = G.pr_begin; it < G.pr_end;) {
          Batch b;
          b.it_begin = it;
          b.row0 = P.prwork[it].row0;
          int end_row = b.row0;
          while (it < G.pr_end && P.prwork[it].row0 + P.prwork[it].nr - b.row0 <= batch_rows &&
                 P.prwork[it].row0 >= b.row0) {
            end_row = std::max(end_row, P.prwork[it].row0 + P.prwork[it].nr);
            ++it;
          }
          b.it_end = it;
          b.nrows = end_row - b.row0;
          P.batches.push_back(b);
        }
        G.bt_end = (int)P.batches.size();
        gids.push_back((int)P.groups.size());
        gsrc.push_back(std::vector<std::pair<int, int>>(srcs.begin() + s0, srcs.begin() + s1));
        P.groups.push_back(G);
        P.max_dar = std::max(P.max_dar, G.d_ar);
        P.max_nsrc = std::max(P.max_nsrc, G.nsrc);
      }
    }
    // tasks: CH consecutive neutron states (columns) of the output block
    const int jbl = B.jidx(ob.J2b);
    for (int c0 = 0; c0 < ob.db; c0 += CH) {
      PnTask t;
      t.out = ob.off + (int64_t)c0 * ob.da;
      t.d_al = ob.da;
      t.nq = std::min(CH, ob.db - c0);
      t.g_begin = (int)P.tgroups.size();
      double cost = 0;
      for (size_t gi = 0; gi < gids.size(); ++gi) {
        const Group &G = P.groups[gids[gi]];
        TGroup tg;
        tg.grp = gids[gi];
        tg.src_begin = (int)P.tsrcs.size();
        for (int s = 0; s < (int)gsrc[gi].size(); ++s) {
          int hb = gsrc[gi][s].first, bkey = gsrc[gi][s].second;
          int J2br = h->blocks[hb].J2b;
          TSrc ts;
          ts.piece_begin = (int)P.pieces.size();
          ts.cover = 0u;
          ts.sidx = s;
          // left partitions overlapping [c0, c0 + nq)
          for (int ql = 0; ql < B.nspart; ++ql) {
            int q0 = B.poff[jbl][ql], q1 = B.poff[jbl][ql + 1];
            int a0 = std::max(q0, c0), a1 = std::min(q1, c0 + t.nq);
            if (a0 >= a1) continue;
            auto lk = bl_lookup[bkey][ql];
            if (lk.first < 0) continue;
            Piece pc;
            pc.c = h->blocks[hb].off + (int64_t)B.poff[B.jidx(J2br)][lk.first] * G.d_ar;
            pc.rho = lk.second + (a0 - q0);
            pc.ld = q1 - q0;
            pc.nr = B.njt_of(lk.first, J2br);
            pc.cs = a0 - c0;
            pc.w = a1 - a0;
            for (int c = pc.cs; c < pc.cs + pc.w; ++c) ts.cover |= (1u << c);
            P.pieces.push_back(pc);
            cost += (double)G.d_ar * pc.w * pc.nr;
          }
          ts.piece_end = (int)P.pieces.size();
          if (ts.piece_end == ts.piece_begin) continue;
          P.tsrcs.push_back(ts);
        }
        tg.src_end = (int)P.tsrcs.size();
        if (tg.src_end == tg.src_begin) continue;
        cost += (double)(G.pr_end - G.pr_begin) * IR * CH * (tg.src_end - tg.src_begin);
        P.tgroups.push_back(tg);
      }
      t.g_end = (int)P.tgroups.size();
      if (t.g_end == t.g_begin) continue;
      P.tasks.push_back(t);
      P.task_cost.push_back(cost);
      P.max_dal = std::max(P.max_dal, ob.da);
    }
  }
  // longest tasks first (greedy balance over the persistent CTAs)
  std::vector<int> order(P.tasks.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return P.task_cost[a] > P.task_cost[b]; });
  std::vector<PnTask> sorted;
  for (int i : order) sorted.push_back(P.tasks[i]);
  P.tasks.swap(sorted);
}

}  // namespace nsx
