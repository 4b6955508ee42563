// The compressed pn interaction of NuTRLZ (src/NuTRLZ/NuCoreXZ.f90:1613-1887, "prd"; the .dop
// file of src/NuDiop/NuDiop.f90): the multipole interaction of each (lam, parity) is given as
// its eigen-decomposition V = sum_e e u_e u_e^T (possibly truncated), and the one-body
// densities are folded into combined operators
//
//     proton  (e, lam, parity):  sum_a e * u_e(a) * rho_a      (renorm enters through V = 1)
//     neutron (e, lam, parity):  sum_b u_e(b) * rho_b
//
// whose pn table pairs equal e with the Racah weight alone.  Here that is a rewrite of the
// problem before planning: the combined operators become the species' densities (keys
// (2Jl, 2Jr, e, 200 + (parity+3)/2, 2lam), as prd names them, sub-blocks = the union of the
// folded densities' sub-blocks) and the pn interaction becomes V = 1 between the proton and
// neutron operator of the same key bytes.  The H.v kernels and the plan are the same.
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <tuple>
#include "nsx_internal.h"

namespace nsx {

namespace {

struct CombinedSpecies {
  std::vector<uint8_t> keys;
  std::vector<int64_t> val_off{0};
  std::vector<double> vals;
  std::vector<uint32_t> masks;
};

struct ZStore {
  CombinedSpecies a, b;
  std::vector<uint8_t> op_keys;
  std::vector<double> op_vals;
};

struct DopTerm {
  int sal, sar, sbl, sbr;
  double u;
};
struct DopVec {
  double e = 0;
  std::vector<DopTerm> terms;
};

int njt_of(const nsx_species &s, int ip, int J2) {
  if (J2 < s.minJ2 || J2 > s.maxJ2 || (J2 - s.minJ2) % 2) return 0;
  return s.njt[(size_t)((J2 - s.minJ2) / 2) * s.nspart + ip];
}

// Density key bytes -> its index; sub-blocks of key k as (l, r, value offset) in .trd order.
struct DensityIndex {
  const nsx_species &s;
  std::map<std::tuple<int, int, int, int, int>, int> key;
  explicit DensityIndex(const nsx_species &sp) : s(sp) {
    for (int k = 0; k < s.nkeys; ++k) {
      const uint8_t *b = s.keys + 8 * (size_t)k;
      key[{b[0], b[1], b[2], b[3], b[4]}] = k;
    }
  }
  std::vector<std::tuple<int, int, int64_t>> blocks(int k) const {
    std::vector<std::tuple<int, int, int64_t>> out;
    const uint8_t *kb = s.keys + 8 * (size_t)k;
    int64_t v = s.val_off[k];
    for (int r = 0; r < s.nspart; ++r) {
      const uint32_t *m = s.masks + ((size_t)k * s.nspart + r) * s.words;
      for (int l = 0; l < s.nspart; ++l) {
        if (!((m[l / 32] >> (l % 32)) & 1u)) continue;
        out.emplace_back(l, r, v);
        v += (int64_t)njt_of(s, l, kb[0]) * njt_of(s, r, kb[1]);
      }
    }
    if (v != s.val_off[k + 1]) fail(NSX_E_ARG, "density key size disagrees with its masks");
    return out;
  }
};

// Folds the densities of one species into the combined operators.  proton: coefficient e*u.
void combine(const nsx_species &s, const std::map<std::tuple<int, int, int>, DopVec> &ops, bool proton,
             CombinedSpecies &out) {
  DensityIndex di(s);
  std::vector<int> J2s;
  for (int J2 = s.minJ2; J2 <= s.maxJ2; J2 += 2) J2s.push_back(J2);
  for (const auto &op : ops) {
    const int lam = std::get<0>(op.first), par = std::get<1>(op.first), eig = std::get<2>(op.first);
    const DopVec &dv = op.second;
    for (int jl : J2s)
      for (int jr : J2s) {
        std::map<std::pair<int, int>, std::vector<double>> acc;   // (r, l) -> nl x nr block
        for (const DopTerm &t : dv.terms) {
          const int sl = proton ? t.sal : t.sbl, sr = proton ? t.sar : t.sbr;
          auto it = di.key.find({jl, jr, sl, sr, lam});
          if (it == di.key.end()) continue;
          const double c = proton ? dv.e * t.u : t.u;
          for (const auto &bl : di.blocks(it->second)) {
            const int l = std::get<0>(bl), r = std::get<1>(bl);
            const int nl = njt_of(s, l, jl), nr = njt_of(s, r, jr);
            auto &blk = acc[{r, l}];
            if (blk.empty()) blk.assign((size_t)nl * nr, 0.0);
            const double *src = s.vals + std::get<2>(bl);
            for (int64_t e = 0; e < (int64_t)nl * nr; ++e) blk[e] += c * src[e];
          }
        }
        if (acc.empty()) continue;
        const uint8_t kb[8] = {(uint8_t)jl, (uint8_t)jr, (uint8_t)eig, (uint8_t)(200 + (par + 3) / 2), (uint8_t)lam,
                               0, 0, 0};
        out.keys.insert(out.keys.end(), kb, kb + 8);
        const size_t m0 = out.masks.size();
        out.masks.resize(m0 + (size_t)s.nspart * s.words, 0u);
        for (auto &kv : acc) {   // .trd order: right partition, then left partition
          const int r = kv.first.first, l = kv.first.second;
          out.masks[m0 + (size_t)r * s.words + l / 32] |= 1u << (l % 32);
          out.vals.insert(out.vals.end(), kv.second.begin(), kv.second.end());
        }
        out.val_off.push_back((int64_t)out.vals.size());
      }
  }
}

}  // namespace

// The problem rewritten with the combined operators of `dop`; the arrays live in the returned holder.
std::shared_ptr<void> compress_problem(const nsx_problem *p, const nsx_dop *d, nsx_problem *out) {
  if (!p || !d) fail(NSX_E_ARG, "null argument");
  if (d->nterms < 0 || (d->nterms > 0 && (!d->lam2 || !d->parity || !d->eig || !d->e || !d->shells || !d->u)))
    fail(NSX_E_ARG, "bad compressed interaction arrays");
  std::map<std::tuple<int, int, int>, DopVec> ops;   // (2lam, parity, eigenvector number)
  for (int32_t i = 0; i < d->nterms; ++i) {
    if (d->eig[i] < 1 || d->eig[i] > 199 || (d->parity[i] != 1 && d->parity[i] != -1) || d->lam2[i] < 0 ||
        d->lam2[i] > 255)
      fail(NSX_E_ARG, "compressed interaction term " + std::to_string(i) + ": bad lam, parity or number");
    if (!std::isfinite(d->e[i]) || !std::isfinite(d->u[i]))
      fail(NSX_E_ARG, "compressed interaction term " + std::to_string(i) + " is not finite");
    DopVec &v = ops[{d->lam2[i], d->parity[i], d->eig[i]}];
    v.e = d->e[i];
    const uint8_t *sh = d->shells + 4 * (size_t)i;
    v.terms.push_back({sh[0], sh[1], sh[2], sh[3], d->u[i]});
  }
  auto st = std::make_shared<ZStore>();
  combine(p->a, ops, true, st->a);
  combine(p->b, ops, false, st->b);
  for (const auto &op : ops) {
    const int lam = std::get<0>(op.first), par = std::get<1>(op.first), eig = std::get<2>(op.first);
    const uint8_t kb[8] = {(uint8_t)eig, (uint8_t)(200 + (par + 3) / 2), (uint8_t)eig,
                           (uint8_t)(200 + (par + 3) / 2), (uint8_t)lam, 0, 0, 0};
    st->op_keys.insert(st->op_keys.end(), kb, kb + 8);
    st->op_vals.push_back(1.0);
  }
  *out = *p;
  auto fill = [](nsx_species &s, const CombinedSpecies &c) {
    s.nkeys = (int32_t)(c.keys.size() / 8);
    s.keys = c.keys.data();
    s.val_off = c.val_off.data();
    s.vals = c.vals.data();
    s.masks = c.masks.data();
  };
  fill(out->a, st->a);
  fill(out->b, st->b);
  out->nop = (int32_t)st->op_vals.size();
  out->op_keys = st->op_keys.data();
  out->op_vals = st->op_vals.data();
  return st;
}

// Reads a .dop file (list-directed text as NuDiop writes it) into term arrays.
std::shared_ptr<DopArrays> read_dop(const std::string &path) {
  std::ifstream f(path);
  if (!f) fail(NSX_E_IO, "cannot open " + path);
  auto a = std::make_shared<DopArrays>();
  auto need = [&](bool ok) {
    if (!ok) fail(NSX_E_IO, path + ": malformed or short");
  };
  int max_lmo = 0;
  need(bool(f >> max_lmo));
  if (max_lmo < 0 || max_lmo > 255) fail(NSX_E_IO, path + ": bad maximum multipole");
  for (int blk = 0; blk < 2 * (max_lmo / 2 + 1); ++blk) {
    int lam = 0, pt = 0, nel = 0;
    need(bool(f >> lam >> pt >> nel));
    if (nel < 0 || nel > 199) fail(NSX_E_IO, path + ": bad eigenvalue count");
    for (int i = 1; i <= nel; ++i) {
      double e = 0;
      int nle = 0;
      need(bool(f >> e >> nle));
      if (nle < 0) fail(NSX_E_IO, path + ": bad component count");
      for (int j = 0; j < nle; ++j) {
        int s1, s3, s2, s4;
        double u;
        need(bool(f >> s1 >> s3 >> s2 >> s4 >> u));
        if (s1 < 1 || s1 > 255 || s3 < 1 || s3 > 255 || s2 < 1 || s2 > 255 || s4 < 1 || s4 > 255)
          fail(NSX_E_IO, path + ": shell number out of range");
        a->lam2.push_back(lam);
        a->parity.push_back(pt);
        a->eig.push_back(i);
        a->e.push_back(e);
        a->u.push_back(u);
        const uint8_t sh[4] = {(uint8_t)s1, (uint8_t)s3, (uint8_t)s2, (uint8_t)s4};
        a->shells.insert(a->shells.end(), sh, sh + 4);
      }
    }
  }
  return a;
}

}  // namespace nsx
