// Reader of the reference's input file set for the Lanczos hot path
// (src/NuLnz/NuCoreX.f90:838-873, 1133-1206, 1216-1319, 1659-1670): Intel
// Fortran unformatted sequential records with 4-byte length markers.  Any
// missing file, short record or inconsistent size is reported as NSX_E_IO /
// NSX_E_ARG, never as a crash.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include "nsx_internal.h"

namespace nsx {

namespace {
struct Records {
  std::string path;
  std::vector<char> data;
  size_t pos = 0;
  explicit Records(const std::string &p) : path(p) {
    std::ifstream f(p, std::ios::binary);
    if (!f) fail(NSX_E_IO, "cannot open " + p);
    data.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  // next record payload
  std::pair<const char *, size_t> next() {
    if (pos + 4 > data.size()) fail(NSX_E_IO, path + ": unexpected end of file");
    int32_t n1;
    std::memcpy(&n1, data.data() + pos, 4);
    if (n1 < 0 || pos + 8 + (size_t)n1 > data.size()) fail(NSX_E_IO, path + ": truncated record");
    int32_t n2;
    std::memcpy(&n2, data.data() + pos + 4 + n1, 4);
    if (n1 != n2) fail(NSX_E_IO, path + ": record length markers differ");
    const char *p = data.data() + pos + 4;
    pos += 8 + (size_t)n1;
    return {p, (size_t)n1};
  }
};
template <typename T>
T get(const char *p, size_t i) {
  T v;
  std::memcpy(&v, p + i * sizeof(T), sizeof(T));
  return v;
}
const char AN_CODE[] =
    "0123456789_$cdefghijklmnopqrstuvwxyz@ABCDEFGHIJKLMNMPQRSTUVWXYZ\xa3"
    "a%^&=b-+#";
constexpr int MAX_CODE = 72;

struct SpeciesStore {
  std::vector<int32_t> njt, par;
  std::vector<int16_t> occ;   // [nspart][nshell] the species' own shells
  std::vector<uint8_t> keys;
  std::vector<int64_t> val_off;
  std::vector<double> vals;
  std::vector<uint32_t> masks;
  std::vector<int32_t> seg_J2, seg_np, seg_npr;
  std::vector<int64_t> seg_off;
  std::vector<double> seg_vals;
};

void read_species(const nsx_files *f, const char *base, const char *like, int T2, int nmp, SpeciesStore &st,
                  nsx_species &s) {
  std::string b(base);
  // .tri
  Records tri(b + ".tri");
  auto r1 = tri.next();
  if (r1.second < 36) fail(NSX_E_IO, b + ".tri: short header record");
  int nspart = get<int32_t>(r1.first, 0), minJ2 = get<int32_t>(r1.first, 1), maxJ2 = get<int32_t>(r1.first, 2);
  int32_t is_proton = get<int32_t>(r1.first, 3);
  if (nspart <= 0 || maxJ2 < minJ2) fail(NSX_E_IO, b + ".tri: bad header");
  int nJ = (maxJ2 - minJ2) / 2 + 1;
  auto r2 = tri.next();
  if (r2.second != sizeof(int32_t) * (size_t)nspart * nJ) fail(NSX_E_IO, b + ".tri: nJT record size");
  st.njt.resize((size_t)nspart * nJ);
  std::memcpy(st.njt.data(), r2.first, r2.second);
  auto r3 = tri.next();
  if (r3.second != 64 * (size_t)nspart) fail(NSX_E_IO, b + ".tri: partition record size");
  st.par.resize(nspart);
  for (int p = 0; p < nspart; ++p) {
    int par = 1;
    for (int i = 0; i < f->nshells && i < 32; ++i) {
      int16_t occ = get<int16_t>(r3.first + 64 * (size_t)p, i);
      if (occ > 0 && f->shell_parity[i] < 0 && (occ % 2)) par = -par;
    }
    st.par[p] = par;
  }
  s.nspart = nspart;
  s.minJ2 = minJ2;
  s.maxJ2 = maxJ2;
  s.njt = st.njt.data();
  s.parity = st.par.data();
  s.shell_first = is_proton ? 1 : f->nshells_p + 1;
  s.nshell = is_proton ? f->nshells_p : f->nshells - f->nshells_p;
  if (s.shell_first - 1 + s.nshell > 32) fail(NSX_E_IO, b + ".tri: more than 32 shells");
  st.occ.resize((size_t)nspart * s.nshell);
  for (int p = 0; p < nspart; ++p)
    for (int o = 0; o < s.nshell; ++o)
      st.occ[(size_t)p * s.nshell + o] = get<int16_t>(r3.first + 64 * (size_t)p, s.shell_first - 1 + o);
  s.occ = st.occ.data();
  // .trd
  Records trd(b + ".trd");
  auto d1 = trd.next();
  if (d1.second < 24) fail(NSX_E_IO, b + ".trd: short header record");
  int trdd = get<int32_t>(d1.first, 0);
  int words = get<int32_t>(d1.first, 3), nspartr = get<int32_t>(d1.first, 4);
  if (trdd < 0 || nspartr != nspart || words != (nspart - 1) / 32 + 1) fail(NSX_E_IO, b + ".trd: header inconsistent with .tri");
  s.nkeys = trdd;
  s.words = words;
  st.keys.assign((size_t)trdd * 8, 0);
  st.val_off.assign(trdd + 1, 0);
  st.masks.assign((size_t)trdd * nspart * words, 0u);
  if (trdd > 0) {
    auto kr = trd.next();
    if (kr.second != 8 * (size_t)trdd) fail(NSX_E_IO, b + ".trd: key record size");
    std::memcpy(st.keys.data(), kr.first, kr.second);
    auto dr = trd.next();
    if (dr.second != 4 * (size_t)trdd) fail(NSX_E_IO, b + ".trd: dims record size");
    std::vector<int32_t> dims(trdd);
    std::memcpy(dims.data(), dr.first, dr.second);
    for (int k = 0; k < trdd; ++k) st.val_off[k + 1] = st.val_off[k] + dims[k];
    st.vals.resize(st.val_off[trdd]);
    for (int k = 0; k < trdd; ++k) {
      if (dims[k] == 0) continue;
      auto vr = trd.next();
      if (vr.second != 4 * (size_t)dims[k]) fail(NSX_E_IO, b + ".trd: value record size");
      for (int i = 0; i < dims[k]; ++i) {
        double v = (double)get<float>(vr.first, i);
        if (std::abs(v) < 1e-11) v = 0.0;  // NuCoreX.f90:1156-1158
        st.vals[st.val_off[k] + i] = v;
      }
      auto mr = trd.next();
      if (mr.second != 4 * (size_t)words * nspart) fail(NSX_E_IO, b + ".trd: mask record size");
      std::memcpy(st.masks.data() + (size_t)k * nspart * words, mr.first, mr.second);
    }
  }
  s.keys = st.keys.data();
  s.val_off = st.val_off.data();
  s.vals = st.vals.data();
  s.masks = st.masks.data();
  // .sgt / .mat per J
  st.seg_off.assign(1, 0);
  for (int J2 = minJ2; J2 <= maxJ2; J2 += 2) {
    char code[4];
    nsx_file_code(J2 / 2, T2 / 2, nmp / 2 + MAX_CODE / 2, code);
    std::string name = std::string(like) + code + std::string(1, f->xtra);
    Records sgt(name + ".sgt");
    sgt.next();
    auto g = sgt.next();
    if (g.second < 8) fail(NSX_E_IO, name + ".sgt: short record");
    int nseg = get<int32_t>(g.first, 0);
    Records mat(name + ".mat");
    mat.next();
    for (int k = 0; k < nseg; ++k) {
      auto m = mat.next();
      if (m.second < 16) fail(NSX_E_IO, name + ".mat: short segment record");
      int dimpt = get<int32_t>(m.first, 0), dimptr = get<int32_t>(m.first, 1);
      int np = get<int32_t>(m.first, 2), npr = get<int32_t>(m.first, 3);
      if (dimpt < 0 || dimptr < 0 || m.second < 16 + 4 * (size_t)dimpt * dimptr)
        fail(NSX_E_IO, name + ".mat: segment size");
      st.seg_J2.push_back(J2);
      st.seg_np.push_back(np);
      st.seg_npr.push_back(npr);
      for (int64_t i = 0; i < (int64_t)dimpt * dimptr; ++i) st.seg_vals.push_back((double)get<float>(m.first + 16, i));
      st.seg_off.push_back((int64_t)st.seg_vals.size());
    }
  }
  s.nseg = (int32_t)st.seg_J2.size();
  s.seg_J2 = st.seg_J2.data();
  s.seg_np = st.seg_np.data();
  s.seg_npr = st.seg_npr.data();
  s.seg_off = st.seg_off.data();
  s.seg_vals = st.seg_vals.data();
}
}  // namespace

struct FileStore {
  SpeciesStore a, b;
  std::vector<uint8_t> op_keys;
  std::vector<double> op_vals;
};

std::shared_ptr<void> load_files(const nsx_files *f, nsx_problem *p) {
  if (!f->a || !f->b || !f->inter || !f->like_a || !f->like_b || !f->shell_parity || f->nshells <= 0)
    fail(NSX_E_ARG, "incomplete nsx_files");
  auto owner = std::make_shared<FileStore>();
  FileStore *fs = owner.get();
  p->J2 = f->J2;
  p->parity = f->parity;
  read_species(f, f->a, f->like_a, f->T2_a, f->nmp_a, fs->a, p->a);
  read_species(f, f->b, f->like_b, f->T2_b, f->nmp_b, fs->b, p->b);
  Records oph(std::string(f->inter) + ".oph");
  auto h = oph.next();
  if (h.second < 8) fail(NSX_E_IO, "oph: short header");
  int nop = get<int32_t>(h.first, 0);
  for (int i = 0; i < nop; ++i) {
    auto r = oph.next();
    if (r.second < 16) fail(NSX_E_IO, "oph: short record");
    for (int k = 0; k < 8; ++k) fs->op_keys.push_back((uint8_t)r.first[k]);
    fs->op_vals.push_back(get<double>(r.first + 8, 0));
  }
  p->nop = nop;
  p->op_keys = fs->op_keys.data();
  p->op_vals = fs->op_vals.data();
  std::ifstream spe(std::string(f->inter) + ".spe");
  if (!spe) fail(NSX_E_IO, std::string("cannot open ") + f->inter + ".spe");
  std::string line;
  std::getline(spe, line);
  double renorm = 1.0;
  if (!(spe >> renorm)) fail(NSX_E_IO, "spe: cannot read renorm (line 2)");
  p->renorm = renorm;
  return owner;
}

}  // namespace nsx

extern "C" int nsx_file_code(int32_t i, int32_t j, int32_t k, char out[4]) {
  using nsx::MAX_CODE;
  if (i < 0) i += MAX_CODE;
  if (j < 0) j += MAX_CODE;
  if (k < 0) k += MAX_CODE;
  if (i < 0 || j < 0 || k < 0 || i > MAX_CODE || j > MAX_CODE || k > MAX_CODE) return NSX_E_ARG;
  out[0] = nsx::AN_CODE[i];
  out[1] = nsx::AN_CODE[j];
  out[2] = nsx::AN_CODE[k];
  out[3] = 0;
  return NSX_OK;
}
