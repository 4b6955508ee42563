// The solver's results in the reference's output files, as NuTRL leaves them for NuVec.
//
//   <prefix>.abz  unformatted sequential (4-byte record markers), thick-restart form
//                 (written at src/NuLnz/NuCoreX.f90:526-533, read by NuVec at
//                 src/NuVec/NuVec.f90:126-130 and by a TRL restart at NuCoreX.f90:270-275):
//       record 1: isave (i4), alpha(1:isave), betat(1:isave), matrix(1:isave,1:isave) (r4)
//       record 2: imax, no_level (i4), tt (r4), no_state, basd, count, no_keep, no_conv,
//                 first_iter, second_iter, noiter (i4)
//       record 3: bas(1:basd), 8 bytes each: char(2Ja) char(2Jb) and six zero bytes
//                 (NuCoreX.f90:937-947)
//       record 4: alpha_copy(1:noiter), betat(isave+1) (r4), indx(1:noiter) (i4)
//   <prefix>.trl  direct access, one record of no_state r4 values per basis vector
//                 (recl = no_state * 4 bytes, NuCoreX.f90:280-281)
//   <prefix>.lev  formatted: the header NuVec's output_results writes after its program
//                 banner (NuVec.f90:298-321) and the levels as 5(f10.3,a1), each with its
//                 parity character (NuVec.f90:239-241, 285-286)
//   <prefix>.xvc  unformatted sequential, as NuVec writes its eigenvectors (NuVec.f90:182,
//                 281): record 1: no_state, number of levels (i4); then one record per
//                 level: energy (r4), vector(1:no_state) (r4)
//   <prefix>.xva  unformatted sequential, NuVec's averages (NuVec.f90:210-283): one record
//                 per level: energy (r4), ava(1:no_shells), avb(1:no_shells) (r4: the
//                 proton and neutron occupation of every shell, weighted by |c|^2), and
//                 spartpc(no_sparta, no_spartb, min_cJ2a/2:max_cJ2a/2, min_cJ2b/2:max_cJ2b/2)
//                 (r4, column-major: the percentage of |c|^2 in each partition pair and 2J pair)
//   <prefix>.lp   formatted: the .lev header, the partitions' shell occupations, and per
//                 level the average occupations, the parity split and the partition pairs
//                 holding at least 1 % (NuVec.f90:199-290)
//                 (.xva and .lp need the partitions' shell occupations, nsx_species.occ)
//
// The basis written is the converged Ritz vectors themselves (isave = nev), with
// matrix = diag(E), alpha = E, betat = 0 and count = 2: NuVec's reconstruction
// psi_i = sum_j matrix-eigenvector(j, i) * record(j) then returns exactly these
// eigenpairs, and the files have the reference's layout.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "nsx_internal.h"

namespace nsx {

namespace {
constexpr int NOITER = 300;        // the reference's noiter (src/NuCommonX/NuCommonX.f90:25)
constexpr int FIRST_ITER_T = 80;   // first_iterT of the TRL form (NuCoreX.f90:251, 333)

struct RecordWriter {
  FILE *f = nullptr;
  std::vector<unsigned char> buf;
  explicit RecordWriter(const std::string &path) : f(std::fopen(path.c_str(), "wb")) {
    if (!f) fail(NSX_E_IO, "cannot write " + path);
  }
  ~RecordWriter() {
    if (f) std::fclose(f);
  }
  template <typename V>
  void put(const V &v) {
    const unsigned char *p = reinterpret_cast<const unsigned char *>(&v);
    buf.insert(buf.end(), p, p + sizeof(V));
  }
  void put_bytes(const void *p, size_t n) {
    const unsigned char *q = static_cast<const unsigned char *>(p);
    buf.insert(buf.end(), q, q + n);
  }
  void end_record() {
    if (buf.size() > 0x7fffffffu) fail(NSX_E_ARG, "record longer than a 4-byte Fortran record marker can state");
    const uint32_t n = (uint32_t)buf.size();
    if (std::fwrite(&n, 4, 1, f) != 1 || (n && std::fwrite(buf.data(), 1, n, f) != n) || std::fwrite(&n, 4, 1, f) != 1)
      fail(NSX_E_IO, "write failed");
    buf.clear();
  }
};

// Share of the squared amplitude of v in positive-parity partition pairs.
double positive_parity_share(const nsx_handle *h, const double *v) {
  double pos = 0.0, tot = 0.0;
  for (const Block &b : h->blocks) {
    int64_t n = b.off;
    for (int pb = 0; pb < h->B.nspart; ++pb)
      for (int kb = 0; kb < h->B.njt_of(pb, b.J2b); ++kb)
        for (int pa = 0; pa < h->A.nspart; ++pa) {
          const int na = h->A.njt_of(pa, b.J2a);
          const bool plus = h->A.par[pa] * h->B.par[pb] >= 0;
          for (int ka = 0; ka < na; ++ka, ++n) {
            const double a = v[n] * v[n];
            tot += a;
            if (plus) pos += a;
          }
        }
  }
  return tot > 0 ? pos / tot : 0.0;
}
}  // namespace

// NuVec's per-level averages: .xva records and the .lp listing (NuVec.f90:199-290).  For each
// level the squared amplitudes are summed per (proton partition, neutron partition, 2J_a, 2J_b);
// the shell averages follow from the partition sums and the partitions' shell occupations.
static void write_xva_lp(const nsx_handle *h, const std::string &base, const double *evals, const double *evecs,
                         int nev, const char *intfile, int T2) {
  const SpeciesPlan &A = h->A, &B = h->B;
  if (A.occ.empty() || B.occ.empty()) return;   // occupations not given: no averages
  const int64_t n = h->no_state;
  const int nsa = A.nspart, nsb = B.nspart, nJa = A.nJ, nJb = B.nJ;
  const int nshells = std::max(A.shell_first - 1 + A.nshell, B.shell_first - 1 + B.nshell);
  const size_t ncell = (size_t)nsa * nsb * nJa * nJb;
  RecordWriter xva(base + ".xva");
  FILE *lp = std::fopen((base + ".lp").c_str(), "w");
  if (!lp) fail(NSX_E_IO, "cannot write " + base + ".lp");
  std::fprintf(lp, "  %s\n\n", intfile ? intfile : "");
  std::fprintf(lp, "  2*J,   2*T %11d %11d\n\n", h->J2, T2);
  std::fprintf(lp, "  Lowest Energy Levels\n\n");
  std::fprintf(lp, "\n  Type a = protons   Type b = neutrons\n  A partitions\n");
  auto partition_line = [&](int p, const SpeciesPlan &S) {
    std::fprintf(lp, "%8d", -(p + 1));
    for (int s = 0; s < nshells; ++s) {
      const int o = s - (S.shell_first - 1);
      std::fprintf(lp, "%4d", (o >= 0 && o < S.nshell) ? S.occ[(size_t)p * S.nshell + o] : 0);
    }
    std::fprintf(lp, "\n");
  };
  for (int p = 0; p < nsa; ++p) partition_line(p, A);
  std::fprintf(lp, "  B partitions\n");
  for (int p = 0; p < nsb; ++p) partition_line(p, B);
  std::vector<char> chpar(nev, '?');
  std::vector<double> cell(ncell), wa(nsa), wb(nsb);
  for (int i = 0; i < nev; ++i) {
    const double *v = evecs + (size_t)i * n;
    std::fill(cell.begin(), cell.end(), 0.0);
    std::fill(wa.begin(), wa.end(), 0.0);
    std::fill(wb.begin(), wb.end(), 0.0);
    double tot = 0.0, pos = 0.0, neg = 0.0;
    for (const Block &b : h->blocks) {
      const int ja = A.jidx(b.J2a), jb = B.jidx(b.J2b);
      int64_t k = b.off;
      for (int pb = 0; pb < nsb; ++pb)
        for (int kb = 0; kb < B.njt_of(pb, b.J2b); ++kb)
          for (int pa = 0; pa < nsa; ++pa) {
            double s = 0.0;
            for (int ka = 0; ka < A.njt_of(pa, b.J2a); ++ka, ++k) s += v[k] * v[k];
            cell[(((size_t)jb * nJa + ja) * nsb + pb) * nsa + pa] += s;
            wa[pa] += s;
            wb[pb] += s;
            tot += s;
            if (A.par[pa] * B.par[pb] >= 0) pos += s;
            else neg += s;
          }
    }
    std::vector<float> ava(nshells, 0.f), avb(nshells, 0.f);
    for (int p = 0; p < nsa; ++p)
      for (int o = 0; o < A.nshell; ++o) ava[A.shell_first - 1 + o] += (float)(A.occ[(size_t)p * A.nshell + o] * wa[p]);
    for (int p = 0; p < nsb; ++p)
      for (int o = 0; o < B.nshell; ++o) avb[B.shell_first - 1 + o] += (float)(B.occ[(size_t)p * B.nshell + o] * wb[p]);
    const double t = tot > 0 ? tot : 1.0;
    if (pos / t > 0.95) chpar[i] = '+';
    if (neg / t > 0.95) chpar[i] = '-';
    // .xva: E, ava, avb (sums of occupation x |c|^2), spartpc in percent
    xva.put<float>((float)evals[i]);
    for (float x : ava) xva.put<float>(x);
    for (float x : avb) xva.put<float>(x);
    for (size_t c = 0; c < ncell; ++c) xva.put<float>((float)(cell[c] * 100.0 / t));
    xva.end_record();
    // .lp
    std::fprintf(lp, "\n State %11d %14.6f %c\n\n Average A type nucleons\n", i + 1, evals[i], chpar[i]);
    for (int s = 0; s < nshells; ++s) std::fprintf(lp, "%7.2f%s", ava[s] / t, (s % 11 == 10 || s == nshells - 1) ? "\n" : "");
    std::fprintf(lp, "\n Average B type nucleons\n");
    for (int s = 0; s < nshells; ++s) std::fprintf(lp, "%7.2f%s", avb[s] / t, (s % 11 == 10 || s == nshells - 1) ? "\n" : "");
    std::fprintf(lp, "  Positive and Negative Parity\n  +ve %8.2f%% -ve %8.2f%%\n", pos * 100.0 / t, neg * 100.0 / t);
    for (int jb = 0; jb < nJb; ++jb)
      for (int ja = 0; ja < nJa; ++ja) {
        double amp = 0.0;
        for (int pb = 0; pb < nsb; ++pb)
          for (int pa = 0; pa < nsa; ++pa) amp += cell[(((size_t)jb * nJa + ja) * nsb + pb) * nsa + pa];
        amp *= 100.0 / t;
        if (amp < 1.0) continue;
        std::fprintf(lp, "\n  2*JA, 2*JB, amplitude %11d %11d %14.6f\n", A.minJ2 + 2 * ja, B.minJ2 + 2 * jb, amp);
        for (int pb = 0; pb < nsb; ++pb) {
          double ab = 0.0;
          for (int pa = 0; pa < nsa; ++pa) ab += cell[(((size_t)jb * nJa + ja) * nsb + pb) * nsa + pa];
          ab *= 100.0 / t;
          if (ab < 1.0) continue;
          std::fprintf(lp, "  B partition, amplitude %11d %14.6f\n  A partitions, amplitudes\n", pb + 1, ab);
          for (int pa = 0; pa < nsa; ++pa)
            std::fprintf(lp, "(%3d,%7.2f)%s", pa + 1, cell[(((size_t)jb * nJa + ja) * nsb + pb) * nsa + pa] * 100.0 / t,
                         (pa % 6 == 5 || pa == nsa - 1) ? "\n" : "");
        }
      }
  }
  std::fprintf(lp, "\n");
  for (int i = 0; i < nev; ++i) std::fprintf(lp, "%10.3f%c%s", evals[i], chpar[i], (i % 5 == 4 || i == nev - 1) ? "\n" : "");
  std::fclose(lp);
}

// NuVec's .xvc eigenvector file and the .lev level list for these eigenpairs.
static void write_lev_xvc(const nsx_handle *h, const std::string &base, const double *evals, const double *evecs,
                          int nev, const char *intfile, int T2) {
  const int64_t n = h->no_state;
  // .xvc
  {
    RecordWriter w(base + ".xvc");
    w.put<int32_t>((int32_t)n);
    w.put<int32_t>(nev);
    w.end_record();
    for (int i = 0; i < nev; ++i) {
      w.put<float>((float)evals[i]);
      const double *v = evecs + (size_t)i * n;
      for (int64_t k = 0; k < n; ++k) w.put<float>((float)v[k]);
      w.end_record();
    }
  }
  // .lev
  {
    FILE *f = std::fopen((base + ".lev").c_str(), "w");
    if (!f) fail(NSX_E_IO, "cannot write " + base + ".lev");
    std::fprintf(f, "  %s\n\n", intfile ? intfile : "");
    std::fprintf(f, "  2*J,   2*T %11d %11d\n\n", h->J2, T2);
    std::fprintf(f, "  Lowest Energy Levels\n\n");
    for (int i = 0; i < nev; ++i) {
      const double share = positive_parity_share(h, evecs + (size_t)i * n);
      const char par = share > 0.95 ? '+' : (share < 0.05 ? '-' : '?');
      std::fprintf(f, "%10.3f%c", evals[i], par);
      if (i % 5 == 4 || i == nev - 1) std::fprintf(f, "\n");
    }
    std::fclose(f);
  }
  write_xva_lp(h, base, evals, evecs, nev, intfile, T2);
}

void write_results(const nsx_handle *h, const char *prefix, const double *evals, const double *evecs, int nev,
                   int iterations, const char *intfile, int T2) {
  if (!prefix || !evals || !evecs) fail(NSX_E_ARG, "null argument");
  if (nev <= 0 || nev > NOITER) fail(NSX_E_ARG, "nev out of range (1 .. 300)");
  const std::string base(prefix);
  const int64_t n = h->no_state;
  // .abz
  {
    RecordWriter w(base + ".abz");
    w.put<int32_t>(nev);
    for (int i = 0; i < nev; ++i) w.put<float>((float)evals[i]);
    for (int i = 0; i < nev; ++i) w.put<float>(0.f);
    for (int j = 0; j < nev; ++j)
      for (int i = 0; i < nev; ++i) w.put<float>(i == j ? (float)evals[i] : 0.f);
    w.end_record();
    const int32_t rec2[] = {iterations, nev};
    w.put_bytes(rec2, sizeof(rec2));
    w.put<float>(0.f);  // tt: multiplication time, not tracked
    const int32_t rec2b[] = {(int32_t)n, (int32_t)h->blocks.size(), 2, nev, nev, FIRST_ITER_T, FIRST_ITER_T / 2, NOITER};
    w.put_bytes(rec2b, sizeof(rec2b));
    w.end_record();
    for (const Block &b : h->blocks) {
      unsigned char bas[8] = {(unsigned char)b.J2a, (unsigned char)b.J2b, 0, 0, 0, 0, 0, 0};
      w.put_bytes(bas, 8);
    }
    w.end_record();
    for (int i = 0; i < NOITER; ++i) w.put<float>(i < nev ? (float)evals[i] : 0.f);
    w.put<float>(0.f);
    for (int i = 0; i < NOITER; ++i) w.put<int32_t>(i < nev ? i + 1 : 0);
    w.end_record();
  }
  // .trl
  {
    FILE *f = std::fopen((base + ".trl").c_str(), "wb");
    if (!f) fail(NSX_E_IO, "cannot write " + base + ".trl");
    std::vector<float> rec((size_t)n);
    for (int i = 0; i < nev; ++i) {
      const double *v = evecs + (size_t)i * n;
      for (int64_t k = 0; k < n; ++k) rec[k] = (float)v[k];
      if (std::fwrite(rec.data(), 4, (size_t)n, f) != (size_t)n) {
        std::fclose(f);
        fail(NSX_E_IO, "write failed: " + base + ".trl");
      }
    }
    std::fclose(f);
  }
  write_lev_xvc(h, base, evals, evecs, nev, intfile, T2);
}


// The solver's thick-restart state as the reference's TRL leaves it (NuCoreX.f90:526-533 and the
// .trl records): .abz with isave = m, alpha = diag T, betat = the subdiagonal, matrix = T, the
// counters, and betat(isave+1) = beta; .trl with the m basis vectors and the next vector.  NuVec's
// reconstruction (eigenvectors of the matrix times the records) gives the Ritz vectors; a resume
// (read_state) continues from them.  .lev / .xvc carry the given eigenpairs (evecs may be null:
// no .xvc then).
void write_state(const nsx_handle *h, const char *prefix, const nsx_state *st, const double *evals,
                 const double *evecs, int nev, const char *intfile, int T2) {
  if (!prefix || !st || !evals || !st->V || !st->T || !st->next) fail(NSX_E_ARG, "null argument");
  const int m = st->m;
  if (m <= 0 || m + 1 > NOITER) fail(NSX_E_ARG, "state size out of range (1 .. 299)");
  if (nev <= 0 || nev > m) fail(NSX_E_ARG, "nev out of range (1 .. state size)");
  const std::string base(prefix);
  const int64_t n = h->no_state;
  {
    RecordWriter w(base + ".abz");
    w.put<int32_t>(m);
    for (int i = 0; i < m; ++i) w.put<float>((float)st->T[i + (size_t)m * i]);
    for (int i = 0; i < m; ++i) w.put<float>(i ? (float)st->T[i + (size_t)m * (i - 1)] : 0.f);
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) w.put<float>((float)st->T[i + (size_t)m * j]);
    w.end_record();
    const int32_t rec2[] = {st->iterations, nev};
    w.put_bytes(rec2, sizeof(rec2));
    w.put<float>(0.f);
    const int32_t rec2b[] = {(int32_t)n, (int32_t)h->blocks.size(), 2, m, nev, FIRST_ITER_T, FIRST_ITER_T / 2, NOITER};
    w.put_bytes(rec2b, sizeof(rec2b));
    w.end_record();
    for (const Block &b : h->blocks) {
      unsigned char bas[8] = {(unsigned char)b.J2a, (unsigned char)b.J2b, 0, 0, 0, 0, 0, 0};
      w.put_bytes(bas, 8);
    }
    w.end_record();
    for (int i = 0; i < NOITER; ++i) w.put<float>(i < nev ? (float)evals[i] : 0.f);
    w.put<float>((float)st->beta);
    for (int i = 0; i < NOITER; ++i) w.put<int32_t>(i < nev ? i + 1 : 0);
    w.end_record();
  }
  {
    FILE *f = std::fopen((base + ".trl").c_str(), "wb");
    if (!f) fail(NSX_E_IO, "cannot write " + base + ".trl");
    std::vector<float> rec((size_t)n);
    for (int i = 0; i <= m; ++i) {
      const double *v = i < m ? st->V + (size_t)i * n : st->next;
      for (int64_t k = 0; k < n; ++k) rec[k] = (float)v[k];
      if (std::fwrite(rec.data(), 4, (size_t)n, f) != (size_t)n) {
        std::fclose(f);
        fail(NSX_E_IO, "write failed: " + base + ".trl");
      }
    }
    std::fclose(f);
  }
  if (evecs) write_lev_xvc(h, base, evals, evecs, nev, intfile, T2);
}

// The state written by write_state, for a resume (NuCoreX.f90:268-292 reads the same records).
// st->m is the room of st->V / st->T in vectors on entry and the vectors read on return.
void read_state(const nsx_handle *h, const char *prefix, nsx_state *st) {
  if (!prefix || !st || !st->V || !st->T || !st->next) fail(NSX_E_ARG, "null argument");
  const std::string base(prefix);
  const int64_t n = h->no_state;
  std::vector<std::vector<char>> recs;
  {
    FILE *f = std::fopen((base + ".abz").c_str(), "rb");
    if (!f) fail(NSX_E_IO, "cannot open " + base + ".abz");
    for (;;) {
      uint32_t n1 = 0, n2 = 0;
      if (std::fread(&n1, 4, 1, f) != 1) break;
      std::vector<char> r(n1);
      if ((n1 && std::fread(r.data(), 1, n1, f) != n1) || std::fread(&n2, 4, 1, f) != 1 || n1 != n2) {
        std::fclose(f);
        fail(NSX_E_IO, base + ".abz: truncated or inconsistent record");
      }
      recs.push_back(std::move(r));
    }
    std::fclose(f);
  }
  if (recs.size() < 4 || recs[0].size() < 4) fail(NSX_E_IO, base + ".abz: fewer than 4 records");
  int32_t m;
  std::memcpy(&m, recs[0].data(), 4);
  if (m <= 0 || m + 1 > NOITER || recs[0].size() != 4 + 4 * (size_t)(2 * m + m * m))
    fail(NSX_E_IO, base + ".abz: bad basis size in record 1");
  if (m > st->m) fail(NSX_E_ARG, base + ": the state holds " + std::to_string(m) + " vectors, room for " +
                                     std::to_string(st->m));
  if (recs[1].size() < 12 || recs[3].size() < 4 * (size_t)(2 * NOITER + 1)) fail(NSX_E_IO, base + ".abz: short records");
  int32_t imax, ns;
  std::memcpy(&imax, recs[1].data(), 4);
  std::memcpy(&ns, recs[1].data() + 12, 4);
  if (ns != n) fail(NSX_E_ARG, base + ".abz: vector length differs from the handle's");
  const char *mat = recs[0].data() + 4 + 8 * (size_t)m;
  for (size_t e = 0; e < (size_t)m * m; ++e) {
    float x;
    std::memcpy(&x, mat + 4 * e, 4);
    st->T[e] = x;
  }
  float b;
  std::memcpy(&b, recs[3].data() + 4 * NOITER, 4);
  FILE *f = std::fopen((base + ".trl").c_str(), "rb");
  if (!f) fail(NSX_E_IO, "cannot open " + base + ".trl");
  std::vector<float> rec((size_t)n);
  for (int i = 0; i <= m; ++i) {
    if (std::fread(rec.data(), 4, (size_t)n, f) != (size_t)n) {
      std::fclose(f);
      fail(NSX_E_IO, base + ".trl: fewer records than the .abz states");
    }
    double *v = i < m ? st->V + (size_t)i * n : st->next;
    for (int64_t k = 0; k < n; ++k) v[k] = rec[k];
  }
  std::fclose(f);
  st->m = m;
  st->beta = b;
  st->iterations = imax;
  st->restarts = 0;
}

}  // namespace nsx
