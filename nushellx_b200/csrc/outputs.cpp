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
}

}  // namespace nsx
