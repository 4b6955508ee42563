// <psi_i|H|psi_j> between given vectors: the B200 counterpart of NuXpct's matrixs
// (src/NuXpct/NuCoreXE.f90:1417-1471), which reads the eigenvectors of a .xvc file, applies
// multiplyx/multiplya/multiplyb to each and forms matrixc(i, j) = (H psi_i) . psi_j, written
// as text (.ovl, 8f10.4 per column) and as unformatted records (.ovx: no_levels, then each
// column).  Here the vectors go to the GPU once, H psi_i is the library's H.v, and the
// overlaps are one deterministic reduction per vector.  For eigenvectors the matrix is
// diagonal with the eigenvalues on it: the reference's own check of a solve.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "nsx_internal.h"

namespace nsx {

namespace {
constexpr int XP_CTAS = 592;     // 148 SMs x 4
constexpr int XP_MAXV = 64;

// partial[cta][j] = sum over the CTA's rows of V[j][r] * w[r], j < cnt
__global__ void __launch_bounds__(256) k_xp_dot(const double *__restrict__ V, int64_t n, int cnt,
                                                const double *__restrict__ w, double *__restrict__ partial) {
  __shared__ double acc[8][XP_MAXV];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < 8 * XP_MAXV; e += 256) (&acc[0][0])[e] = 0.0;
  __syncthreads();
  for (int64_t r0 = (int64_t)blockIdx.x * 256; r0 < n; r0 += (int64_t)gridDim.x * 256) {
    const int64_t r = r0 + tid;
    const double wr = r < n ? w[r] : 0.0;
    for (int j = 0; j < cnt; ++j) {
      double v = r < n ? V[(int64_t)j * n + r] * wr : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) acc[warp][j] += v;
    }
  }
  __syncthreads();
  for (int j = tid; j < cnt; j += 256) {
    double v = 0.0;
    for (int q = 0; q < 8; ++q) v += acc[q][j];
    partial[(int64_t)blockIdx.x * XP_MAXV + j] = v;
  }
}
__global__ void k_xp_reduce(const double *__restrict__ partial, int nparts, int cnt, double *__restrict__ out) {
  const int j = threadIdx.x;
  if (j >= cnt) return;
  double v = 0.0;
  for (int p = 0; p < nparts; ++p) v += partial[(int64_t)p * XP_MAXV + j];
  out[j] = v;
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

// out[i + nvec * j] = (H v_i) . v_j for host vectors v (nvec x no_state, row i = vector i).
void expectation_matrix(nsx_handle *h, const double *vecs, int nvec, int precision, double *out) {
  if (nvec <= 0 || nvec > XP_MAXV) fail(NSX_E_ARG, "vector count must be in 1..64");
  if (precision != NSX_FP64 && precision != NSX_FP32) fail(NSX_E_ARG, "unknown precision");
  const int64_t n = h->no_state;
  cudaStream_t s = solve_stream(h);
  DevBuf V, HV, part, res;
  NSX_CUDA(cudaMalloc(&V.p, sizeof(double) * n * nvec));
  NSX_CUDA(cudaMalloc(&HV.p, sizeof(double) * n * nvec));
  NSX_CUDA(cudaMalloc(&part.p, sizeof(double) * XP_CTAS * XP_MAXV));
  NSX_CUDA(cudaMalloc(&res.p, sizeof(double) * nvec * nvec));
  double *dV = static_cast<double *>(V.p), *dHV = static_cast<double *>(HV.p);
  NSX_CUDA(cudaMemcpyAsync(dV, vecs, sizeof(double) * n * nvec, cudaMemcpyHostToDevice, s));
  for (int i = 0; i < nvec; ++i) matvec_device(h, dV + (int64_t)i * n, dHV + (int64_t)i * n, precision, s);
  for (int i = 0; i < nvec; ++i) {
    k_xp_dot<<<XP_CTAS, 256, 0, s>>>(dV, n, nvec, dHV + (int64_t)i * n, static_cast<double *>(part.p));
    k_xp_reduce<<<1, XP_MAXV, 0, s>>>(static_cast<const double *>(part.p), XP_CTAS, nvec,
                                      static_cast<double *>(res.p) + (int64_t)i * nvec);
    h->launches += 2;
  }
  NSX_CUDA(cudaGetLastError());
  std::vector<double> r((size_t)nvec * nvec);
  NSX_CUDA(cudaMemcpyAsync(r.data(), res.p, sizeof(double) * nvec * nvec, cudaMemcpyDeviceToHost, s));
  NSX_CUDA(cudaStreamSynchronize(s));
  // r[i * nvec + j] = v_j . (H v_i) = matrixc(i, j); out is column-major matrixc
  for (int i = 0; i < nvec; ++i)
    for (int j = 0; j < nvec; ++j) out[i + (size_t)nvec * j] = r[(size_t)i * nvec + j];
}

namespace {
struct RecordReader {
  std::vector<char> data;
  size_t pos = 0;
  std::string path;
  explicit RecordReader(const std::string &p) : path(p) {
    FILE *f = std::fopen(p.c_str(), "rb");
    if (!f) fail(NSX_E_IO, "cannot open " + p);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    data.resize(sz > 0 ? (size_t)sz : 0);
    if (sz > 0 && std::fread(data.data(), 1, (size_t)sz, f) != (size_t)sz) {
      std::fclose(f);
      fail(NSX_E_IO, "cannot read " + p);
    }
    std::fclose(f);
  }
  std::pair<const char *, size_t> next() {
    if (pos + 4 > data.size()) fail(NSX_E_IO, path + ": unexpected end of file");
    uint32_t n1, n2;
    std::memcpy(&n1, data.data() + pos, 4);
    if (pos + 8 + (size_t)n1 > data.size()) fail(NSX_E_IO, path + ": truncated record");
    std::memcpy(&n2, data.data() + pos + 4 + n1, 4);
    if (n1 != n2) fail(NSX_E_IO, path + ": record length markers differ");
    const char *p = data.data() + pos + 4;
    pos += 8 + (size_t)n1;
    return {p, (size_t)n1};
  }
};
void put_record(FILE *f, const void *p, uint32_t n) {
  if (std::fwrite(&n, 4, 1, f) != 1 || (n && std::fwrite(p, 1, n, f) != n) || std::fwrite(&n, 4, 1, f) != 1)
    fail(NSX_E_IO, "write failed");
}
}  // namespace

// NuXpct's matrixs on files: the eigenvectors of <xvc_path> in, <out_prefix>.ovl / .ovx out.
void xpct_files(nsx_handle *h, const char *xvc_path, const char *out_prefix, int precision) {
  if (!xvc_path || !out_prefix) fail(NSX_E_ARG, "null path");
  RecordReader rd(xvc_path);
  auto hd = rd.next();
  if (hd.second < 8) fail(NSX_E_IO, std::string(xvc_path) + ": short header");
  int32_t no_st, nlev;
  std::memcpy(&no_st, hd.first, 4);
  std::memcpy(&nlev, hd.first + 4, 4);
  if (no_st != h->no_state) fail(NSX_E_ARG, std::string(xvc_path) + ": vector length differs from the handle's");
  if (nlev <= 0 || nlev > XP_MAXV) fail(NSX_E_IO, std::string(xvc_path) + ": level count out of range (1..64)");
  std::vector<double> v((size_t)nlev * no_st);
  for (int i = 0; i < nlev; ++i) {
    auto r = rd.next();
    if (r.second != 4 + 4 * (size_t)no_st) fail(NSX_E_IO, std::string(xvc_path) + ": level record of wrong length");
    for (int64_t k = 0; k < no_st; ++k) {
      float x;
      std::memcpy(&x, r.first + 4 + 4 * k, 4);
      v[(size_t)i * no_st + k] = x;
    }
  }
  std::vector<double> m((size_t)nlev * nlev);
  expectation_matrix(h, v.data(), nlev, precision, m.data());
  const std::string base(out_prefix);
  FILE *f = std::fopen((base + ".ovl").c_str(), "w");
  if (!f) fail(NSX_E_IO, "cannot write " + base + ".ovl");
  std::fprintf(f, " Expectation Values and Off Diagonal Matrix Elements\n\n");
  std::fprintf(f, " Initial levels from 1 ... No_Levels left to right\n");
  std::fprintf(f, " Final   levels from 1 ... No_Levels top  to bottom\n\n");
  for (int j = 0; j < nlev; ++j) {
    for (int i = 0; i < nlev; ++i) {
      std::fprintf(f, "%10.4f", m[i + (size_t)nlev * j]);
      if (i % 8 == 7 || i == nlev - 1) std::fprintf(f, "\n");
    }
    std::fprintf(f, "\n");
  }
  std::fclose(f);
  FILE *g = std::fopen((base + ".ovx").c_str(), "wb");
  if (!g) fail(NSX_E_IO, "cannot write " + base + ".ovx");
  put_record(g, &nlev, 4);
  for (int j = 0; j < nlev; ++j) {
    std::vector<float> col(nlev);
    for (int i = 0; i < nlev; ++i) col[i] = (float)m[i + (size_t)nlev * j];
    put_record(g, col.data(), 4 * (uint32_t)nlev);
  }
  std::fclose(g);
}

}  // namespace nsx
