// nulnz_gpu: the Lanczos step of NuShellX (NuLnz / NuTRL) on one B200, as a command.
//
// It reads the reference's input files (the proton and neutron .tri/.trd densities, the
// .oph pn interaction, the .spe header with renorm and no_level, and the like-particle
// .sgt/.mat files found by file code), finds the no_level lowest states with the GPU
// solver (FP32 H.v + FP64 thick-restart Lanczos + FP64 Rayleigh-Ritz by default) and
// writes <nucleus><file_code(J2/2, nprot, nneut)>.abz / .trl (what NuVec reads) and
// .lev / .xvc (what NuVec writes) in the reference's formats (src/NuLnz/NuCoreX.f90:526-533,
// src/NuVec/NuVec.f90:120-131, 182, 281).
// Like the reference it stops with a message and a non-zero exit status on failure.
//
// The reference's lanc takes its file names from NuShellX's interactive setup
// (src/NuShellx/NuShellx.f90:1060-1061); here they are explicit options:
//
//   nulnz_gpu --a <base> --b <base> --int <base> --like-a <prefix> --like-b <prefix>
//             --nprot N --nneut N --J2 2J --parity +1|-1|0 --shell-parity p1,p2,...
//             --nshells-p n --nucleus <name> [--xtra c] [--nev n] [--tol t]
//             [--precision fp32|fp64] [--window m] [--max-iter n] [--device d]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>
#include "nsx.h"

static void die(const std::string &msg, int code = 1) {
  std::fprintf(stderr, " nulnz_gpu: %s\n", msg.c_str());
  std::exit(code);
}

int main(int argc, char **argv) {
  std::map<std::string, std::string> o;
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    if (k.rfind("--", 0) != 0 || i + 1 >= argc) die("bad argument " + k + " (options are --name value)");
    o[k.substr(2)] = argv[++i];
  }
  for (const char *req : {"a", "b", "int", "like-a", "like-b", "nprot", "nneut", "J2", "parity", "shell-parity",
                          "nshells-p", "nucleus"})
    if (!o.count(req)) die(std::string("missing --") + req);
  std::vector<int32_t> sp;
  {
    std::stringstream ss(o["shell-parity"]);
    std::string t;
    while (std::getline(ss, t, ',')) sp.push_back(std::atoi(t.c_str()));
  }
  const int nprot = std::atoi(o["nprot"].c_str()), nneut = std::atoi(o["nneut"].c_str());
  nsx_files f;
  std::memset(&f, 0, sizeof(f));
  f.a = o["a"].c_str();
  f.b = o["b"].c_str();
  f.inter = o["int"].c_str();
  f.like_a = o["like-a"].c_str();
  f.like_b = o["like-b"].c_str();
  f.T2_a = nprot;
  f.nmp_a = -nprot;
  f.T2_b = nneut;
  f.nmp_b = nneut;
  f.xtra = o.count("xtra") ? o["xtra"][0] : 'x';
  f.J2 = std::atoi(o["J2"].c_str());
  f.parity = std::atoi(o["parity"].c_str());
  f.nshells = (int32_t)sp.size();
  f.nshells_p = std::atoi(o["nshells-p"].c_str());
  f.shell_parity = sp.data();
  // no_level: third line of <int>.spe (src/NuLnz/NuCoreX.f90:1664-1670), unless --nev
  int nev = 0;
  if (o.count("nev")) {
    nev = std::atoi(o["nev"].c_str());
  } else {
    std::ifstream spe(o["int"] + ".spe");
    std::string l1, l2, l3;
    if (!spe || !std::getline(spe, l1) || !std::getline(spe, l2) || !std::getline(spe, l3))
      die("cannot open " + o["int"] + ".spe or read no_level from its third line");
    nev = std::atoi(l3.c_str());
  }
  if (nev <= 0 || nev > 64) die("no_level out of range (1 .. 64)");
  const int device = o.count("device") ? std::atoi(o["device"].c_str()) : 0;

  nsx_handle *h = nullptr;
  if (nsx_load_files(&f, device, &h) != NSX_OK) die(nsx_last_error());
  const int64_t n = nsx_dim(h);
  if (nev > n) nev = (int)n;
  nsx_params p;
  std::memset(&p, 0, sizeof(p));
  p.nev = nev;
  p.tol = o.count("tol") ? std::atof(o["tol"].c_str()) : 1e-4;
  p.precision = (o.count("precision") && o["precision"] == "fp64") ? NSX_FP64 : NSX_FP32;
  p.window = o.count("window") ? std::atoi(o["window"].c_str()) : 100;
  p.keep = 0;
  p.max_iter = o.count("max-iter") ? std::atoi(o["max-iter"].c_str()) : 3000;
  p.pre_iter = 2;
  p.seed = 5;
  p.start = nullptr;
  p.refine = p.precision == NSX_FP32 ? 1 : 0;
  std::vector<double> ev(nev), vecs((size_t)nev * n);
  nsx_report rep;
  int rc = nsx_solve(h, &p, ev.data(), vecs.data(), &rep);
  if (rc != NSX_OK) die(nsx_last_error());
  char code[4];
  if (nsx_file_code(f.J2 / 2, nprot, nneut, code) != NSX_OK) die(nsx_last_error());
  const std::string prefix = o["nucleus"] + code;
  const int T2 = std::abs(nprot - nneut);
  rc = nsx_write_results(h, prefix.c_str(), ev.data(), vecs.data(), nev, rep.iterations, o["int"].c_str(), T2);
  if (rc != NSX_OK) die(nsx_last_error());
  std::printf(" dimension %lld, %d Lanczos steps, %d H.v, %.3f s (H.v %.3f s)\n", (long long)n, rep.iterations,
              rep.matvecs, rep.seconds, rep.matvec_seconds);
  for (int i = 0; i < nev; ++i) std::printf("%10.3f%s", ev[i], (i % 5 == 4 || i == nev - 1) ? "\n" : "");
  std::printf(" wrote %s.abz .trl .lev .xvc\n", prefix.c_str());
  nsx_destroy(h);
  return 0;
}
