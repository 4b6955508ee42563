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
// Two forms.  NuShellX's own command line for the Lanczos step (src/NuShellx/NuShellx.f90:
// 1060-1061), so that the command drops into its .bat sequence:
//
//   nulnz_gpu NucleusJ Nucleus'a' Nucleus'b' Nucleus+xtra intfile [--options]
//
// reads NucleusJ.nus for the model space (the reader of src/NuCommon/NuCommon.f90:2546-2736:
// nucleus name, valence protons and neutrons, parity, shells with their parities, the 2J of
// the run), the proton and neutron .tri/.trd and .sgt/.mat under Nucleus'a' / Nucleus'b', and
// the .oph/.spe under Nucleus+xtra (xtra = its last character); and the explicit form
//
//   nulnz_gpu --a <base> --b <base> --int <base> --like-a <prefix> --like-b <prefix>
//             --nprot N --nneut N --J2 2J --parity +1|-1|0 --shell-parity p1,p2,...
//             --nshells-p n --nucleus <name> [--xtra c]
//
// Options of both: [--nev n] [--tol t] [--precision fp32|fp64] [--window m] [--max-iter n]
// [--device d].
#include <cstdio>
#include <cstdlib>
#include <algorithm>
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

// The values of the .nus model-space file this command needs, read in the order of the
// reference's reader (comment lines start with '!').
struct Nus {
  std::string nucleus;
  int nprot = 0, nneut = 0, parity = 0, nshells = 0, nshells_p = 0, J2 = 0;
  std::vector<int32_t> shell_parity;
};
static Nus read_nus(const std::string &path) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::vector<std::string> lines;
  for (std::string l; std::getline(f, l);) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    if (l.rfind("!QSpin", 0) == 0) die(path + ": the isospin (QSpin) formalism is not supported");
    if (!l.empty() && l[0] == '!') continue;
    lines.push_back(l);
  }
  size_t li = 0;
  auto line = [&]() -> std::string {
    if (li >= lines.size()) die("end of file reading " + path);
    return lines[li++];
  };
  Nus n;
  {
    std::string nm = line();
    const size_t a = nm.find_first_not_of(' ');
    n.nucleus = a == std::string::npos ? "" : nm.substr(a, nm.find_last_not_of(' ') - a + 1);
  }
  for (int i = 0; i < 3; ++i) line();   // description
  {
    std::istringstream ss(line());
    if (!(ss >> n.nprot >> n.nneut)) die(path + ": bad nucleon numbers");
  }
  {
    std::istringstream ss(line());
    if (!(ss >> n.parity)) die(path + ": bad parity");
  }
  {
    std::istringstream ss(line());
    if (!(ss >> n.nshells) || n.nshells <= 0 || n.nshells > 64) die(path + ": bad shell count");
  }
  const std::string nucleons = line();
  for (int s = 0; s < n.nshells; ++s) {
    std::istringstream ss(line());
    int cn, sn, sl, sj2, st2, sp;
    if (!(ss >> cn >> sn >> sl >> sj2 >> st2 >> sp) || (sp != 1 && sp != -1)) die(path + ": bad shell line");
    n.shell_parity.push_back(sp);
    if (s < (int)nucleons.size() && nucleons[s] == 'p') ++n.nshells_p;
  }
  {
    std::istringstream ss(line());
    int jmax = 0;
    if (!(ss >> n.J2 >> jmax)) die(path + ": bad 2J range");
  }
  if (n.nshells_p == 0) n.nshells_p = n.nshells / 2;
  return n;
}

int main(int argc, char **argv) {
  std::map<std::string, std::string> o;
  int first = 1;
  if (argc >= 5 && std::strncmp(argv[1], "--", 2) != 0) {   // NuShellX's positional form
    const Nus nus = read_nus(std::string(argv[1]) + ".nus");
    o["a"] = o["like-a"] = argv[2];
    o["b"] = o["like-b"] = argv[3];
    o["int"] = argv[4];
    o["xtra"] = std::string(1, argv[4][std::strlen(argv[4]) - 1]);
    o["nprot"] = std::to_string(nus.nprot);
    o["nneut"] = std::to_string(nus.nneut);
    o["J2"] = std::to_string(nus.J2);
    o["parity"] = std::to_string(nus.parity);
    o["nshells-p"] = std::to_string(nus.nshells_p);
    o["nucleus"] = nus.nucleus;
    std::string sp;
    for (size_t i = 0; i < nus.shell_parity.size(); ++i) sp += (i ? "," : "") + std::to_string(nus.shell_parity[i]);
    o["shell-parity"] = sp;
    first = (argc >= 6 && std::strncmp(argv[5], "--", 2) != 0) ? 6 : 5;   // intfile (the interaction's name)
  }
  for (int i = first; i < argc; ++i) {
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
  // no_level: third line of <int>.spe, unless --nev; restart: its optional fourth line
  // (src/NuLnz/NuCoreX.f90:1664-1670)
  int nev = 0, restart = 0;
  {
    std::ifstream spe(o["int"] + ".spe");
    std::string l1, l2, l3, l4;
    if (!spe || !std::getline(spe, l1) || !std::getline(spe, l2) || !std::getline(spe, l3))
      die("cannot open " + o["int"] + ".spe or read no_level from its third line");
    nev = std::atoi(l3.c_str());
    if (std::getline(spe, l4)) restart = std::atoi(l4.c_str());
  }
  if (o.count("nev")) nev = std::atoi(o["nev"].c_str());
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
  char code[4];
  if (nsx_file_code(f.J2 / 2, nprot, nneut, code) != NSX_OK) die(nsx_last_error());
  const std::string prefix = o["nucleus"] + code;
  const int T2 = std::abs(nprot - nneut);
  // the thick-restart state: written at the end, read back for a restart (.spe line 4 > 0 and
  // the files of an earlier run present, as the reference's TRL does at NuCoreX.f90:266-292)
  const int cap = std::min(p.window, 112) + 1;
  std::vector<double> sV((size_t)cap * n), sT((size_t)cap * cap), sN((size_t)n), rV, rT, rN;
  nsx_state out_state{cap, sV.data(), sT.data(), sN.data(), 0.0, 0, 0}, in_state{};
  bool resuming = false;
  if (restart > 0) {
    std::ifstream probe(prefix + ".abz");
    if (probe) {
      rV.resize((size_t)cap * n);
      rT.resize((size_t)cap * cap);
      rN.resize((size_t)n);
      in_state = nsx_state{cap, rV.data(), rT.data(), rN.data(), 0.0, 0, 0};
      if (nsx_read_state(h, prefix.c_str(), &in_state) != NSX_OK) die(nsx_last_error());
      resuming = true;
      std::printf(" resuming from %s.abz / .trl (%d basis vectors, %d steps)\n", prefix.c_str(), in_state.m,
                  in_state.iterations);
    }
  }
  std::vector<double> ev(nev), vecs((size_t)nev * n);
  nsx_report rep;
  int rc = nsx_solve_ex(h, &p, resuming ? &in_state : nullptr, &out_state, ev.data(), vecs.data(), &rep);
  if (rc != NSX_OK) die(nsx_last_error());
  rc = nsx_write_state(h, prefix.c_str(), &out_state, ev.data(), vecs.data(), nev, o["int"].c_str(), T2);
  if (rc != NSX_OK) die(nsx_last_error());
  std::printf(" dimension %lld, %d Lanczos steps, %d H.v, %.3f s (H.v %.3f s)\n", (long long)n, rep.iterations,
              rep.matvecs, rep.seconds, rep.matvec_seconds);
  for (int i = 0; i < nev; ++i) std::printf("%10.3f%s", ev[i], (i % 5 == 4 || i == nev - 1) ? "\n" : "");
  std::printf(" wrote %s.abz .trl .lev .xvc\n", prefix.c_str());
  nsx_destroy(h);
  return 0;
}
