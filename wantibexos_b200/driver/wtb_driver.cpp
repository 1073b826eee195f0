// Host driver of the BSE exciton + optics path: the C++ counterpart of the reference's
// Fortran driver layer for BSE=T / BSE_BND=T / SPEC=T runs.  It keeps the reference's input
// grammar (stdin deck, params file) and writes the same output files, and calls the GPU
// through the C-ABI of libwtbgpu.so (include/wtbgpu.h).
//
// Reference structure mirrored here:
//   wtb_main.f90:60-357          program main (deck, params header, mesh, tool dispatch)
//   module_input_read.f90:235-816 input_read / param_out (log.dat)
//   module_input_read.f90:32-176  hamiltonian_input_read (params file, incl. SP merge)
//   bse_solver-tool-diel.f90      bsesolver  -> log_bse-diel.dat, sp_optics*.dat, tm_coef*.dat,
//                                               bse_opt_diel*.dat, exc_wf_n.dat
//   bse_kpath-tool.f90            bsebnds    -> bands_bse.dat, log_bse_kpath.dat, KLABELS-BSE.dat
//   bse_diel-tool(-pol).f90       bsedielraw(pol) -> bse_diel_*.dat / bse_diel-pol_*.dat
//   sp_diel-tool(-pol).f90        spdielraw(pol)  -> sp_diel_*.dat / sp_diel-pol_*.dat
//   diel-pp-*.f90, diel-pp-subs   bseoptprop(pol), spoptprop(pol) -> refractive index, ...
//   exciton_lifetime.f90          lifetime(pol) -> exciton_lifetime(-pol).dat
// Fortran list-directed output is compiler-specific; numeric parity (not byte parity) is the
// contract, and every number is printed with enough digits to be read back exactly.
#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/wtbgpu.h"
#include "../../include/wtb_driver.h"

namespace {

// ------------------------------------------------------------------------------ errors
struct Stop : std::runtime_error {
  explicit Stop(const std::string& m) : std::runtime_error(m) {}
};

void gpu_check(wtbg_ctx* ctx, int st, const char* where) {
  if (st != 0) {
    std::string m = std::string(where) + ": " + wtbg_error_string(st) + " (" + wtbg_last_error(ctx) + ")";
    throw Stop(m);
  }
}

// ------------------------------------------------------------------------------ deck
struct Deck {
  int nthreads = 1;
  int ngrid[3] = {1, 1, 1};
  double rk = 0.0;
  int nc = 1, nv = 1;
  double numdos = 6001, ebse0 = 0.0, ebsef = 3.0, numbse = 6001;
  double sme = (double)0.08f, cshift = (double)0.01f, exc = 0.0;
  double mshift[3] = {0, 0, 0};
  double ktol = (double)0.001f;
  std::string outputfolder = "./", calcparms = "./", meshtype = "MKH", coultype = "V3D";
  std::string orbw = "non declared file", kpaths = "non declared file", kpathsbse = "non declared file";
  std::string params;
  std::string sysdim = "3D", dft = "V", ta = "FA", ses = "AM15G";
  bool bandscalc = false, doscalc = false, bse = false, bsepol = false, bsekpath = false, spdiel = false;
  bool spdielpol = false, sppolbz = false, spec = false, berryk = false, berrybz = false, pponly = false;
  bool bsewf = false, tmcoef = false, dtfull = false, cpol = false, bset = false, bsetbnd = false;
  bool pce = false, renorm = true;
  int excwf0 = 1, excwff = 2;
  double ediel[3] = {1, 1, 1};
  double ez = 1.0, w = 0.0, lc = 1.0, r0 = 1.0;
  double st = 0, phavg = 0, temp = 0;
  double ctemp = (double)298.15f, tmax = (double)5e-6f, eg = 0, egd = 0, egs = 0, ebgs = 0;
  // keys of this implementation (the reference ignores unknown keys, so decks stay valid there):
  // GPU_SOLVER= DENSE | DAVIDSON, GPU_PRECISION= FP64 | BF16X3 (alias FAST), GPU_NEV=, GPU_TOL= (eV),
  // GPU_MAXIT=, GPU_HAYDOCK= (Lanczos steps of the fast spectrum), GPU_WARMSTART= (.npy network file)
  std::string gpu_solver = "DENSE", gpu_precision = "FP64", gpu_warmstart;
  int gpu_nev = 32, gpu_maxit = 400, gpu_haydock = 150;
  double gpu_tol = 1e-6;
};

// what bsesolver leaves for the spectrum stage of the same run
struct RunState {
  bool fast = false;      // the fast form produced the exciton table (GPU_SOLVER= DAVIDSON, converged)
  long long rows = 0;     // rows of bse_opt_diel.dat
  double e1 = 0, emax = 0;
};

// one record split into list-directed character items (quotes keep blanks)
std::vector<std::string> items_of(const std::string& line) {
  std::vector<std::string> out;
  size_t i = 0, n = line.size();
  while (i < n) {
    char c = line[i];
    if (c == ' ' || c == '\t' || c == ',' || c == '\r') {
      ++i;
      continue;
    }
    if (c == '"' || c == '\'') {
      size_t j = line.find(c, i + 1);
      if (j == std::string::npos) j = n;
      out.push_back(line.substr(i + 1, j - i - 1));
      i = j + 1;
      continue;
    }
    size_t j = i;
    while (j < n && line[j] != ' ' && line[j] != '\t' && line[j] != ',' && line[j] != '\r') ++j;
    out.push_back(line.substr(i, j - i));
    i = j;
  }
  return out;
}

std::string upper(std::string s) {
  for (char& c : s) c = (char)toupper(c);
  return s;
}

double num(const std::string& s) {
  std::string t = s;
  for (char& c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  double v = strtod(t.c_str(), &end);
  if (end == t.c_str()) throw Stop("bad number in deck: " + s);
  return v;
}

bool logical(const std::string& s) {
  size_t i = 0;
  while (i < s.size() && s[i] == '.') ++i;
  if (i >= s.size()) throw Stop("bad logical in deck");
  char c = (char)toupper(s[i]);
  if (c == 'T') return true;
  if (c == 'F') return false;
  throw Stop("bad logical in deck: " + s);
}

// input_read (module_input_read.f90:235-663): each READ takes two items "a b" starting on a
// fresh record; unknown keys are ignored.
Deck parse_deck(const std::string& text) {
  Deck d;
  std::vector<std::vector<std::string>> recs;
  {
    std::istringstream is(text);
    std::string line;
    while (std::getline(is, line)) recs.push_back(items_of(line));
  }
  std::vector<std::pair<std::string, std::string>> pairs;
  size_t r = 0;
  while (r < recs.size()) {
    while (r < recs.size() && recs[r].empty()) ++r;
    if (r >= recs.size()) break;
    if (recs[r].size() >= 2) {
      pairs.emplace_back(recs[r][0], recs[r][1]);
      ++r;
      continue;
    }
    std::string a = recs[r][0];
    ++r;
    while (r < recs.size() && recs[r].empty()) ++r;
    if (r >= recs.size()) break;
    pairs.emplace_back(a, recs[r][0]);
    ++r;
  }
  auto trunc = [](const std::string& s, size_t n) { return s.substr(0, std::min(n, s.size())); };
  for (auto& p : pairs) {
    const std::string& a = p.first;
    const std::string& b = p.second;
    if (a == "RNMD=") d.renorm = logical(b);
    else if (a == "PCE=") d.pce = logical(b);
    else if (a == "SES=") d.ses = trunc(b, 6);
    else if (a == "CTEMP=") d.ctemp = num(b);
    else if (a == "THMAX=") d.tmax = num(b);
    else if (a == "EG=") d.eg = num(b);
    else if (a == "EGD=") d.egd = num(b);
    else if (a == "EGS=") d.egs = num(b);
    else if (a == "EBGS=") d.ebgs = num(b);
    else if (a == "TA=") d.ta = trunc(b, 2);
    else if (a == "BSET=") d.bset = logical(b);
    else if (a == "BSET_BND=") d.bsetbnd = logical(b);
    else if (a == "TEMP=") d.temp = num(b);
    else if (a == "PHAVG=") d.phavg = num(b);
    else if (a == "ST=") d.st = num(b);
    else if (a == "DFT=") d.dft = trunc(b, 1);
    else if (a == "CSHIFT=") d.cshift = num(b);
    else if (a == "DTDIAG=") d.dtfull = logical(b);
    else if (a == "CPOL=") d.cpol = logical(b);
    else if (a == "SYSDIM=") d.sysdim = trunc(b, 5);
    else if (a == "R_0=") d.r0 = num(b);
    else if (a == "LC=") d.lc = num(b);
    else if (a == "EDIEL_Z=") d.ez = num(b);
    else if (a == "W_COUL=") d.w = num(b);
    else if (a == "TMCOEF=") d.tmcoef = logical(b);
    else if (a == "EXC_WF_F=") d.excwff = (int)num(b);
    else if (a == "EXC_WF_I=") d.excwf0 = (int)num(b);
    else if (a == "BSE_WF=") d.bsewf = logical(b);
    else if (a == "PP_ONLY=") d.pponly = logical(b);
    else if (a == "BERRY_BZ=") d.berrybz = logical(b);
    else if (a == "BERRY=") d.berryk = logical(b);
    else if (a == "SPEC=") d.spec = logical(b);
    else if (a == "OPT_BZ=") d.sppolbz = logical(b);
    else if (a == "DIEL=") d.spdiel = logical(b);
    else if (a == "BSE_BND=") d.bsekpath = logical(b);
    else if (a == "BSE=") d.bse = logical(b);
    else if (a == "DOS=") d.doscalc = logical(b);
    else if (a == "BANDS=") d.bandscalc = logical(b);
    else if (a == "RK=") d.rk = num(b);
    else if (a == "COULOMB_POT=") d.coultype = trunc(b, 5);
    else if (a == "MESH_TYPE=") d.meshtype = trunc(b, 70);
    else if (a == "OUTPUT=") d.outputfolder = trunc(b, 70);
    else if (a == "CALC_DATA=") d.calcparms = trunc(b, 70);
    else if (a == "NGX=") d.ngrid[0] = (int)num(b);
    else if (a == "NGY=") d.ngrid[1] = (int)num(b);
    else if (a == "NGZ=") d.ngrid[2] = (int)num(b);
    else if (a == "NBANDSC=") d.nc = (int)num(b);
    else if (a == "NBANDSV=") d.nv = (int)num(b);
    else if (a == "NEDOS=") d.numdos = num(b);
    else if (a == "ENSPECI=") d.ebse0 = num(b);
    else if (a == "ENSPECF=") d.ebsef = num(b);
    else if (a == "NESPEC=") d.numbse = num(b);
    else if (a == "SIGMA=") d.sme = num(b);
    else if (a == "KTOL=") d.ktol = num(b);
    else if (a == "PARAMS_FILE=") d.params = trunc(b, 70);
    else if (a == "KPATH_FILE=") d.kpaths = trunc(b, 70);
    else if (a == "KPATH_BSE=") d.kpathsbse = trunc(b, 70);
    else if (a == "ORB_W=") d.orbw = trunc(b, 70);
    else if (a == "EDIEL_T=") d.ediel[0] = num(b);
    else if (a == "EDIEL=") d.ediel[1] = num(b);
    else if (a == "EDIEL_B=") d.ediel[2] = num(b);
    else if (a == "EXC_CORR=") d.exc = num(b);
    else if (a == "NTHREADS=") d.nthreads = (int)num(b);
    else if (a == "SHIFT_1=") d.mshift[0] = num(b);
    else if (a == "SHIFT_2=") d.mshift[1] = num(b);
    else if (a == "SHIFT_3=") d.mshift[2] = num(b);
    else if (a == "GPU_SOLVER=") d.gpu_solver = upper(trunc(b, 10));
    else if (a == "GPU_PRECISION=") d.gpu_precision = upper(trunc(b, 10));
    else if (a == "GPU_NEV=") d.gpu_nev = (int)num(b);
    else if (a == "GPU_TOL=") d.gpu_tol = num(b);
    else if (a == "GPU_MAXIT=") d.gpu_maxit = (int)num(b);
    else if (a == "GPU_HAYDOCK=") d.gpu_haydock = (int)num(b);
    else if (a == "GPU_WARMSTART=") d.gpu_warmstart = trunc(b, 200);
  }
  if (d.gpu_solver != "DENSE" && d.gpu_solver != "DAVIDSON") throw Stop("GPU_SOLVER= must be DENSE or DAVIDSON");
  if (d.gpu_precision == "FAST") d.gpu_precision = "BF16X3";
  if (d.gpu_precision != "FP64" && d.gpu_precision != "BF16X3")
    throw Stop("GPU_PRECISION= must be FP64 or BF16X3 (FAST)");
  if (d.gpu_nev < 1 || d.gpu_nev > 32) throw Stop("GPU_NEV= must be between 1 and 32");
  if (!(d.gpu_tol > 0) || d.gpu_maxit < 1 || d.gpu_haydock < 2) throw Stop("bad GPU_TOL=, GPU_MAXIT= or GPU_HAYDOCK=");
  return d;
}

// ------------------------------------------------------------------------------ params
struct double2v {
  double x, y;
};

struct Model {
  std::string systype;
  double scs = 0, efermi = 0;
  double rlat[3][3] = {{0}};
  int w = 0, nvec = 0;
  std::vector<int> rvec;       // (nvec,3) column-major
  std::vector<int> deg;        // (nvec)
  std::vector<double> hre, him;  // (nvec,w,w) column-major
};

struct Reader {
  std::vector<std::string> lines;
  size_t pos = 0;
  explicit Reader(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Stop("Error opening wannier90 hr input file");
    std::string l;
    while (std::getline(f, l)) lines.push_back(l);
  }
  std::vector<std::string> rec() {
    while (pos < lines.size()) {
      auto it = items_of(lines[pos++]);
      if (!it.empty()) return it;
    }
    throw Stop("params file ended early");
  }
};

// hamiltonian_input_read (module_input_read.f90:32-176)
Model read_params(const std::string& path) {
  Reader rd(path);
  Model m;
  m.systype = rd.rec()[0].substr(0, 4);
  m.scs = num(rd.rec()[0]);
  m.efermi = num(rd.rec()[0]);
  for (int i = 0; i < 3; ++i) {
    auto t = rd.rec();
    if (t.size() < 3) throw Stop("bad lattice line in params file");
    for (int c = 0; c < 3; ++c) m.rlat[i][c] = num(t[c]);
  }
  struct Block {
    int w, nvec;
    std::vector<int> deg, rvec;
    std::vector<double> hre, him;
  };
  auto block = [&]() {
    Block b;
    rd.rec();  // header
    b.w = (int)num(rd.rec()[0]);
    b.nvec = (int)num(rd.rec()[0]);
    while ((int)b.deg.size() < b.nvec)
      for (auto& t : rd.rec()) b.deg.push_back((int)num(t));
    b.deg.resize(b.nvec);
    b.rvec.assign(3 * (size_t)b.nvec, 0);
    b.hre.assign((size_t)b.nvec * b.w * b.w, 0.0);
    b.him.assign((size_t)b.nvec * b.w * b.w, 0.0);
    for (int i = 0; i < b.nvec; ++i)
      for (int n = 0; n < b.w; ++n)
        for (int mm = 0; mm < b.w; ++mm) {
          auto t = rd.rec();
          if (t.size() < 7) throw Stop("bad hopping row in params file");
          for (int c = 0; c < 3; ++c) b.rvec[i + (size_t)b.nvec * c] = (int)num(t[c]);
          const size_t idx = (size_t)i + (size_t)b.nvec * ((size_t)mm + (size_t)b.w * n);
          b.hre[idx] = num(t[5]);
          b.him[idx] = num(t[6]);
        }
    return b;
  };
  std::string st = m.systype;
  while (!st.empty() && st.back() == ' ') st.pop_back();
  if (st == "SP") {
    Block u = block(), dn = block();
    m.w = u.w + dn.w;
    m.nvec = u.nvec + dn.nvec;
    m.deg = u.deg;
    m.deg.insert(m.deg.end(), dn.deg.begin(), dn.deg.end());
    m.rvec.assign(3 * (size_t)m.nvec, 0);
    m.hre.assign((size_t)m.nvec * m.w * m.w, 0.0);
    m.him.assign((size_t)m.nvec * m.w * m.w, 0.0);
    for (int i = 0; i < m.nvec; ++i) {
      const bool up = i < u.nvec;
      const Block& b = up ? u : dn;
      const int ib = up ? i : i - u.nvec, off = up ? 0 : u.w;
      for (int c = 0; c < 3; ++c) m.rvec[i + (size_t)m.nvec * c] = b.rvec[ib + (size_t)b.nvec * c];
      for (int n = 0; n < b.w; ++n)
        for (int mm = 0; mm < b.w; ++mm) {
          const size_t s = (size_t)ib + (size_t)b.nvec * ((size_t)mm + (size_t)b.w * n);
          const size_t d = (size_t)i + (size_t)m.nvec * ((size_t)(mm + off) + (size_t)m.w * (n + off));
          m.hre[d] = b.hre[s];
          m.him[d] = b.him[s];
        }
    }
  } else {
    Block b = block();
    m.w = b.w;
    m.nvec = b.nvec;
    m.deg = b.deg;
    m.rvec = b.rvec;
    m.hre = b.hre;
    m.him = b.him;
  }
  return m;
}

// ------------------------------------------------------------------------------ lattice
const double kPi32 = (double)3.14159274101257324219f;   // acos(-1.) in real(4)

void cross(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

// recvec (mhkpack_subs.f90:409-432)
void recvec(const double r[3][3], double b[3][3]) {
  double v23[3], v31[3], v12[3];
  cross(r[1], r[2], v23);
  cross(r[2], r[0], v31);
  cross(r[0], r[1], v12);
  const double vol = fabs(r[0][0] * v23[0] + r[0][1] * v23[1] + r[0][2] * v23[2]);
  const double s = (2.0 * kPi32) / vol;
  for (int c = 0; c < 3; ++c) {
    b[0][c] = s * v23[c];
    b[1][c] = s * v31[c];
    b[2][c] = s * v12[c];
  }
}

double vcell2d(const double r[3][3]) {
  double v[3];
  cross(r[0], r[1], v);
  return sqrt((v[0] * v[0]) + (v[1] * v[1]) + (v[2] * v[2]));
}

double vcell3d(const double r[3][3]) {
  double v[3];
  cross(r[0], r[1], v);
  return fabs(v[0] * r[2][0] + v[1] * r[2][1] + v[2] * r[2][2]);
}

// monhkhorst_pack / monhkhorst_packq (mhkpack_subs.f90:305-407); kpt (nk,3) column-major
std::vector<double> kmesh(const int n[3], const double shift[3], const double r[3][3], const double* q) {
  double b[3][3];
  recvec(r, b);
  double ks[3];
  for (int c = 0; c < 3; ++c) ks[c] = b[0][c] * shift[0] + b[1][c] * shift[1] + b[2][c] * shift[2];
  const int nk = n[0] * n[1] * n[2];
  std::vector<double> k(3 * (size_t)nk);
  int cnt = 0;
  for (int i = 0; i < n[0]; ++i)
    for (int j = 0; j < n[1]; ++j)
      for (int l = 0; l < n[2]; ++l) {
        for (int c = 0; c < 3; ++c) {
          double v;
          if (q)
            v = q[c] + (b[0][c] / (double)n[0]) * (double)i + (b[1][c] / (double)n[1]) * (double)j +
                (b[2][c] / (double)n[2]) * (double)l + ks[c];
          else
            v = (b[0][c] / (double)n[0]) * (double)i + (b[1][c] / (double)n[1]) * (double)j +
                (b[2][c] / (double)n[2]) * (double)l + ks[c];
          k[cnt + (size_t)nk * c] = v;
        }
        ++cnt;
      }
  return k;
}

// rkmesh / rkmesh2D (mhkpack_subs.f90:2-52)
void rkmesh(double rk, const double r[3][3], int ng[3], bool twod) {
  double b[3][3];
  recvec(r, b);
  for (int i = 0; i < 3; ++i) {
    const double vs = sqrt(b[i][0] * b[i][0] + b[i][1] * b[i][1] + b[i][2] * b[i][2]) / (2 * kPi32);
    ng[i] = (int)std::max(1.0, (rk * vs) + 0.5);
  }
  if (twod) ng[2] = 1;
}

// ------------------------------------------------------------------------------ formats
std::string F(double x, int w, int d) {
  char buf[64];
  snprintf(buf, sizeof buf, "%*.*f", w, d, x);
  std::string s(buf);
  if ((int)s.size() > w) return std::string(w, '*');
  if (s.find("nan") != std::string::npos || s.find("inf") != std::string::npos) {
    std::string t = std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity");
    return std::string(std::max(0, w - (int)t.size()), ' ') + t;
  }
  return s;
}

// F(x, w, d) appended to out without temporaries (the large per-state tables)
void append_F(std::string& out, double x, int w, int d) {
  if (std::isnan(x) || std::isinf(x)) {
    out += F(x, w, d);
    return;
  }
  char buf[64];
  const int n = snprintf(buf, sizeof buf, "%*.*f", w, d, x);
  if (n > w || n < 0) out.append((size_t)w, '*');
  else out.append(buf, (size_t)n);
}

// Rows [0, n) of a table formatted by fmt(i, out) on several host threads, joined in row order
// (the text is the same as one sequential pass).
template <class Fn>
std::string format_rows(long long n, size_t per_row, Fn fmt) {
  const unsigned hw = std::thread::hardware_concurrency();
  const int nt = (int)std::max<long long>(1, std::min<long long>(std::min<unsigned>(hw ? hw : 1u, 32u), n / 2048 + 1));
  std::vector<std::string> part(nt);
  auto work = [&](int t) {
    const long long a = n * t / nt, b = n * (t + 1) / nt;
    part[t].reserve((size_t)(b - a) * per_row);
    for (long long i = a; i < b; ++i) fmt(i, part[t]);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < nt; ++t) th.emplace_back(work, t);
  work(0);
  for (auto& x : th) x.join();
  size_t tot = 0;
  for (auto& q : part) tot += q.size();
  std::string out;
  out.reserve(tot);
  for (auto& q : part) out += q;
  return out;
}

// Ew.d with the 0.dddd mantissa of Fortran output
std::string E(double x, int w, int d) {
  if (std::isnan(x) || std::isinf(x)) {
    std::string t = std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity");
    return std::string(std::max(0, w - (int)t.size()), ' ') + t;
  }
  std::string body;
  if (x == 0.0) {
    body = "0." + std::string(d, '0') + "E+00";
  } else {
    // format |x| with d significant digits, then shift the decimal point
    char buf[64];
    snprintf(buf, sizeof buf, "%.*e", d - 1, fabs(x));
    // buf = m.mmmE+xx  -> 0.mmmm E(xx+1)
    std::string s(buf);
    const size_t epos = s.find('e');
    std::string mant = s.substr(0, epos);
    int ex = atoi(s.c_str() + epos + 1) + 1;
    mant.erase(std::remove(mant.begin(), mant.end(), '.'), mant.end());
    char eb[16];
    if (std::abs(ex) < 100) snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    body = (x < 0 ? "-0." : "0.") + mant + eb;
  }
  if ((int)body.size() > w) return std::string(w, '*');
  return std::string(w - body.size(), ' ') + body;
}

std::string I(long long v, int w) {
  char buf[64];
  snprintf(buf, sizeof buf, "%*lld", w, v);
  return buf;
}

std::string LD(double x) {   // list-directed real(8)
  char buf[64];
  snprintf(buf, sizeof buf, " %24.16E", x);
  return buf;
}
std::string LS(float x) {    // list-directed real(4)
  char buf[64];
  snprintf(buf, sizeof buf, " %15.8E", (double)x);
  return buf;
}
std::string LI(long long v) { return I(v, 12); }

std::string join_path(const std::string& folder, const std::string& name) { return folder + name; }

struct Out {
  FILE* f = nullptr;
  std::string path;
  Out(const std::string& p, const char* errmsg) : path(p) {
    f = fopen(p.c_str(), "w");
    if (!f) throw Stop(errmsg);
  }
  ~Out() {
    if (f) fclose(f);
  }
  void line(const std::string& s) { fprintf(f, "%s\n", s.c_str()); }
  void flush() { fflush(f); }
};

std::string stamp(const char* what) {
  time_t t = time(nullptr);
  struct tm lt;
  localtime_r(&t, &lt);
  char buf[160];
  snprintf(buf, sizeof buf, " %s  day%12d%12d hours%12d min%12d seg", what, lt.tm_mday, lt.tm_hour, lt.tm_min,
           lt.tm_sec);
  return buf;
}

int coul_code(const std::string& s0) {
  std::string s = s0;
  while (!s.empty() && s.back() == ' ') s.pop_back();
  if (s == "V2DK") return WTBG_V2DK;
  if (s == "V3D") return WTBG_V3D;
  if (s == "V3DL") return WTBG_V3DL;
  if (s == "V2DT") return WTBG_V2DT;
  if (s == "V2DT2") return WTBG_V2DT2;
  if (s == "V2DOH") return WTBG_V2DOH;
  if (s == "V2DRK") return WTBG_V2DRK;
  if (s == "V1DT") return WTBG_V1DT;
  if (s == "V0DT") return WTBG_V0DT;
  throw Stop("Wrong Coulomb Potential");
}

wtbg_coulomb coulomb_of(const Deck& d) {
  wtbg_coulomb p{};
  p.coultype = coul_code(d.coultype);
  for (int i = 0; i < 3; ++i) {
    p.ngrid[i] = d.ngrid[i];
    p.ediel[i] = d.ediel[i];
  }
  p.ktol = d.ktol;
  p.lc = d.lc;
  p.ez = d.ez;
  p.w = d.w;
  p.r0 = d.r0;
  return p;
}

void upload_model(wtbg_ctx* ctx, const Model& m) {
  double rl[9];
  for (int i = 0; i < 3; ++i)
    for (int c = 0; c < 3; ++c) rl[i + 3 * c] = m.rlat[i][c];
  gpu_check(ctx, wtbg_set_model(ctx, m.w, m.nvec, m.hre.data(), m.him.data(), m.rvec.data(), m.deg.data(), rl,
                                m.efermi, m.scs),
            "wtbg_set_model");
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------------------ log.dat
void param_out(Out& o, const Deck& d) {
  auto L = [&](const std::string& s) { o.line(s); };
  auto pad = [](const std::string& s, size_t n) {
    std::string t = s.substr(0, std::min(n, s.size()));
    return t + std::string(n - t.size(), ' ');
  };
  auto f84 = [](double x) { return F(x, 8, 4); };
  auto l1 = [](bool b) { return std::string(b ? "T" : "F"); };
  L("NTHREADS= " + std::to_string(d.nthreads));
  L("SYSDIM= " + pad(d.sysdim, 2));
  L("DFT= " + pad(d.dft, 1));
  L("");
  L(" INPUT/OUTPUT FILES");
  L("");
  L("OUTPUT= " + pad(d.outputfolder, 70));
  L("CALC_DATA= " + pad(d.calcparms, 70));
  L("PARAMS_FILE= " + pad(d.params, 70));
  L("KPATH_FILE= " + pad(d.kpaths, 70));
  L("KPATH_BSE= " + pad(d.kpathsbse, 70));
  L("ORB_W= " + pad(d.orbw, 70));
  L("");
  L(" CONTROL");
  L("");
  L("BANDS= " + l1(d.bandscalc));
  L("DOS= " + l1(d.doscalc));
  L("BSE= " + l1(d.bse));
  L("BSET= " + l1(d.bset));
  L("BSE_BND= " + l1(d.bsekpath));
  L("BSET_BND= " + l1(d.bsetbnd));
  L("DIEL= " + l1(d.spdiel));
  L("OPT_BZ= " + l1(d.sppolbz));
  L("SPEC= " + l1(d.spec));
  L("BERRY_BZ= " + l1(d.berrybz));
  L("BERRY= " + l1(d.berryk));
  L("PP_ONLY= " + l1(d.pponly));
  L("BSE_WF= " + l1(d.bsewf));
  L("TMCOEF= " + l1(d.tmcoef));
  L("DTDIAG= " + l1(d.dtfull));
  L("CPOL= " + l1(d.cpol));
  L("PCE= " + l1(d.pce));
  L("");
  L(" K-MESH");
  L("");
  L("NGX= " + std::to_string(d.ngrid[0]));
  L("NGY= " + std::to_string(d.ngrid[1]));
  L("NGZ= " + std::to_string(d.ngrid[2]));
  L("SHIFT_1= " + f84(d.mshift[0]));
  L("SHIFT_2= " + f84(d.mshift[1]));
  L("SHIFT_3= " + f84(d.mshift[2]));
  L("");
  L(" DOS");
  L("");
  L("NEDOS= " + std::to_string((long long)d.numdos));
  L("SIGMA= " + f84(d.sme));
  L("");
  L(" BSE/OPTICAL PROPERTIES");
  L("");
  L("NBANDSC= " + std::to_string(d.nc));
  L("NBANDSV= " + std::to_string(d.nv));
  L("ENSPECI= " + f84(d.ebse0));
  L("ENSPECF= " + f84(d.ebsef));
  L("NESPEC= " + std::to_string((long long)d.numbse));
  L("KTOL= " + f84(d.ktol));
  L("EXC_WF_I= " + std::to_string(d.excwf0));
  L("EXC_WF_F= " + std::to_string(d.excwff));
  L("COULOMB_POT= " + pad(d.coultype, 5));
  L("CSHIFT= " + f84(d.cshift));
  L("RNMD= " + l1(d.renorm));
  L("");
  L(" PARAMETERS FOR COULOMB POTENTIALS");
  L("");
  L("EDIEL_Z= " + f84(d.ez));
  L("W_COUL= " + f84(d.w));
  L("LC= " + f84(d.lc));
  L("R_0= " + f84(d.r0));
  L("EDIEL_T= " + f84(d.ediel[0]));
  L("EDIEL_B= " + f84(d.ediel[2]));
  L("EDIEL= " + f84(d.ediel[1]));
  L("");
  L(" PARAMETERS FOR BSE with Temperature Effects");
  L("");
  L("TA= " + pad(d.ta, 2));
  L("ST= " + f84(d.st));
  L("PHAVG= " + f84(d.phavg));
  L("TEMP= " + f84(d.temp));
  L("");
  L(" PARAMETERS FOR PCE");
  L("");
  L("SES= " + pad(d.ses, 6));
  L("CTEMP= " + f84(d.ctemp));
  L("THMAX= " + E(d.tmax, 15, 4));
  L("EG= " + f84(d.eg));
  L("EGD= " + f84(d.egd));
  L("EGS= " + f84(d.egs));
  L("EBGS= " + f84(d.ebgs));
  L("");
  L("");
  o.flush();
}

// ------------------------------------------------------------------------------ bsesolver
// Temperature gap correction tcor of bsesolvertemp / bsebndstemp (TA= FA | VE | BE):
// gapcortemp (general_subs.f90:569-586) and gapcortemp2 (:588-605), kB a real(4) literal.
double temperature_shift(const Deck& d) {
  const double kb = (double)8.617330350e-5f;
  if (d.ta == "VE") {
    const double aux1 = d.phavg / (2.0 * kb * d.temp);
    return -d.st * d.phavg * ((1.0 / std::tanh(aux1)) - 1.0);
  }
  if (d.ta == "BE") return -((2.0 * d.st) / (std::exp(d.phavg / d.temp) - 1.0));
  return 0.0;
}

// The model with the temperature scissors (scs + tcor) and the context's temperature mode.
void upload_model_temp(wtbg_ctx* ctx, const Model& m, const Deck& d, bool temp) {
  Model mm = m;
  if (temp) mm.scs += temperature_shift(d);
  upload_model(ctx, mm);
  gpu_check(ctx, wtbg_set_temperature(ctx, temp ? 1 : 0, d.temp), "wtbg_set_temperature");
}

// bsesolver (bse_solver-tool-diel.f90) and, with d.bset, bsesolvertemp
// (bse_solver-tool-diel-temp.f90): same files; the temperature run adds the log line, the
// scissors tcor and the occupation factors.
// sp_optics.dat, sp_optics-pol.dat and (TM_COEF) tm_coef*.dat from the device sp table
// (bse_solver-tool-diel.f90:338-423, sp_solver-tool-diel.f90:98-175; Bubblem order)
void write_sp_tables(const Deck& d, int nk, long long N, const std::vector<float>& vr, Out& f401, Out& f403, FILE* f402,
                     FILE* f404) {
  f401.line(" #  energy  xx  yy  zz  xy  xz  yz");
  f403.line(" #  energy  xx  yy  zz  sp  sm");
  if (d.tmcoef) {
    fprintf(f402, " number of kpoints:%12d\n number of conduction states%12d\n number of valence states%12d\n", nk,
            d.nc, d.nv);
    fprintf(f402, " #  kx  ky  kz  nocp  nc  nv  energy  xx  yy  zz  xy  xz  yz\n");
    fprintf(f404, " number of kpoints:%12d\n number of conduction states%12d\n number of valence states%12d\n", nk,
            d.nc, d.nv);
    fprintf(f404, " #  kx  ky  kz  nocp  nc  nv  energy  xx  yy  zz  sp  sm\n");
  }
  auto col = [&](long long i, int c) { return (double)vr[i + (size_t)N * c]; };
  auto i100 = [](double v) {   // I10.0: a zero value prints as blanks
    long long k = (long long)v;
    return k == 0 ? std::string(10, ' ') : I(k, 10);
  };
  {
    const std::string b401 = format_rows(N, 106, [&](long long i, std::string& o) {
      for (int c = 6; c <= 12; ++c) append_F(o, col(i, c), 15, 4);
      o += '\n';
    });
    fputs(b401.c_str(), f401.f);
    const std::string b403 = format_rows(N, 91, [&](long long i, std::string& o) {
      for (int c : {6, 7, 8, 9, 13, 14}) append_F(o, col(i, c), 15, 4);
      o += '\n';
    });
    fputs(b403.c_str(), f403.f);
    if (d.tmcoef) {
      auto head = [&](long long i, std::string& o) {
        for (int c = 0; c < 3; ++c) append_F(o, col(i, c), 10, 4);
        for (int c = 3; c < 6; ++c) o += i100(col(i, c));
        for (int c = 6; c < 10; ++c) append_F(o, col(i, c), 10, 4);
      };
      const std::string b402 = format_rows(N, 131, [&](long long i, std::string& o) {
        head(i, o);
        for (int c = 10; c <= 12; ++c) append_F(o, col(i, c), 10, 4);
        o += '\n';
      });
      fputs(b402.c_str(), f402);
      const std::string b404 = format_rows(N, 121, [&](long long i, std::string& o) {
        head(i, o);
        for (int c = 13; c <= 14; ++c) append_F(o, col(i, c), 10, 4);
        o += '\n';
      });
      fputs(b404.c_str(), f404);
    }
  }
}

// Network parameters of the learned warm start as saved by warmstart_sweep (--save FILE.npy):
// a little-endian float32 .npy vector of wtbg_net_num_params() values.
std::vector<float> read_npy_f32(const std::string& path, long long n) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) throw Stop("Error opening GPU_WARMSTART file " + path);
  unsigned char magic[8];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "\x93NUMPY", 6) != 0) {
    fclose(f);
    throw Stop("GPU_WARMSTART file is not a .npy file");
  }
  size_t hlen = 0;
  if (magic[6] == 1) {
    unsigned char b[2];
    if (fread(b, 1, 2, f) != 2) hlen = 0;
    else hlen = b[0] | (b[1] << 8);
  } else {
    unsigned char b[4];
    if (fread(b, 1, 4, f) != 4) hlen = 0;
    else hlen = b[0] | (b[1] << 8) | (b[2] << 16) | ((size_t)b[3] << 24);
  }
  std::string hdr(hlen, ' ');
  if (hlen == 0 || fread(&hdr[0], 1, hlen, f) != hlen || hdr.find("<f4") == std::string::npos ||
      hdr.find("'fortran_order': False") == std::string::npos) {
    fclose(f);
    throw Stop("GPU_WARMSTART file must hold a C-ordered float32 vector");
  }
  std::vector<float> p((size_t)n);
  const size_t got = fread(p.data(), 4, (size_t)n, f);
  fclose(f);
  if ((long long)got != n) throw Stop("GPU_WARMSTART file holds fewer values than the network has parameters");
  return p;
}

// Start block of the fast form from the learned network: the 32 predicted vectors, then
// nb - 32 fixed pseudo-random columns (glob = Q = 0, R_0, EDIEL_T as in the training sweep).
std::vector<double> warm_start_block(wtbg_ctx* ctx, const Deck& d, long long N, int nb) {
  std::vector<float> p = read_npy_f32(d.gpu_warmstart, wtbg_net_num_params());
  wtbg_net* net = nullptr;
  gpu_check(ctx, wtbg_net_create(ctx, &net, 1), "wtbg_net_create");
  std::vector<double> X0(2 * (size_t)N * nb, 0.0);
  const double glob[5] = {0.0, 0.0, 0.0, d.r0, d.ediel[0]};
  int st = wtbg_net_set_params(net, p.data());
  if (st == 0) st = wtbg_net_predict(net, glob, X0.data());
  wtbg_net_destroy(net);
  gpu_check(ctx, st, "wtbg_net_predict");
  uint64_t x = 0x9E3779B97F4A7C15ull;
  for (size_t i = 2 * (size_t)N * 32; i < X0.size(); ++i) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    X0[i] = (double)(x >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  return X0;
}

// The exciton solve of bsesolver.  GPU_SOLVER= DENSE (default): ZHEEV's role, every eigenpair
// (wtbg_bse_solve).  GPU_SOLVER= DAVIDSON: the GPU_NEV lowest excitons by block Davidson to
// residual GPU_TOL, with the split-BF16 tensor-core product under GPU_PRECISION= BF16X3, and the
// highest exciton to 1e-3 eV for the broadening rule; if the Davidson run ends above GPU_TOL after
// GPU_MAXIT iterations, or in the temperature form, the dense solve runs instead and the run
// continues exactly as a dense run (logged in log_bse-diel.dat).
RunState exciton_solve(wtbg_ctx* ctx, const Deck& d, long long N, bool temp, Out& log, std::vector<double>& W,
                       std::vector<double>& act, std::vector<double>& Xfast) {
  RunState rs;
  rs.rows = N;
  if (d.gpu_solver == "DAVIDSON") {
    const int nev = (int)std::min<long long>(d.gpu_nev, N);
    const int nb = std::min(40, ((nev + 8 + 7) / 8) * 8);
    if (temp) {
      log.line(" fast form: no temperature form; dense FP64 solve used");
    } else if (N < 4LL * nb) {
      log.line(" fast form: BSE dimension below four Davidson blocks; dense FP64 solve used");
    } else {
      gpu_check(ctx, wtbg_set_fast_product(ctx, d.gpu_precision == "BF16X3" ? 1 : 0), "wtbg_set_fast_product");
      std::vector<double> X0;
      if (!d.gpu_warmstart.empty()) X0 = warm_start_block(ctx, d, N, nb);
      std::vector<double> w(nev), a(8 * (size_t)nev), X(d.bsewf ? 2 * (size_t)N * nev : 0);
      int it = 0;
      double mr = 0.0;
      const int st = wtbg_bse_davidson(ctx, nev, nb, 0, d.gpu_maxit, d.gpu_tol, X0.empty() ? nullptr : X0.data(),
                                       d.dtfull, d.cpol, w.data(), a.data(), d.bsewf ? X.data() : nullptr, &it, &mr);
      if (st == WTBG_OK) {
        double top = 0.0, mr2 = 0.0;
        int it2 = 0;
        const int st2 = wtbg_bse_davidson(ctx, 1, 8, 1, 300, 1e-3, nullptr, 0, 0, &top, nullptr, nullptr, &it2, &mr2);
        if (st2 != WTBG_OK && st2 != WTBG_ERR_NOCONV) gpu_check(ctx, st2, "wtbg_bse_davidson (highest exciton)");
        rs.fast = true;
        rs.rows = nev;
        rs.e1 = w[0];
        rs.emax = top;
        W = w;
        act = a;
        Xfast = X;
        log.line(" fast form: lowest" + LI(nev) + " excitons by block Davidson," + LI(it) +
                 " iterations, max residual" + LD(mr) + " eV");
        return rs;
      }
      if (st != WTBG_ERR_NOCONV) gpu_check(ctx, st, "wtbg_bse_davidson");
      log.line(" fast form: block Davidson stopped at max residual" + LD(mr) + " eV after" + LI(it) +
               " iterations; dense FP64 solve used");
    }
    log.flush();
  }
  W.assign((size_t)N, 0.0);
  act.assign(8 * (size_t)N, 0.0);
  gpu_check(ctx, wtbg_bse_solve(ctx, d.dtfull, d.cpol, W.data(), act.data()), "wtbg_bse_solve");
  return rs;
}

RunState bsesolver(wtbg_ctx* ctx, const Deck& d, const Model& m, Timings* tm) {
  const std::string of = d.outputfolder;
  Out log(join_path(of, "log_bse-diel.dat"), "Error opening log_bse-diel output file");
  Out f301(join_path(of, "bse_opt_diel.dat"), "Error opening bse_opt_diel output file");
  Out f302(join_path(of, "bse_opt_diel-pol.dat"), "Error opening output file");
  Out f401(join_path(of, "sp_optics.dat"), "Error opening bse_opt_diel-pol output file");
  FILE* f402 = nullptr;
  FILE* f404 = nullptr;
  if (d.tmcoef) {
    f402 = fopen(join_path(of, "tm_coef.dat").c_str(), "w");
    f404 = fopen(join_path(of, "tm_coef-pol.dat").c_str(), "w");
    if (!f402 || !f404) throw Stop("Error opening tm_coef output file");
  }
  Out f403(join_path(of, "sp_optics-pol.dat"), "Error opening sp_optics-pol output file");
  double t0 = now_s();
  const bool temp = d.bset && !d.bse;
  upload_model_temp(ctx, m, d, temp);
  gpu_check(ctx, wtbg_set_precision(ctx, d.gpu_precision == "BF16X3" ? 1 : 0), "wtbg_set_precision");
  f301.line(" #  exciton energy  xx  yy  zz xy  xz  yz");
  f302.line(" #  exciton energy  xx  yy  zz sp  sm");
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  const long long N = (long long)nk * d.nc * d.nv;
  log.line("");
  log.line("");
  log.line("");
  log.line(" threads:" + LI(d.nthreads));
  log.line("");
  if (temp) {
    log.line(" temperature" + LD(d.temp));
    log.line("");
  }
  log.line(" grid:" + LI(d.ngrid[0]) + LI(d.ngrid[1]) + LI(d.ngrid[2]));
  log.line("");
  log.line("  ktol-coulomb:" + E(d.ktol, 15, 4));
  log.line("");
  log.line(" kmesh shift:" + F(d.mshift[0], 15, 4) + F(d.mshift[1], 15, 4) + F(d.mshift[2], 15, 4));
  log.line("");
  log.line(" conduction bands, nc:" + LI(d.nc) + "   valence bands, nv:" + LI(d.nv));
  log.line("");
  log.line("");
  log.line(stamp("begin"));
  log.line("");
  log.flush();
  std::vector<double> kpt = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  const int nb = d.nc + d.nv;
  std::vector<double> eigv((size_t)nk * nb);
  std::vector<int> nocpk(nk);
  double egap = 0;
  gpu_check(ctx, wtbg_bands(ctx, nk, kpt.data(), d.nv, d.nc, eigv.data(), nullptr, nocpk.data(), &egap), "wtbg_bands");
  double t1 = now_s();
  if (tm) tm->bands = t1 - t0;
  log.line(" direct gap:" + LD(egap));
  log.line(" eigenvalues and eigenvectors calculated");
  log.line(" quantum numbers for exciton basis set finished");
  log.flush();
  // single-particle optics (bse_solver-tool-diel.f90:338-423)
  std::vector<double> hr(2 * 5 * (size_t)N);
  gpu_check(ctx, wtbg_velocity(ctx, d.cshift, hr.data()), "wtbg_velocity");
  std::vector<float> vr(15 * (size_t)N);
  gpu_check(ctx, wtbg_sp_table(ctx, vr.data()), "wtbg_sp_table");
  write_sp_tables(d, nk, N, vr, f401, f403, f402, f404);
  log.line(" single particle optics finished");
  log.flush();
  double t2 = now_s();
  if (tm) tm->sp = t2 - t1;
  wtbg_coulomb p = coulomb_of(d);
  gpu_check(ctx, wtbg_bse_build(ctx, &p), "wtbg_bse_build");
  log.line(" exciton Hamiltonian matrix finished");
  log.flush();
  double t3 = now_s();
  if (tm) tm->build = t3 - t2;
  if (d.gpu_precision == "BF16X3") log.line(" GPU_PRECISION= BF16X3: split-BF16 tensor-core Fourier sums and overlaps");
  std::vector<double> W, act, Xfast;
  RunState rs = exciton_solve(ctx, d, N, temp, log, W, act, Xfast);
  const long long rows = rs.rows;
  double t4 = now_s();
  if (tm) tm->solve = t4 - t3;
  if (d.bsewf) {
    const int a0 = std::max(1, d.excwf0), a1 = (int)std::min<long long>(d.excwff, rows);
    if (a1 >= a0) {
      std::vector<double> A(2 * (size_t)N * (a1 - a0 + 1));
      if (rs.fast) {
        for (int n = a0; n <= a1; ++n) {   // gauge of wtbg_bse_eigvecs: unit norm, last component real >= 0
          const double* x = Xfast.data() + 2 * (size_t)N * (n - 1);
          double* y = A.data() + 2 * (size_t)N * (n - a0);
          double nrm = 0.0;
          for (long long i = 0; i < N; ++i) nrm += x[2 * i] * x[2 * i] + x[2 * i + 1] * x[2 * i + 1];
          const double lr = x[2 * (N - 1)], li = x[2 * (N - 1) + 1], r = std::hypot(lr, li);
          const double cr = r > 0 ? lr / r : 1.0, ci = r > 0 ? -li / r : 0.0, sc = nrm > 0 ? 1.0 / std::sqrt(nrm) : 1.0;
          for (long long i = 0; i < N; ++i) {
            y[2 * i] = sc * (x[2 * i] * cr - x[2 * i + 1] * ci);
            y[2 * i + 1] = sc * (x[2 * i] * ci + x[2 * i + 1] * cr);
          }
          y[2 * (N - 1) + 1] = 0.0;
        }
      } else {
        gpu_check(ctx, wtbg_bse_eigvecs(ctx, a0, a1, A.data()), "wtbg_bse_eigvecs");
      }
      for (int n = a0; n <= a1; ++n) {
        // excwf2 (bse_subs.f90:534-576)
        Out o(join_path(of, "exc_wf_" + std::to_string(n) + ".dat"), "Error opening wf BSE output file");
        o.line(" # excitonic state" + LI(n));
        o.line(" # exciton energy:" + LD(W[n - 1]));
        o.line(" # number occupied states" + LI(nocpk[0]) + "(not valid for metallic systems)");
        o.line(" # Number of conduction states" + LI(d.nc));
        o.line(" # Number of valence states" + LI(d.nv));
        o.line(" # Number of kpoints" + LI(nk));
        o.line(" # nocpk kx ky kz nc nv re_wf imag_wf");
        std::string buf;
        const double* an = A.data() + 2 * (size_t)N * (n - a0);
        for (long long i = 0; i < N; ++i) {
          const int k = (int)(i / (d.nc * d.nv)), c = (int)((i % (d.nc * d.nv)) / d.nv) + d.nv + 1,
                    v = (int)(i % d.nv) + 1;
          buf += I(nocpk[k], 12) + F(kpt[k], 15, 4) + F(kpt[k + (size_t)nk], 15, 4) + F(kpt[k + 2 * (size_t)nk], 15, 4) +
                 I(nocpk[k] + c - d.nv, 12) + I(nocpk[k] - d.nv + v, 12) + E(an[2 * i], 15, 4) +
                 E(an[2 * i + 1], 15, 4) + "\n";
        }
        fputs(buf.c_str(), o.f);
      }
    }
  }
  log.line(" exciton Hamiltonian diagonalized");
  log.line(" exciton ground state" + LD(W[0]));
  const char* comps[] = {"xx tensor component", "yy tensor component", "zz tensor component"};
  for (auto c : comps) log.line(std::string(" ") + c);
  if (d.dtfull) {
    log.line(" xy tensor component");
    log.line(" xz tensor component");
    log.line(" yz tensor component");
  } else {
    log.line(" xy tensor component set to 0");
    log.line(" xz tensor component set to 0");
    log.line(" yz tensor component set to 0");
  }
  log.line(d.cpol ? " sp polarization" : " sp polarization set to 0");
  log.line(d.cpol ? " sm polarization" : " sm polarization set to 0");
  log.line(" optics finished");
  log.flush();
  {
    const std::string b301 = format_rows(rows, 106, [&](long long i, std::string& o) {
      append_F(o, W[i], 15, 4);
      for (int c = 0; c < 6; ++c) append_F(o, act[i + (size_t)rows * c], 15, 4);
      o += '\n';
    });
    fputs(b301.c_str(), f301.f);
    if (d.cpol) {
      const std::string b302 = format_rows(rows, 91, [&](long long i, std::string& o) {
        append_F(o, W[i], 15, 4);
        for (int c : {0, 1, 2, 6, 7}) append_F(o, act[i + (size_t)rows * c], 15, 4);
        o += '\n';
      });
      fputs(b302.c_str(), f302.f);
    }
  }
  log.line("");
  log.line(stamp("end"));
  log.line("");
  if (f402) fclose(f402);
  if (f404) fclose(f404);
  if (tm) tm->write_opt = now_s() - t4;
  return rs;
}

// ------------------------------------------------------------------------------ bsebnds
void bsebnds(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  std::ifstream kf(d.kpathsbse);
  if (!kf) throw Stop("Error opening bse-kpath input file");
  Out log(join_path(of, "log_bse_kpath.dat"), "Error opening log_bse_kpath output file");
  Out f400(join_path(of, "bands_bse.dat"), "Error opening bands_bse output file");
  const bool temp = d.bsetbnd && !d.bsekpath;
  upload_model_temp(ctx, m, d, temp);
  std::vector<std::string> kl;
  {
    std::string l;
    while (std::getline(kf, l))
      if (!items_of(l).empty()) kl.push_back(l);
  }
  if (kl.size() < 2) throw Stop("bad bse-kpath file");
  const int nks = (int)num(items_of(kl[0])[0]);
  const int npts = (int)num(items_of(kl[1])[0]);
  if ((int)kl.size() < 2 + nks) throw Stop("bad bse-kpath file");
  std::vector<std::array<double, 3>> ks(nks);
  for (int i = 0; i < nks; ++i) {
    auto t = items_of(kl[2 + i]);
    for (int c = 0; c < 3; ++c) ks[i][c] = num(t[c]);
  }
  // kpathbse (mhkpack_subs.f90:132-208): the fraction (i-1.)/(npts-1.) is real(4)
  double b[3][3];
  recvec(m.rlat, b);
  std::vector<std::array<double, 3>> kx(nks);
  for (int i = 0; i < nks; ++i)
    for (int c = 0; c < 3; ++c) kx[i][c] = ks[i][0] * b[0][c] + ks[i][1] * b[1][c] + ks[i][2] * b[2][c];
  const int half = nks / 2;
  std::vector<double> kdis(half);
  double tot = 0.0;
  for (int i = 0; i < half; ++i) {
    const double dx = kx[2 * i + 1][0] - kx[2 * i][0], dy = kx[2 * i + 1][1] - kx[2 * i][1],
                 dz = kx[2 * i + 1][2] - kx[2 * i][2];
    kdis[i] = sqrt(dx * dx + dy * dy + dz * dz);
    tot += kdis[i];
  }
  for (auto& v : kdis) v = v / tot;
  const int nq = half * npts;
  std::vector<std::array<double, 4>> qp(nq);
  {
    Out kl_out(join_path(of, "KLABELS-BSE.dat"), "Error opening KLABELS-BSE output file");
    double acc = 0.0;
    kl_out.line(LS(0.0f));
    for (int j = 0; j < half; ++j) {
      for (int i = 0; i < npts; ++i) {
        const double t = (double)((float)i / (float)(npts - 1));
        auto& q = qp[(size_t)j * npts + i];
        q[0] = acc + kdis[j] * t;
        for (int c = 0; c < 3; ++c) q[1 + c] = kx[2 * j][c] + (kx[2 * j + 1][c] - kx[2 * j][c]) * t;
      }
      acc += kdis[j];
      kl_out.line(LS((float)acc));
    }
  }
  log.line(" threads:" + LI(d.nthreads));
  log.line("");
  if (temp) {
    log.line(" temperature" + LD(d.temp));
    log.line("");
  }
  log.line(" grid:" + LI(d.ngrid[0]) + LI(d.ngrid[1]) + LI(d.ngrid[2]));
  log.line("");
  log.line(" ktol-coulomb:" + LD(d.ktol));
  log.line("");
  log.line(" kmesh shift:" + LD(d.mshift[0]) + LD(d.mshift[1]) + LD(d.mshift[2]));
  log.line("");
  log.line(" conduction bands, nc:" + LI(d.nc) + "   valence bands, nv:" + LI(d.nv));
  log.line("");
  log.line(" number of kpoints in the path:   " + LI(nq));
  log.line("");
  log.line("");
  log.line(stamp("begin"));
  log.line("");
  log.flush();
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  const long long N = (long long)nk * d.nc * d.nv;
  std::vector<double> kpt = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  gpu_check(ctx, wtbg_bands(ctx, nk, kpt.data(), d.nv, d.nc, nullptr, nullptr, nullptr, nullptr), "wtbg_bands");
  log.line(" quantum numbers for exciton basis set finished");
  log.flush();
  wtbg_coulomb p = coulomb_of(d);
  std::vector<double> exk((size_t)N * nq);
  // every Q in one batch call: the tridiagonalisation is a CUDA graph replayed per Q
  std::vector<double> kqs, q4s;
  kqs.reserve((size_t)nq * nk * 3);
  for (int iq = 0; iq < nq; ++iq) {
    const double q3[3] = {qp[iq][1], qp[iq][2], qp[iq][3]};
    std::vector<double> kq = kmesh(d.ngrid, d.mshift, m.rlat, q3);
    kqs.insert(kqs.end(), kq.begin(), kq.end());
    for (int c = 0; c < 4; ++c) q4s.push_back(qp[iq][c]);
  }
  gpu_check(ctx, wtbg_bse_q_batch(ctx, nk, nq, kqs.data(), q4s.data(), &p, 1, exk.data(), nullptr),
            "wtbg_bse_q_batch");
  for (int iq = 0; iq < nq; ++iq) log.line(" progress:" + LI(iq + 1) + " /" + LI(nq));
  log.flush();
  std::string buf;
  for (long long i2 = 0; i2 < N; ++i2) {
    for (int iq = 0; iq < nq; ++iq) buf += LS((float)qp[iq][0]) + LD(exk[i2 + (size_t)N * iq]) + "\n";
    buf += "\n";
  }
  fputs(buf.c_str(), f400.f);
  log.line("");
  log.line(stamp("end"));
  log.line("");
}

// ------------------------------------------------------------------------------ band and DOS tools
// orbital weights of ORB_W= (one value a line), 1.0 each when the file cannot be opened
std::vector<double> orbital_weights(const Deck& d, int w) {
  std::vector<double> ow(w, 1.0);
  std::ifstream f(d.orbw);
  if (!f) return ow;
  std::vector<std::string> toks;
  std::string l;
  while ((int)toks.size() < w && std::getline(f, l))
    for (auto& t : items_of(l)) toks.push_back(t);
  if ((int)toks.size() < w) throw Stop("Error reading orbital weight file");
  for (int i = 0; i < w; ++i) ow[i] = num(toks[i]);
  return ow;
}

// layercont (dos_subs.f90:154-181): sum |wf_i|^2 orbweight_i
double layercont(const double2v* wf, int w, const std::vector<double>& ow) {
  double re = 0.0;
  for (int i = 0; i < w; ++i) re += (wf[i].x * wf[i].x + wf[i].y * wf[i].y) * ow[i];
  return re;
}

// spin projection: the diagonal spin operator of spinvl (hamiltonian_tb.f90:281-368) and the
// up/down split of spincont (dos_subs.f90:37-100); +1 up, -1 down, 0 for NP
int spin_of(const std::string& systype, const std::string& dft, int i, int w) {
  const int w2 = w / 2;
  if (systype.rfind("NP", 0) == 0) return 0;
  if (systype.rfind("SP", 0) == 0 || (systype.rfind("SOC", 0) == 0 && dft == "V")) return i < w2 ? 1 : -1;
  return (i % 2 == 0) ? 1 : -1;
}

// bandstool (bands-kpath-tool.f90): eigsys along the k path of KPATH_FILE=; bands.dat with
// (k distance, E, <Sz>, layer weight) per band, KLABELS.dat from kpath2 (mhkpack_subs.f90:54-130)
// spoptics (sp_solver-tool-diel.f90): the single-particle half of bsesolver on its own (DIEL=T)
void spoptics_tool(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  Out f401(join_path(of, "sp_optics.dat"), "Error opening sp_optics output file");
  FILE* f402 = nullptr;
  FILE* f404 = nullptr;
  if (d.tmcoef) {
    f402 = fopen(join_path(of, "tm_coef.dat").c_str(), "w");
    if (!f402) throw Stop("Error opening tm_coef output file");
    f404 = fopen(join_path(of, "tm_coef-pol.dat").c_str(), "w");
    if (!f404) throw Stop("Error opening tm_coef-pol output file");
  }
  Out f403(join_path(of, "sp_optics-pol.dat"), "Error opening sp_optics-pol output file");
  upload_model(ctx, m);
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  const long long N = (long long)nk * d.nc * d.nv;
  std::vector<double> kpt = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  gpu_check(ctx, wtbg_bands(ctx, nk, kpt.data(), d.nv, d.nc, nullptr, nullptr, nullptr, nullptr), "wtbg_bands");
  gpu_check(ctx, wtbg_velocity(ctx, d.cshift, nullptr), "wtbg_velocity");
  std::vector<float> vr(15 * (size_t)N);
  gpu_check(ctx, wtbg_sp_table(ctx, vr.data()), "wtbg_sp_table");
  write_sp_tables(d, nk, N, vr, f401, f403, f402, f404);
  if (f402) fclose(f402);
  if (f404) fclose(f404);
}

// spoptpolbz (sp_opt_bz-tool.f90): bz_act_{x,y,z,sp,sm}.dat and dichroism.dat, list-directed rows
// (real(4) kx, ky, kz, value) on the Monkhorst-Pack mesh (OPT_BZ=T)
void spoptpolbz_tool(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  const char* names[6] = {"bz_act_x", "bz_act_y", "bz_act_z", "bz_act_sp", "bz_act_sm", "dichroism"};
  std::vector<std::unique_ptr<Out>> files;
  for (const char* n : names)
  {
    const std::string msg = std::string("Error opening ") + n + " output file";
    files.emplace_back(new Out(join_path(of, std::string(n) + ".dat"), msg.c_str()));
  }
  upload_model(ctx, m);
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  std::vector<double> kpt = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  std::vector<double> s((size_t)nk * 5);
  gpu_check(ctx, wtbg_sp_optbz(ctx, nk, kpt.data(), d.nv, d.nc, d.cshift, s.data()), "wtbg_sp_optbz");
  std::vector<std::string> buf(6);
  for (int k = 0; k < nk; ++k) {
    const std::string kk = LS((float)kpt[k]) + LS((float)kpt[k + (size_t)nk]) + LS((float)kpt[k + 2 * (size_t)nk]);
    double v[6];
    for (int c = 0; c < 5; ++c) v[c] = s[k + (size_t)nk * c];
    v[5] = (v[3] - v[4]) / (v[3] + v[4]);
    for (int c = 0; c < 6; ++c) buf[c] += kk + LD(v[c]) + "\n";
  }
  for (int c = 0; c < 6; ++c) fputs(buf[c].c_str(), files[c]->f);
}

// kpath2 (mhkpack_subs.f90:54-130) on the path of KPATH_FILE=: distances kp (nk) and
// Cartesian points kc (nk,3), KLABELS.dat written to the output folder
void kpath_points(const Deck& d, const Model& m, std::vector<double>& kp, std::vector<double>& kc) {
  const std::string of = d.outputfolder;
  std::ifstream kf(d.kpaths);
  if (!kf) throw Stop("Error opening kpath input file");
  std::vector<std::string> kl;
  {
    std::string l;
    while (std::getline(kf, l))
      if (!items_of(l).empty()) kl.push_back(l);
  }
  if (kl.size() < 2) throw Stop("bad kpath file");
  const int nks = (int)num(items_of(kl[0])[0]);
  const int npts = (int)num(items_of(kl[1])[0]);
  if ((int)kl.size() < 2 + nks) throw Stop("bad kpath file");
  std::vector<std::array<double, 3>> ks(nks);
  for (int i = 0; i < nks; ++i) {
    auto t = items_of(kl[2 + i]);
    for (int c = 0; c < 3; ++c) ks[i][c] = num(t[c]);
  }
  double b[3][3];
  recvec(m.rlat, b);
  std::vector<std::array<double, 3>> kx(nks);
  for (int i = 0; i < nks; ++i)
    for (int c = 0; c < 3; ++c) kx[i][c] = ks[i][0] * b[0][c] + ks[i][1] * b[1][c] + ks[i][2] * b[2][c];
  const int half = nks / 2;
  std::vector<double> kdis(half);
  double tot = 0.0;
  for (int i = 0; i < half; ++i) {
    const double dx = kx[2 * i + 1][0] - kx[2 * i][0], dy = kx[2 * i + 1][1] - kx[2 * i][1],
                 dz = kx[2 * i + 1][2] - kx[2 * i][2];
    kdis[i] = sqrt(dx * dx + dy * dy + dz * dz);
    tot += kdis[i];
  }
  for (auto& v : kdis) v = v / tot;
  const int nk = half * npts;
  kp.assign(nk, 0.0);
  kc.assign(3 * (size_t)nk, 0.0);
  Out kl_out(join_path(of, "KLABELS.dat"), "Error opening KLABELS output file");
  double acc = 0.0;
  kl_out.line(LS(0.0f));
  for (int j = 0; j < half; ++j) {
    for (int i = 0; i < npts; ++i) {
      const double t = (double)((float)i / (float)(npts - 1));
      const size_t r = (size_t)j * npts + i;
      kp[r] = acc + kdis[j] * t;
      for (int c = 0; c < 3; ++c) kc[r + (size_t)nk * c] = kx[2 * j][c] + (kx[2 * j + 1][c] - kx[2 * j][c]) * t;
    }
    acc += kdis[j];
    kl_out.line(LS((float)acc));
  }
}

void bandstool(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  if (!std::ifstream(d.kpaths)) throw Stop("Error opening kpath input file");
  Out f300(join_path(of, "bands.dat"), "Error opening bands output file");
  upload_model(ctx, m);
  const std::vector<double> ow = orbital_weights(d, m.w);
  std::vector<double> kp, kc;
  kpath_points(d, m, kp, kc);
  const int nk = (int)kp.size();
  const int w = m.w;
  std::vector<double> e((size_t)nk * w), vec((size_t)nk * w * w * 2);
  gpu_check(ctx, wtbg_eigsys(ctx, nk, kc.data(), e.data(), vec.data(), nullptr), "wtbg_eigsys");
  std::string buf;
  std::vector<double2v> wf(w);
  for (int n = 0; n < w; ++n) {
    buf += " #band" + LI(n + 1) + "\n";
    for (int k = 0; k < nk; ++k) {
      double sz = 0.0;
      for (int c = 0; c < w; ++c) {
        const size_t o = k + (size_t)nk * (n + (size_t)w * c);
        wf[c] = {vec[2 * o], vec[2 * o + 1]};
        sz += (wf[c].x * wf[c].x + wf[c].y * wf[c].y) * (double)spin_of(m.systype, d.dft, c, w);
      }
      if (m.systype.rfind("NP", 0) == 0) {
        sz = 0.0;
        for (int c = 0; c < w; ++c) sz += wf[c].x * wf[c].x + wf[c].y * wf[c].y;
      }
      buf += LS((float)kp[k]) + LS((float)e[k + (size_t)nk * n]) + LS((float)sz) + LS((float)layercont(wf.data(), w, ow)) +
             "\n";
    }
    buf += "\n";
  }
  fputs(buf.c_str(), f300.f);
}

// Berry curvature tools. berryct2 (berry_curvature_subs.f90:1-128) runs on the device
// (wtbg_berry) with the tools' constants gammas = 0.001 and the degeneracy cut 0.0001, both
// single-precision literals. berryct2 hands hlm a kz it never sets; the k-point's own kz is
// used here (every 2D model has R_z = 0, where kz drops out of the phases).
constexpr double kBerryGamma = (double)0.001f, kBerryDegTol = (double)0.0001f;

// berrycurv (berry_curvature_kpath-tool.f90): berry_curv_kpath.dat, rows (kp, yz, xz, xy)
void berrytool_kpath(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  if (!std::ifstream(d.kpaths)) throw Stop("Error opening kpath input file");
  Out f300(join_path(of, "berry_curv_kpath.dat"), "Error opening berry_curv_kpath output file");
  upload_model(ctx, m);
  std::vector<double> kp, kc;
  kpath_points(d, m, kp, kc);
  const int nk = (int)kp.size();
  std::vector<double> b((size_t)nk * 6);
  gpu_check(ctx, wtbg_berry(ctx, nk, kc.data(), kBerryGamma, kBerryDegTol, b.data()), "wtbg_berry");
  std::string buf = " kp yz xz xy\n";
  for (int k = 0; k < nk; ++k)
    buf += F(kp[k], 15, 4) + F(b[k + (size_t)nk * 4], 15, 4) + F(b[k + (size_t)nk * 2], 15, 4) +
           F(b[k + (size_t)nk * 1], 15, 4) + "\n";
  fputs(buf.c_str(), f300.f);
}

// berrycurvbz (berry_curvature_bz-tool.f90): berry_curv_bz.dat on the Monkhorst-Pack mesh,
// rows (real(4) kx, ky, kz, yz, xz, xy)
void berrytool_bz(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  Out f300(join_path(of, "berry_curv_bz.dat"), "Error opening berry_curv_bz output file");
  upload_model(ctx, m);
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  std::vector<double> kpt = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  std::vector<double> b((size_t)nk * 6);
  gpu_check(ctx, wtbg_berry(ctx, nk, kpt.data(), kBerryGamma, kBerryDegTol, b.data()), "wtbg_berry");
  std::string buf = " kx ky kz yz xz xy\n";
  for (int k = 0; k < nk; ++k) {
    for (int c = 0; c < 3; ++c) buf += F((double)(float)kpt[k + (size_t)nk * c], 15, 4);
    buf += F(b[k + (size_t)nk * 4], 15, 4) + F(b[k + (size_t)nk * 2], 15, 4) + F(b[k + (size_t)nk * 1], 15, 4) + "\n";
  }
  fputs(buf.c_str(), f300.f);
}

// dostool (tdos-tool.f90): eigsys on the k mesh, Gaussian smearing (endos) of the total,
// spin-resolved and orbital-weighted DOS on NEDOS points between min(0, E_min) and
// max(0, E_max); dos.dat (4F15.4) for NP, (6F15.4) otherwise, with the running trapezoid sum
void dostool(wtbg_ctx* ctx, const Deck& d, const Model& m) {
  const std::string of = d.outputfolder;
  Out f300(join_path(of, "dos.dat"), "Error opening dos output file");
  upload_model(ctx, m);
  const bool np = m.systype.rfind("NP", 0) == 0;
  const double spinf = np ? 2.0 : 1.0;
  f300.line(np ? " #energy tdos sumdos awdos" : " #energy tdos sumdos updos dndos awdos");
  const std::vector<double> ow = orbital_weights(d, m.w);
  std::vector<double> kc = kmesh(d.ngrid, d.mshift, m.rlat, nullptr);
  const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
  const int w = m.w;
  std::vector<double> e((size_t)nk * w), vec((size_t)nk * w * w * 2);
  gpu_check(ctx, wtbg_eigsys(ctx, nk, kc.data(), e.data(), vec.data(), nullptr), "wtbg_eigsys");
  const long long ndim = (long long)nk * w;
  std::vector<double> etb(ndim), wts((size_t)ndim * 4);
  double edos0 = 0.0, edosf = 0.0;
  std::vector<double2v> wf(w);
  long long cnt = 0;
  for (int k = 0; k < nk; ++k) {
    if (e[k] < edos0) edos0 = e[k];
    if (e[k + (size_t)nk * (w - 1)] > edosf) edosf = e[k + (size_t)nk * (w - 1)];
    for (int n = 0; n < w; ++n) {
      double cup = 0.0, cdn = 0.0;
      for (int c = 0; c < w; ++c) {
        const size_t o = k + (size_t)nk * (n + (size_t)w * c);
        wf[c] = {vec[2 * o], vec[2 * o + 1]};
        const int sp = spin_of(m.systype, d.dft, c, w);
        const double a2 = wf[c].x * wf[c].x + wf[c].y * wf[c].y;
        if (sp > 0) cup += a2;
        if (sp < 0) cdn += a2;
      }
      etb[cnt] = e[k + (size_t)nk * n];
      wts[cnt] = 1.0;
      wts[ndim + cnt] = cup;
      wts[2 * ndim + cnt] = cdn;
      wts[3 * ndim + cnt] = layercont(wf.data(), w, ow);
      ++cnt;
    }
  }
  const int nw = (int)d.numdos;
  std::vector<double> en(nw), out((size_t)nw * 4);
  const double deltaen = (edosf - edos0) / (d.numdos - 1.0);
  for (int i = 0; i < nw; ++i) en[i] = edos0 + ((edosf - edos0) * (double)i) / (d.numdos - 1.0);
  gpu_check(ctx, wtbg_dos(ctx, ndim, etb.data(), wts.data(), 4, nk, nw, en.data(), d.sme, out.data()), "wtbg_dos");
  std::string buf;
  double sumdos = 0.0;
  for (int i = 0; i < nw; ++i) {
    const double at = spinf * out[i], up = out[(size_t)nw + i], dn = out[2 * (size_t)nw + i], aw = spinf * out[3 * (size_t)nw + i];
    if (np)
      buf += F(en[i], 15, 4) + F(at, 15, 4) + F(sumdos, 15, 4) + F(aw, 15, 4) + "\n";
    else
      buf += F(en[i], 15, 4) + F(at, 15, 4) + F(sumdos, 15, 4) + F(up, 15, 4) + F(-dn, 15, 4) + F(aw, 15, 4) + "\n";
    if (i > 0) sumdos = sumdos + (deltaen * (spinf * out[i - 1] + at) * 0.5);
  }
  fputs(buf.c_str(), f300.f);
}

// ------------------------------------------------------------------------------ spectra
struct Table {
  std::vector<double> E;
  std::vector<double> Fv;   // (n, ncomp) column-major
  int n = 0, ncomp = 0;
};

// read_back of a (7F15.4)/(6F15.4) file written above (header line + n rows)
Table read_table(const std::string& path, int n, int ncol, const char* errmsg) {
  FILE* f = fopen(path.c_str(), "r");
  if (!f) throw Stop(errmsg);
  Table t;
  t.n = n;
  t.ncomp = ncol - 1;
  t.E.resize(n);
  t.Fv.resize((size_t)n * t.ncomp);
  char* line = nullptr;
  size_t cap = 0;
  if (getline(&line, &cap, f) < 0) throw Stop(std::string(errmsg) + " (empty)");
  for (int i = 0; i < n; ++i) {
    if (getline(&line, &cap, f) < 0) throw Stop(std::string(errmsg) + " (short)");
    char* p = line;
    for (int c = 0; c < ncol; ++c) {
      char* end = nullptr;
      const double v = strtod(p, &end);
      if (end == p) throw Stop(std::string(errmsg) + " (bad row)");
      p = end;
      if (c == 0) t.E[i] = v;
      else t.Fv[i + (size_t)n * (c - 1)] = v;
    }
  }
  free(line);
  fclose(f);
  return t;
}

struct Spec {
  std::vector<double> om;
  std::vector<float> eps;   // (nw, 2, ncomp)
  int nw = 0, ncomp = 0;
  float re(int j, int c) const { return eps[j + (size_t)nw * (0 + 2 * c)]; }
  float im(int j, int c) const { return eps[j + (size_t)nw * (1 + 2 * c)]; }
};

Spec run_spectrum(wtbg_ctx* ctx, const Deck& d, const Model& m, const Table& t, const std::vector<int>& rtype) {
  Spec s;
  s.nw = (int)d.numbse;
  s.ncomp = t.ncomp;
  s.om.resize(s.nw);
  s.eps.resize((size_t)s.nw * 2 * t.ncomp);
  std::string st = m.systype;
  while (!st.empty() && st.back() == ' ') st.pop_back();
  const double spinf = (st == "NP") ? 2.0 : 1.0;
  gpu_check(ctx, wtbg_spectrum(ctx, t.n, t.ncomp, t.E.data(), t.Fv.data(), rtype.data(), d.ngrid, vcell3d(m.rlat),
                               d.ebse0, d.ebsef, d.numbse, d.cshift, d.renorm, spinf, s.om.data(), s.eps.data()),
            "wtbg_spectrum");
  return s;
}

void write_diel(const std::string& path, const Spec& s, int c) {
  Out o(path, ("Error opening " + path).c_str());
  o.line(" #  energy  real  imag");
  std::string buf;
  for (int j = 0; j < s.nw; ++j) buf += LD(s.om[j]) + LS(s.re(j, c)) + LS(s.im(j, c)) + "\n";
  fputs(buf.c_str(), o.f);
}

// diel-pp-subs.f90:1-73
void optprops(double e1, double e2, double efoton, double out[5]) {
  const double aux = sqrt((e1 * e1) + (e2 * e2));
  const double refr = sqrt((aux + e1) / 2.0);
  const double ext = sqrt((aux - e1) / 2.0);
  const double a1 = (refr - 1.0) * (refr - 1.0), a2 = (refr + 1.0) * (refr + 1.0), a3 = ext * ext;
  const double refl = (a1 + a3) / (a2 + a3);
  const double hc = (double)19.746E-06f;
  const double absc = ((double)sqrtf(2.0f) * efoton) * (1.0 / hc) * sqrt(aux - e1);
  const double eloss = e2 / ((e1 * e1) + (e2 * e2));
  out[0] = refr;
  out[1] = ext;
  out[2] = refl;
  out[3] = absc;
  out[4] = eloss;
}

// bseoptprop / spoptprop (and -pol): reads the diel files back as written, then 5 files
void optprop_files(const std::string& of, const std::string& prefix, const std::vector<std::string>& dielnames,
                   const std::vector<int>& outorder, const std::string& suffix, int nw) {
  const int nc = (int)dielnames.size();
  std::vector<std::vector<double>> re(nc, std::vector<double>(nw)), im(nc, std::vector<double>(nw));
  std::vector<double> energy(nw);
  for (int c = 0; c < nc; ++c) {
    FILE* f = fopen((of + dielnames[c]).c_str(), "r");
    if (!f) throw Stop("Error opening " + dielnames[c] + " input file");
    char* line = nullptr;
    size_t cap = 0;
    if (getline(&line, &cap, f) < 0) throw Stop("empty " + dielnames[c]);
    for (int i = 0; i < nw; ++i) {
      if (getline(&line, &cap, f) < 0) throw Stop("short " + dielnames[c]);
      char* p = line;
      char* end;
      const double e = strtod(p, &end);
      p = end;
      re[c][i] = strtod(p, &end);
      p = end;
      im[c][i] = strtod(p, &end);
      if (c == 0) energy[i] = e;
    }
    free(line);
    fclose(f);
  }
  const char* names[5] = {"refractive_index", "extinction_coef", "reflectibility", "absorption_coef", "en_loss_func"};
  std::string header = " #  energy";
  for (int k : outorder) {
    std::string nm = dielnames[k];
    nm = nm.substr(nm.rfind('_') + 1);
    nm = nm.substr(0, nm.find('.'));
    header += "  " + nm;
  }
  for (int q = 0; q < 5; ++q) {
    Out o(of + prefix + names[q] + suffix + ".dat", "Error opening output file");
    o.line(header);
    std::string buf;
    for (int i = 0; i < nw; ++i) {
      buf += F(energy[i], 15, 4);
      for (int k : outorder) {
        double v[5];
        optprops(re[k][i], im[k][i], energy[i], v);
        buf += F(v[q], 15, 4);
      }
      buf += "\n";
    }
    fputs(buf.c_str(), o.f);
  }
}

// exclft (bse_subs.f90:472-530)
double exclft(const std::string& sysdim0, const int ng[3], const double r[3][3], double fosc, double enexc) {
  std::string s = sysdim0;
  while (!s.empty() && s.back() == ' ') s.pop_back();
  const double cfe = (double)7.297E-3f, lspd = (double)299.792E16f, hbar = (double)6.582E-16f;
  const double nkt = (double)(ng[0] * ng[1] * ng[2]);
  if (s == "3D") {
    const double aux1 = (4.0 * cfe) * (enexc * enexc * enexc);
    const double aux2 = fosc / nkt;
    const double aux3 = 3.0 * (lspd * lspd) * (hbar * hbar * hbar);
    return 1.0 / ((aux1 * aux2) / aux3);
  }
  if (s == "2D") {
    const double aux1 = nkt * vcell2d(r) * hbar;
    const double aux2 = (8.0 * kPi32 * cfe * enexc) * fosc;
    return aux1 / aux2;
  }
  if (s == "1D") {
    const double aux2 = (2.0 * kPi32 * cfe * enexc * enexc) * fosc;
    const double aux1 = nkt * r[0][0] * hbar * hbar * lspd;
    return aux1 / aux2;
  }
  throw Stop("Wrong System dimension");
}

void lifetime_file(const std::string& of, const Deck& d, const Model& m, const Table& t, bool pol) {
  Out o(of + (pol ? "exciton_lifetime-pol.dat" : "exciton_lifetime.dat"), "Error opening exciton_lifetime output file");
  o.line(pol ? " #energy(eV) sum-lft(s)  x-lft(s) y-lft(s) z-lft(s) sp-lft(s) sm-lft(s)"
             : " #energy(eV) sum-lft(s)  x-lft(s) y-lft(s) z-lft(s)");
  std::string buf;
  const int ncol = pol ? 5 : 3;
  for (int i = 0; i < t.n; ++i) {
    const double e = t.E[i];
    auto f = [&](int c) { return t.Fv[i + (size_t)t.n * c]; };
    buf += F(e, 15, 4) + E(exclft(d.sysdim, d.ngrid, m.rlat, f(0) + f(1) + f(2), e), 15, 4);
    for (int c = 0; c < ncol; ++c) buf += E(exclft(d.sysdim, d.ngrid, m.rlat, f(c), e), 15, 4);
    buf += "\n";
  }
  fputs(buf.c_str(), o.f);
}

}  // namespace

// ------------------------------------------------------------------------------ entry
extern "C" int wtb_run(const char* deck_text, int device, Timings* tm, char* errbuf, int errlen) {
  wtbg_ctx* ctx = nullptr;
  auto fail = [&](const std::string& m) {
    if (errbuf && errlen > 0) {
      snprintf(errbuf, (size_t)errlen, "%s", m.c_str());
    }
    if (ctx) wtbg_destroy(ctx);
    return 1;
  };
  try {
    const double t0 = now_s();
    if (tm) *tm = Timings{};
    Deck d = parse_deck(deck_text ? deck_text : "");
    // params header + mesh (wtb_main.f90:77-104)
    Model m;
    if (d.bse || d.bset || d.bsekpath || d.bsetbnd || d.spec || d.spdiel || d.bandscalc || d.doscalc || d.berryk ||
        d.berrybz || d.sppolbz)
      m = read_params(d.params);
    if (d.meshtype.rfind("RK3D", 0) == 0) rkmesh(d.rk, m.rlat, d.ngrid, false);
    else if (d.meshtype.rfind("RK2D", 0) == 0) rkmesh(d.rk, m.rlat, d.ngrid, true);
    Out log(d.calcparms + "log.dat", "Error opening log output file ");
    param_out(log, d);
    log.line("");
    log.line(stamp("Begin"));
    log.line("");
    log.flush();
    int st = wtbg_create(&ctx, device);
    if (st != 0) return fail(std::string("wtbg_create: ") + wtbg_error_string(st));
    RunState rs;
    if (!d.pponly) {
      if (d.bandscalc) {
        bandstool(ctx, d, m);
        log.line(" Band Structure finished");
        log.flush();
      }
      if (d.doscalc) {
        dostool(ctx, d, m);
        log.line(" DOS finished");
        log.flush();
      }
      // wtb_main.f90:154-202
      if (d.bse && d.bset) {
        log.line(" ERROR: Choose BSE=T or BSET=T not both");
        log.flush();
        throw Stop("ERROR: Choose BSE=T or BSET=T not both");
      } else if (d.bse) {
        rs = bsesolver(ctx, d, m, tm);
        log.line(" BSE and Single particle dielectric calculation finished");
        log.flush();
      } else if (d.bset) {
        rs = bsesolver(ctx, d, m, tm);
        log.line(" BSE and Single particle dielectric calculation, with temperature, finished");
        log.flush();
      }
      if (d.bsekpath && d.bsetbnd) {
        log.line(" ERROR: Choose BSE_BND=T or BSET_BND=T not both");
        log.flush();
        throw Stop("ERROR: Choose BSE_BND=T or BSET_BND=T not both");
      } else if (d.bsekpath) {
        bsebnds(ctx, d, m);
        log.line(" BSE exciton band structure finished");
        log.flush();
      } else if (d.bsetbnd) {
        bsebnds(ctx, d, m);
        log.line(" BSE exciton band structure, with temperature, finished");
        log.flush();
      }
      // wtb_main.f90:209-218
      if (d.spdiel) {
        spoptics_tool(ctx, d, m);
        log.line(" Single particle dielectric calculation finished");
        log.flush();
      }
      if (d.sppolbz) {
        spoptpolbz_tool(ctx, d, m);
        log.line(" Single particle optical activity in BZ finished");
        log.flush();
      }
      // wtb_main.f90:232-251
      if (d.berryk) {
        berrytool_kpath(ctx, d, m);
        log.line(" Berry curvature in kpath finished");
        log.flush();
      }
      if (d.berrybz) {
        berrytool_bz(ctx, d, m);
        log.line(" Berry curvature in BZ finished");
        log.flush();
      }
    }
    const double t1 = now_s();
    const int nk = d.ngrid[0] * d.ngrid[1] * d.ngrid[2];
    const int N = nk * d.nc * d.nv;
    const std::string of = d.outputfolder;
    const bool bsex = d.bse || d.bset;
    // the fast form's spectrum: Haydock recursion on the BSE matrix still on the device (all
    // eight components at once; the -pol files take x, y, z, sp, sm = 0, 1, 2, 6, 7)
    Spec sfast;
    if (d.spec && bsex && rs.fast) {
      sfast.nw = (int)d.numbse;
      sfast.ncomp = 8;
      sfast.om.resize(sfast.nw);
      sfast.eps.resize((size_t)sfast.nw * 2 * 8);
      std::string sty = m.systype;
      while (!sty.empty() && sty.back() == ' ') sty.pop_back();
      gpu_check(ctx, wtbg_bse_spectrum_fast(ctx, d.gpu_haydock, d.dtfull, d.cpol, rs.e1, rs.emax, d.ngrid,
                                            vcell3d(m.rlat), d.ebse0, d.ebsef, d.numbse, d.cshift, d.renorm,
                                            (sty == "NP") ? 2.0 : 1.0, sfast.om.data(), sfast.eps.data()),
                "wtbg_bse_spectrum_fast");
    }
    const long long nrow = rs.fast ? rs.rows : (long long)N;
    if (d.spec && bsex) {
      // bsedielraw / bseoptprop / lifetime (wtb_main.f90:257-300; no lifetime after BSET)
      Table t = read_table(of + "bse_opt_diel.dat", (int)nrow, 7, "Error opening bse_opt_diel input file");
      Spec s = rs.fast ? sfast : run_spectrum(ctx, d, m, t, {1, 1, 1, 0, 0, 0});
      const char* nm[6] = {"xx", "yy", "zz", "xy", "xz", "yz"};
      for (int c = 0; c < 6; ++c) write_diel(of + "bse_diel_" + nm[c] + ".dat", s, c);
      if (tm) tm->spectrum = now_s() - t1;
      optprop_files(of, "bse_", {"bse_diel_xx.dat", "bse_diel_yy.dat", "bse_diel_zz.dat", "bse_diel_xy.dat",
                                 "bse_diel_xz.dat", "bse_diel_yz.dat"}, {0, 1, 2, 3, 4, 5}, "", s.nw);
      if (!d.bset) lifetime_file(of, d, m, t, false);
      log.line(" BSE dielectric properties calculated");
      log.flush();
      if (d.cpol) {
        Table tp = read_table(of + "bse_opt_diel-pol.dat", (int)nrow, 6, "Error opening bse_opt_diel-pol input file");
        Spec sp = rs.fast ? sfast : run_spectrum(ctx, d, m, tp, {1, 1, 1, 1, 1});
        const char* pn[5] = {"x", "y", "z", "sp", "sm"};
        const int fast_col[5] = {0, 1, 2, 6, 7};
        for (int c = 0; c < 5; ++c) write_diel(of + "bse_diel-pol_" + pn[c] + ".dat", sp, rs.fast ? fast_col[c] : c);
        optprop_files(of, "bse_", {"bse_diel-pol_x.dat", "bse_diel-pol_y.dat", "bse_diel-pol_z.dat",
                                   "bse_diel-pol_sp.dat", "bse_diel-pol_sm.dat"}, {0, 1, 2, 3, 4}, "-pol", sp.nw);
        if (!d.bset) lifetime_file(of, d, m, tp, true);
        log.line(" BSE absorption spectrum with light polarization calculated");
        log.flush();
      }
    }
    if (d.spec && (d.spdiel || bsex)) {
      // spdielraw / spoptprop (wtb_main.f90:304-313)
      Table t = read_table(of + "sp_optics.dat", N, 7, "Error opening sp_optics input file");
      Spec s = run_spectrum(ctx, d, m, t, {1, 1, 1, 0, 0, 0});
      const char* nm[6] = {"xx", "yy", "zz", "xy", "xz", "yz"};
      for (int c = 0; c < 6; ++c) write_diel(of + "sp_diel_" + nm[c] + ".dat", s, c);
      optprop_files(of, "sp_", {"sp_diel_xx.dat", "sp_diel_yy.dat", "sp_diel_zz.dat", "sp_diel_xy.dat",
                                "sp_diel_xz.dat", "sp_diel_yz.dat"}, {0, 1, 2, 3, 4, 5}, "", s.nw);
      log.line(" Single particle dielectric properties calculated");
      log.flush();
    }
    if (d.spec && (d.cpol || bsex)) {
      // spdielrawpol / spoptproppol (wtb_main.f90:317-326)
      Table t = read_table(of + "sp_optics-pol.dat", N, 6, "Error opening sp_optics-pol input file");
      Spec s = run_spectrum(ctx, d, m, t, {1, 1, 1, 1, 1});
      const char* pn[5] = {"x", "y", "z", "sp", "sm"};
      for (int c = 0; c < 5; ++c) write_diel(of + "sp_diel-pol_" + pn[c] + ".dat", s, c);
      optprop_files(of, "sp_", {"sp_diel-pol_x.dat", "sp_diel-pol_y.dat", "sp_diel-pol_z.dat", "sp_diel-pol_sp.dat",
                                "sp_diel-pol_sm.dat"}, {0, 1, 2, 3, 4}, "-pol", s.nw);
      log.line(" Single particle absorption spectrum with light polarization calculated");
      log.flush();
    }
    log.line("");
    log.line(stamp("End"));
    log.line("");
    if (tm) tm->total = now_s() - t0;
    wtbg_destroy(ctx);
    ctx = nullptr;
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}
