// gpe_host: a C++ driver over the C ABI that runs the reference's time loop
// (anthonyyoud/gpe src/gpe.f90:15-314) from the reference's own input files
// and writes its output files, with the solver path on the GPU.
//
//   gpe_host [--dir D] [--parse-only]
//
// Inputs (in D, default "."):
//   run.in         namelists run_params / eqn_params / io_params / misc_params
//                  (src/parameters.f90:40-87, read as src/io.f90:78-114)
//   parameters.in  precision pr, nx, ny, nz, vl1 = line_param(...),
//                  vr1 = ring_param(...) (src/parameters.in:22-70)
//   ic.in          the active "init_cond = ..." product (src/ic.in), built on
//                  the device by gpe_set_ic
// Outputs: norm.dat, energy.dat, psi_time.dat, mass.dat, timestep.dat
// (Fortran e17.9 records, as src/io.f90:136-207, 304-381, 399-413 and
// src/solve.f90:234-241), proc0000/end_state.dat + save.dat
// (src/io.f90:831-882), proc0000/dens<p>.dat and p_saved.dat when save_3d
// (src/io.f90:480-520), spectrum/, idf/ and eta_time.dat when save_spectrum
// (src/io.f90:623-716), proc0000/filtered<p>.dat when save_filter
// (src/io.f90:524-620); <p> is itos(p), seven zero-padded digits.  Control files: RUNNING
// (delete to stop), SAVE (write a 3-D snapshot), ERROR (written on a fatal
// error, as src/error.f90:24-46).  Restart reads end_state0000.dat
// (src/ic.f90:117-191).
#include <sys/stat.h>
#include <unistd.h>

#include <cctype>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/gpe_cuda.h"

namespace {

std::string g_dir = ".";

std::string path(const std::string& f) { return g_dir + "/" + f; }
bool exists(const std::string& f) {
  struct stat st;
  return stat(path(f).c_str(), &st) == 0;
}

// emergency_stop (src/error.f90:24-46): message, ERROR file, RUNNING removed
[[noreturn]] void emergency_stop(const std::string& msg) {
  fprintf(stderr, "%s\n", msg.c_str());
  FILE* f = fopen(path("ERROR").c_str(), "w");
  if (f) {
    fprintf(f, "%s\n", msg.c_str());
    fclose(f);
  }
  unlink(path("RUNNING").c_str());
  exit(1);
}

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

// Fortran real literal: 1.0, 1e-6, 2.5d0, 0.5_pr
double fnum(std::string v, const std::string& what) {
  v = lower(trim(v));
  const size_t u = v.find('_');
  if (u != std::string::npos) v = v.substr(0, u);
  for (auto& c : v)
    if (c == 'd') c = 'e';
  char* end = nullptr;
  const double x = strtod(v.c_str(), &end);
  if (!end || *end != '\0' || v.empty()) emergency_stop("ERROR: bad number '" + v + "' for " + what);
  return x;
}

bool flogical(std::string v, const std::string& what) {
  v = lower(trim(v));
  if (v == ".true." || v == "t" || v == ".t.") return true;
  if (v == ".false." || v == "f" || v == ".f.") return false;
  emergency_stop("ERROR: bad logical '" + v + "' for " + what);
}

std::string fstring(std::string v) {
  v = trim(v);
  if (v.size() >= 2 && (v[0] == '\'' || v[0] == '"')) v = v.substr(1, v.size() - 2);
  return v;
}

// Namelist groups of run.in: name -> (key -> raw value)
using Group = std::map<std::string, std::string>;

std::map<std::string, Group> read_namelists(const std::string& file) {
  std::ifstream in(path(file));
  if (!in) emergency_stop("ERROR: cannot open " + file);
  std::map<std::string, Group> out;
  std::string line, cur;
  while (std::getline(in, line)) {
    // strip comments outside quotes
    bool q = false;
    for (size_t i = 0; i < line.size(); ++i) {
      if (line[i] == '\'' || line[i] == '"') q = !q;
      if (line[i] == '!' && !q) {
        line = line.substr(0, i);
        break;
      }
    }
    line = trim(line);
    if (line.empty()) continue;
    if (line[0] == '&') {
      cur = lower(trim(line.substr(1)));
      out[cur];
      continue;
    }
    if (line == "/") {
      cur.clear();
      continue;
    }
    if (cur.empty()) continue;
    // key = value pairs, comma separated
    std::string rest = line;
    while (!rest.empty()) {
      const size_t eq = rest.find('=');
      if (eq == std::string::npos) break;
      const std::string key = lower(trim(rest.substr(0, eq)));
      std::string tail = rest.substr(eq + 1);
      // value runs until a comma outside quotes followed by another key=
      bool qq = false;
      size_t cut = tail.size();
      for (size_t i = 0; i < tail.size(); ++i) {
        if (tail[i] == '\'' || tail[i] == '"') qq = !qq;
        if (tail[i] == ',' && !qq && tail.find('=', i) != std::string::npos) {
          cut = i;
          break;
        }
      }
      std::string val = trim(tail.substr(0, cut));
      if (!val.empty() && val.back() == '/') val = trim(val.substr(0, val.size() - 1));
      if (!val.empty() && val.back() == ',') val = trim(val.substr(0, val.size() - 1));
      out[cur][key] = val;
      rest = cut < tail.size() ? tail.substr(cut + 1) : "";
    }
    if (line.back() == '/') cur.clear();
  }
  return out;
}

struct RunIn {
  double tau = 0, end_time = 0, xr = 0, yr = 0, zr = 0;
  std::string scheme = "rk4";
  int eqn = 4, bcs = 2, order = 2;
  bool restart = false, saved_restart = false, multiply_ic_restart = false, renorm = false, imprint_vl = false,
       stop_imag = false, real_time = true;
  double Urhs = 0, diss_amp = 0, scal = 1, nv = 0, enerv = 0, g = 1, mu = 1, nn = 1, omx = 0, omy = 0, omz = 0;
  int save_rate = 10;
  double save_rate2 = 1e300, save_rate3 = 1e300, p_save = 1e300;
  bool save_3d = false, save_spectrum = false, save_filter = false;
  double filter_kc = 10.0;
};

RunIn parse_run_in() {
  auto nl = read_namelists("run.in");
  for (const char* gname : {"run_params", "eqn_params", "io_params", "misc_params"})
    if (!nl.count(gname))
      emergency_stop(std::string("ERROR: There was an error reading namelist ") + gname + " in run.in.");
  RunIn r;
  auto& rp = nl["run_params"];
  auto& ep = nl["eqn_params"];
  auto& io = nl["io_params"];
  auto num = [](Group& g, const char* k, double& v) {
    if (g.count(k)) v = fnum(g[k], k);
  };
  auto inum = [](Group& g, const char* k, int& v) {
    if (g.count(k)) v = (int)llround(fnum(g[k], k));
  };
  auto lg = [](Group& g, const char* k, bool& v) {
    if (g.count(k)) v = flogical(g[k], k);
  };
  num(rp, "tau", r.tau);
  num(rp, "end_time", r.end_time);
  num(rp, "xr", r.xr);
  num(rp, "yr", r.yr);
  num(rp, "zr", r.zr);
  if (rp.count("scheme")) r.scheme = lower(fstring(rp["scheme"]));
  inum(rp, "eqn_to_solve", r.eqn);
  inum(rp, "bcs", r.bcs);
  inum(rp, "order", r.order);
  lg(rp, "restart", r.restart);
  lg(rp, "saved_restart", r.saved_restart);
  lg(rp, "multiply_ic_restart", r.multiply_ic_restart);
  lg(rp, "renorm", r.renorm);
  lg(rp, "imprint_vl", r.imprint_vl);
  lg(rp, "stop_imag", r.stop_imag);
  lg(rp, "real_time", r.real_time);
  num(ep, "urhs", r.Urhs);
  num(ep, "diss_amp", r.diss_amp);
  num(ep, "scal", r.scal);
  num(ep, "nv", r.nv);
  num(ep, "enerv", r.enerv);
  num(ep, "g", r.g);
  num(ep, "mu", r.mu);
  num(ep, "nn", r.nn);
  num(ep, "omx", r.omx);
  num(ep, "omy", r.omy);
  num(ep, "omz", r.omz);
  inum(io, "save_rate", r.save_rate);
  num(io, "save_rate2", r.save_rate2);
  num(io, "save_rate3", r.save_rate3);
  num(io, "p_save", r.p_save);
  lg(io, "save_3d", r.save_3d);
  lg(io, "save_spectrum", r.save_spectrum);
  lg(io, "save_filter", r.save_filter);
  num(io, "filter_kc", r.filter_kc);
  // diagnostics of the reference loop this host does not write
  // (src/gpe.f90:98, 181-217, 237-239): a run that asks for one stops with
  // ERROR instead of silently producing fewer files
  const std::pair<const char*, const char*> unbuilt[] = {
      {"save_contour", "save_surface (src/io.f90:440-476)"},
      {"save_average", "average (src/io.f90:1470-1500)"},
      {"save_pdf", "save_velocity_pdf (src/io.f90:211-274)"},
      {"save_vcf", "save_vel_corr (src/io.f90:278-300)"},
      {"save_ll", "save_linelength (src/io.f90:1397-1429)"},
      {"save_zeros", "get_zeros/get_extra_zeros/get_re_im_zeros (src/io.f90:886-1393)"}};
  for (const auto& u : unbuilt) {
    bool on = false;
    lg(io, u.first, on);
    if (on) emergency_stop(std::string("ERROR: ") + u.first + " = .true. needs " + u.second + ", which this host does not write.");
  }
  auto& mp = nl["misc_params"];
  bool on = false;
  lg(mp, "diagnostic", on);
  if (on) emergency_stop("ERROR: diagnostic = .true. needs diag (src/io.f90:1433-1466), which this host does not write.");
  on = false;
  lg(mp, "pp_filtered_surface", on);
  if (on)
    emergency_stop("ERROR: pp_filtered_surface = .true. needs pp_save_filter (src/io.f90:1504-1554), which this host "
                   "does not run.");
  return r;
}

// ---------------------------------------------------------------------------
// parameters.in: only the uncommented declarations matter

std::vector<std::string> fortran_args(const std::string& s) {
  std::vector<std::string> a;
  std::string cur;
  bool q = false;
  for (char c : s) {
    if (c == '\'' || c == '"') q = !q;
    if (c == ',' && !q) {
      a.push_back(trim(cur));
      cur.clear();
    } else {
      cur += c;
    }
  }
  if (!trim(cur).empty()) a.push_back(trim(cur));
  return a;
}

struct ParamsIn {
  int pr = 8, nx = 0, ny = 0, nz = 0;
  gpe_line vl1{};
  gpe_ring vr1{};
  bool have_vl1 = false, have_vr1 = false;
};

ParamsIn parse_parameters_in() {
  std::ifstream in(path("parameters.in"));
  if (!in) emergency_stop("ERROR: cannot open parameters.in");
  std::string all, line;
  while (std::getline(in, line)) {
    const size_t c = line.find('!');
    if (c != std::string::npos) line = line.substr(0, c);
    line = trim(line);
    if (line.empty()) continue;
    if (!all.empty() && all.back() == '&') all.pop_back();
    else if (!all.empty()) all += '\n';
    all += line;
  }
  ParamsIn P;
  std::istringstream ss(all);
  while (std::getline(ss, line)) {
    const std::string l = lower(line);
    const size_t eq = l.find('=');
    if (eq == std::string::npos) continue;
    const std::string lhs = trim(l.substr(l.find("::") == std::string::npos ? 0 : l.find("::") + 2,
                                          eq - (l.find("::") == std::string::npos ? 0 : l.find("::") + 2)));
    const std::string rhs = trim(line.substr(eq + 1));
    if (lhs == "pr") {
      const size_t a = rhs.find('('), b = rhs.find(')');
      const auto args = fortran_args(rhs.substr(a + 1, b - a - 1));
      P.pr = (!args.empty() && (int)fnum(args[0], "pr") <= 6) ? 4 : 8;
    } else if (lhs == "nx") {
      P.nx = (int)fnum(rhs, "nx");
    } else if (lhs == "ny") {
      P.ny = (int)fnum(rhs, "ny");
    } else if (lhs == "nz") {
      P.nz = (int)fnum(rhs, "nz");
    } else if (lhs == "vl1" || lhs == "vr1") {
      const size_t a = rhs.find('('), b = rhs.rfind(')');
      const auto v = fortran_args(rhs.substr(a + 1, b - a - 1));
      if (lhs == "vl1" && v.size() == 9) {
        // line_param(x0, y0, z0, amp1, amp2, ll, sgn, dir, imprint_phase)
        P.vl1.x0 = fnum(v[0], "vl1");
        P.vl1.y0 = fnum(v[1], "vl1");
        P.vl1.z0 = fnum(v[2], "vl1");
        P.vl1.amp1 = fnum(v[3], "vl1");
        P.vl1.amp2 = fnum(v[4], "vl1");
        P.vl1.ll = fnum(v[5], "vl1");
        P.vl1.sgn = fnum(v[6], "vl1");
        P.vl1.dir = fstring(v[7]).empty() ? 'z' : (char)std::tolower(fstring(v[7])[0]);
        P.vl1.imprint_phase = flogical(v[8], "vl1") ? 1 : 0;
        P.have_vl1 = true;
      } else if (lhs == "vr1" && v.size() == 10) {
        // ring_param(plane, x0, y0, z0, r0, amp, mm, r1, kk, dir)
        const std::string pl = lower(fstring(v[0]));
        P.vr1.plane[0] = pl.size() > 0 ? pl[0] : 'x';
        P.vr1.plane[1] = pl.size() > 1 ? pl[1] : 'y';
        P.vr1.x0 = fnum(v[1], "vr1");
        P.vr1.y0 = fnum(v[2], "vr1");
        P.vr1.z0 = fnum(v[3], "vr1");
        P.vr1.r0 = fnum(v[4], "vr1");
        P.vr1.amp = fnum(v[5], "vr1");
        P.vr1.mm = (int)fnum(v[6], "vr1");
        P.vr1.r1 = fnum(v[7], "vr1");
        P.vr1.kk = (int)fnum(v[8], "vr1");
        P.vr1.dir = fnum(v[9], "vr1");
        P.have_vr1 = true;
      }
    }
  }
  if (P.nx < 6 || P.ny < 6 || P.nz < 6) emergency_stop("ERROR: parameters.in must set nx, ny, nz >= 6");
  return P;
}

// ic.in: the uncommented "init_cond = f1 * f2 ..." line
gpe_ic parse_ic_in(const ParamsIn& P) {
  std::ifstream in(path("ic.in"));
  if (!in) emergency_stop("ERROR: cannot open ic.in");
  std::string line, expr;
  while (std::getline(in, line)) {
    const size_t c = line.find('!');
    if (c != std::string::npos) line = line.substr(0, c);
    line = lower(trim(line));
    if (line.rfind("init_cond", 0) == 0 && line.find('=') != std::string::npos) expr = trim(line.substr(line.find('=') + 1));
  }
  if (expr.empty()) emergency_stop("ERROR: ic.in has no active init_cond line");
  gpe_ic ic;
  memset(&ic, 0, sizeof(ic));
  bool have_pulse = false;
  // factors are separated by '*' outside parentheses (an argument list
  // may hold numbers like 1.0e-1_pr but no products)
  std::vector<std::string> facs;
  {
    std::string cur;
    int depth = 0;
    for (char ch : expr) {
      if (ch == '(') ++depth;
      if (ch == ')') --depth;
      if (ch == '*' && depth == 0) {
        facs.push_back(trim(cur));
        cur.clear();
      } else {
        cur += ch;
      }
    }
    facs.push_back(trim(cur));
  }
  for (const std::string& f : facs) {
    if (ic.nfactors >= 4) emergency_stop("ERROR: ic.in product has more than four factors");
    int code;
    if (f.rfind("fermi", 0) == 0) code = GPE_IC_FERMI;
    else if (f.rfind("vortex_line", 0) == 0) code = GPE_IC_LINE;
    else if (f.rfind("vortex_ring", 0) == 0) code = GPE_IC_RING;
    else if (f.rfind("random_phase", 0) == 0) code = GPE_IC_RANDOM_PHASE;
    else if (f.rfind("vortex_pair", 0) == 0) code = GPE_IC_VORTEX_PAIR;
    else if (f.rfind("sphere2", 0) == 0) code = GPE_IC_SPHERE2;
    else if (f.rfind("sphere", 0) == 0) code = GPE_IC_SPHERE;
    else if (f.rfind("wall", 0) == 0) code = GPE_IC_WALL;
    else if (f.rfind("pade_pulse_ring", 0) == 0) {
      // pade_pulse_ring('pulse' | 'ring', x0, y0, z0, r0), src/ic.f90:518
      const size_t a = f.find('('), b = f.rfind(')');
      if (a == std::string::npos || b == std::string::npos || b < a)
        emergency_stop("ERROR: ic.in factor '" + f + "' has no argument list");
      const std::vector<std::string> args = fortran_args(f.substr(a + 1, b - a - 1));
      if (args.size() != 5) emergency_stop("ERROR: pade_pulse_ring takes (pulse_or_ring, x0, y0, z0, r0)");
      const std::string kind = lower(fstring(args[0]));
      if (kind == "pulse") code = GPE_IC_PADE_PULSE;
      else if (kind == "ring") code = GPE_IC_PADE_RING;
      else emergency_stop("ERROR: pade_pulse_ring: pulse_or_ring must be 'pulse' or 'ring'");
      const gpe_pulse pu{fnum(args[1], "pade_pulse_ring x0"), fnum(args[2], "pade_pulse_ring y0"),
                         fnum(args[3], "pade_pulse_ring z0"), fnum(args[4], "pade_pulse_ring r0")};
      if (have_pulse && (pu.x0 != ic.pulse.x0 || pu.y0 != ic.pulse.y0 || pu.z0 != ic.pulse.z0 || pu.r0 != ic.pulse.r0))
        emergency_stop("ERROR: ic.in: two pade_pulse_ring factors with different arguments are not supported");
      ic.pulse = pu;
      have_pulse = true;
    } else {
      emergency_stop("ERROR: ic.in factor '" + f + "' is not supported");
    }
    if (code == GPE_IC_LINE && !P.have_vl1) emergency_stop("ERROR: parameters.in has no vl1");
    if (code == GPE_IC_RING && !P.have_vr1) emergency_stop("ERROR: parameters.in has no vr1");
    ic.factor[ic.nfactors++] = code;
  }
  ic.line = P.vl1;
  ic.ring = P.vr1;
  ic.seed = 1234;
  ic.kc = 1.5;
  if (const char* s = getenv("GPE_RANDOM_PHASE_SEED")) ic.seed = strtoull(s, nullptr, 10);
  if (const char* s = getenv("GPE_RANDOM_PHASE_KC")) ic.kc = atof(s);
  return ic;
}

// ---------------------------------------------------------------------------
// Fortran formatted output: Ew.d (width w, d digits, 0.ddd...E+xx)

std::string fe(double v, int w = 17, int d = 9) {
  char m[64];
  std::string body;
  if (v == 0.0 || !std::isfinite(v)) {
    if (!std::isfinite(v)) snprintf(m, sizeof m, "%s", std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
    else {
      std::string z = "0.";
      z.append(d, '0');
      snprintf(m, sizeof m, "%sE+00", z.c_str());
    }
    body = m;
  } else {
    char e[64];
    snprintf(e, sizeof e, "%.*e", d - 1, std::fabs(v));  // d.ddd...e+XX
    const std::string s(e);
    const size_t ep = s.find('e');
    std::string digits = s.substr(0, 1) + s.substr(2, ep - 2);
    const int ex = atoi(s.c_str() + ep + 1) + 1;
    char tail[16];
    if (std::abs(ex) <= 99) snprintf(tail, sizeof tail, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
    else snprintf(tail, sizeof tail, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    body = std::string(v < 0 ? "-" : "") + "0." + digits + tail;
  }
  if ((int)body.size() < w) body = std::string(w - body.size(), ' ') + body;
  return body;
}

void append_line(const std::string& file, const std::string& text) {
  FILE* f = fopen(path(file).c_str(), "a");
  if (!f) emergency_stop("ERROR: cannot write " + file);
  fputs(text.c_str(), f);
  fputc('\n', f);
  fclose(f);
}

struct Ctx {
  RunIn r;
  ParamsIn P;
  gpe_params prm{};
  gpe_handle* h = nullptr;
  size_t esz = 16;
  double t = 0, im_t = 0;
  std::complex<double> dt;
  int64_t p = 0;
  std::vector<double> x, y, z;
  std::thread writer;  // background writer of the last snapshot (one at a time)
};

// The run's metadata at the moment a snapshot was taken.
struct Meta {
  int64_t p;
  double t, im_t;
  std::complex<double> dt;
};

void check(Ctx& c, int rc) {
  if (rc != GPE_OK) emergency_stop(std::string("ERROR: ") + gpe_last_error(c.h));
}

std::vector<char> state_bytes(Ctx& c) {
  const size_t n = (size_t)c.P.nx * c.P.ny * c.P.nz;
  std::vector<char> b(n * c.esz);
  check(c, gpe_get_state(c.h, b.data(), c.esz == 16 ? GPE_C128 : GPE_C64));
  return b;
}

void wr_int(FILE* f, int32_t v) { fwrite(&v, 4, 1, f); }
void wr_real(FILE* f, const Ctx& c, double v) {
  if (c.esz == 16) fwrite(&v, 8, 1, f);
  else {
    const float s = (float)v;
    fwrite(&s, 4, 1, f);
  }
}

// end_state (src/io.f90:831-882): stream file proc0000/end_state.dat
void write_end_state(const Ctx& c, const Meta& m, const void* data, size_t bytes) {
  mkdir(path("proc0000").c_str(), 0755);
  FILE* f = fopen(path("proc0000/end_state.dat").c_str(), "wb");
  if (!f) emergency_stop("ERROR: cannot write proc0000/end_state.dat");
  wr_int(f, c.P.nx);
  wr_int(f, c.P.ny);
  wr_int(f, c.P.nz);
  wr_int(f, (int32_t)m.p);
  wr_real(f, c, m.t);
  wr_real(f, c, m.im_t);
  wr_real(f, c, m.dt.real());
  wr_real(f, c, m.dt.imag());
  fwrite(data, 1, bytes, f);
  fclose(f);
  FILE* s = fopen(path("save.dat").c_str(), "w");
  if (s) {
    fprintf(s, " Periodically saved state\n t = %25.16E\n im_t = %25.16E\n dt = (%25.16E,%25.16E)\n", m.t, m.im_t,
            m.dt.real(), m.dt.imag());
    fprintf(s, " nx = %12d\n ny = %12d\n nz = %12d\n p = %12lld\n", c.P.nx, c.P.ny, c.P.nz, (long long)m.p);
    fclose(s);
  }
}

Meta meta(const Ctx& c) { return Meta{c.p, c.t, c.im_t, c.dt}; }

void join_writer(Ctx& c) {
  if (c.writer.joinable()) c.writer.join();
}

// Take a snapshot of the state now and hand it to a writer thread; the time
// loop continues while the device-to-host copy and the file write run.
template <class Write>
void write_async(Ctx& c, Write w) {
  join_writer(c);  // the snapshot buffer is reused
  check(c, gpe_snapshot_begin(c.h, c.esz == 16 ? GPE_C128 : GPE_C64));
  const Meta m = meta(c);
  c.writer = std::thread([&c, m, w]() {
    const void* data = nullptr;
    size_t bytes = 0;
    if (gpe_snapshot_wait(c.h, &data, &bytes) != GPE_OK) emergency_stop("ERROR: snapshot copy failed");
    w(m, data, bytes);
  });
}

void end_state(Ctx& c, bool final_) {
  if (!final_) {
    write_async(c, [&c](const Meta& m, const void* d, size_t n) { write_end_state(c, m, d, n); });
    return;
  }
  join_writer(c);
  const auto b = state_bytes(c);
  write_end_state(c, meta(c), b.data(), b.size());
  if (c.r.save_filter) {
    // the final filtered state (end_state flag 1 -> filtered_surface flag 1,
    // src/io.f90:870-873, 598-607): the input of a saved_restart
    mkdir(path("proc0000").c_str(), 0755);
    const std::string name = "proc0000/end_state_filtered.dat";
    std::vector<char> fb(b.size());
    check(c, gpe_filtered(c.h, 1.0, c.r.filter_kc, fb.data(), c.esz == 16 ? GPE_C128 : GPE_C64));
    FILE* f = fopen(path(name).c_str(), "wb");
    if (!f) emergency_stop("ERROR: cannot write " + name);
    for (int v : {c.P.nx, c.P.ny, c.P.nz, (int)c.p}) wr_int(f, v);
    wr_real(f, c, c.t);
    wr_real(f, c, c.im_t);
    wr_real(f, c, c.dt.real());
    wr_real(f, c, c.dt.imag());
    fwrite(fb.data(), 1, fb.size(), f);
    fclose(f);
  }
  unlink(path("RUNNING").c_str());
}

// proc0000/end_state_filtered.dat as state_restart reads it with
// saved_restart (src/ic.f90:144-157): four integers and two reals are
// skipped, then nx*ny*nz complex values are read.  The writer
// (filtered_surface, src/io.f90:598-607) puts the complex dt between t, im_t
// and the field, so the reference's reader takes dt as the first element and
// drops the field's last one; read the same way, for the same state.
std::vector<std::complex<double>> read_saved_filtered(const Ctx& c) {
  const std::string name = "proc0000/end_state_filtered.dat";
  FILE* f = fopen(path(name).c_str(), "rb");
  if (!f) emergency_stop("ERROR: saved_restart=.true. but " + name + " does not exist.");
  const size_t n = (size_t)c.P.nx * c.P.ny * c.P.nz;
  const size_t rs = c.esz / 2;  // bytes of one real
  std::vector<char> b(n * c.esz);
  bool ok = fseek(f, (long)(4 * 4 + 2 * rs), SEEK_SET) == 0 && fread(b.data(), 1, b.size(), f) == b.size();
  fclose(f);
  if (!ok) emergency_stop("ERROR: " + name + " is truncated");
  std::vector<std::complex<double>> v(n);
  for (size_t q = 0; q < n; ++q) {
    if (c.esz == 16) {
      double w[2];
      memcpy(w, b.data() + q * 16, 16);
      v[q] = {w[0], w[1]};
    } else {
      float w[2];
      memcpy(w, b.data() + q * 8, 8);
      v[q] = {w[0], w[1]};
    }
  }
  return v;
}

// state_restart (src/ic.f90:117-191) from end_state0000.dat
void state_restart(Ctx& c, const gpe_ic& ic) {
  FILE* f = fopen(path("end_state0000.dat").c_str(), "rb");
  if (!f) emergency_stop("ERROR: restart=.true. but end_state0000.dat does not exist.");
  int32_t n[4];
  double v[4];
  bool ok = fread(n, 4, 4, f) == 4;
  if (c.esz == 16) ok = ok && fread(v, 8, 4, f) == 4;
  else {
    float w[4];
    ok = ok && fread(w, 4, 4, f) == 4;
    for (int q = 0; q < 4; ++q) v[q] = w[q];
  }
  if (!ok || n[0] != c.P.nx || n[1] != c.P.ny || n[2] != c.P.nz)
    emergency_stop("ERROR: end_state0000.dat does not match the grid in parameters.in");
  std::vector<char> b((size_t)c.P.nx * c.P.ny * c.P.nz * c.esz);
  if (fread(b.data(), 1, b.size(), f) != b.size()) emergency_stop("ERROR: end_state0000.dat is truncated");
  fclose(f);
  c.p = n[3];
  c.t = v[0];
  c.im_t = v[1];
  std::complex<double> dtp(v[2], v[3]);
  if (c.r.real_time) {
    if (dtp.real() == 0.0) {
      dtp = std::complex<double>(-dtp.imag(), dtp.real());
      c.im_t = 0.0;
    }
  } else if (dtp.imag() == 0.0) {
    dtp = std::complex<double>(dtp.imag(), -dtp.real());
    c.t = 0.0;
  }
  if (c.r.scheme == "rk45") c.dt = dtp;
  else if (dtp != c.dt) c.p = (int64_t)((double)c.p * std::abs(dtp) / std::abs(c.dt));
  // state_restart = out_var1 * out_var2 * init_cond (src/ic.f90:164):
  // out_var2 = the saved filtered state (saved_restart) else 1, init_cond =
  // the ic.in product (multiply_ic_restart) else 1; products taken left to
  // right with the naive complex multiply, the last one on the device
  if (c.r.saved_restart) {
    const auto f2 = read_saved_filtered(c);
    for (size_t q = 0; q < f2.size(); ++q) {
      if (c.esz == 16) {
        double* a = (double*)(b.data() + q * 16);
        const double ar = a[0], ai = a[1];
        a[0] = ar * f2[q].real() - ai * f2[q].imag();
        a[1] = ar * f2[q].imag() + ai * f2[q].real();
      } else {
        float* a = (float*)(b.data() + q * 8);
        const float ar = a[0], ai = a[1], br = (float)f2[q].real(), bi = (float)f2[q].imag();
        a[0] = ar * br - ai * bi;
        a[1] = ar * bi + ai * br;
      }
    }
  }
  check(c, gpe_set_state(c.h, b.data(), c.esz == 16 ? GPE_C128 : GPE_C64));
  if (c.r.multiply_ic_restart) check(c, gpe_multiply_ic(c.h, &ic, 0));
}

// itos (src/io.f90:29-47): the last seven digits of n, zero-padded
std::string itos(int64_t n) {
  char d[8];
  for (int i = 6; i >= 0; --i) {
    d[i] = (char)('0' + (int)(n % 10));
    n /= 10;
  }
  d[7] = 0;
  return d;
}

// idl_surface (src/io.f90:480-520): proc0000/dens<itos(p)>.dat + p_saved.dat,
// written from a snapshot on the writer thread
void write_dens(const Ctx& c, const Meta& m, const void* data, size_t bytes) {
  mkdir(path("proc0000").c_str(), 0755);
  const std::string name = "proc0000/dens" + itos(m.p) + ".dat";
  FILE* f = fopen(path(name).c_str(), "wb");
  if (!f) emergency_stop("ERROR: cannot write " + name);
  wr_real(f, c, m.t + m.im_t);
  for (int v : {c.P.nx, c.P.ny, c.P.nz, 1, 1, 0, c.P.ny - 1, 0, c.P.nz - 1}) wr_int(f, v);
  fwrite(data, 1, bytes, f);
  for (double v : c.x) wr_real(f, c, v);
  for (double v : c.y) wr_real(f, c, v);
  for (double v : c.z) wr_real(f, c, v);
  fclose(f);
  char rec[32];
  snprintf(rec, sizeof rec, "%10lld", (long long)m.p);
  append_line("p_saved.dat", rec);
}

void idl_surface(Ctx& c) {
  write_async(c, [&c](const Meta& m, const void* d, size_t n) { write_dens(c, m, d, n); });
}

double fmodulo(double a, double b) { return a - std::floor(a / b) * b; }

std::string fi(long long v, int w) {
  char b[32];
  snprintf(b, sizeof b, "%*lld", w, v);
  return b;
}

// save_time (src/io.f90:136-184): psi, |psi|^2 and its phase at the centre
// site into psi_time.dat
void save_time(Ctx& c, double time) {
  double v[2];
  check(c, gpe_get_site(c.h, c.P.nx / 2, c.P.ny / 2, c.P.nz / 2, v));
  const double h = std::hypot(v[0], v[1]);
  const double phase = std::atan2(v[1] + 1.0e-6, v[0]);  // get_phase (src/variables.f90:379-391)
  append_line("psi_time.dat", fe(time) + fe(c.im_t) + fe(v[0]) + fe(v[1]) + fe(h * h) + fe(phase));
}

// condensed_particles (src/io.f90:304-395) with spectrum (io.f90:623-716)
// and filtered_surface(a, 0) (io.f90:524-620), all on the device
void condensed_particles(Ctx& c, double time) {
  const int nF = c.P.nx / 2;
  const bool spec = c.r.save_spectrum;
  gpe_condensed_info d;
  std::vector<double> eta(GPE_SPECTRUM_SHELLS), F(nF);
  std::vector<int32_t> nh(GPE_SPECTRUM_SHELLS);
  check(c, gpe_condensed(c.h, &d, spec ? eta.data() : nullptr, spec ? nh.data() : nullptr,
                         spec ? F.data() : nullptr, spec ? nF : 0));
  const double V = (double)c.P.nx * c.P.ny * c.P.nz;
  append_line("mass.dat", fe(time) + fe(c.im_t) + fe(d.mass_density) + fe(d.n0 / V) + fe(d.M) + fe(d.n0) +
                              fe(d.temp) + fe(d.temp2) + fe(d.H / V));
  if (spec) {
    mkdir(path("spectrum").c_str(), 0755);
    mkdir(path("idf").c_str(), 0755);
    std::string body;
    for (int m = 0; m < GPE_SPECTRUM_SHELLS; ++m) body += fi(m + 1, 9) + fi(nh[m], 9) + fe(eta[m]) + "\n";
    FILE* f = fopen(path("spectrum/spectrum" + itos(c.p) + ".dat").c_str(), "w");
    if (!f) emergency_stop("ERROR: cannot write spectrum/spectrum" + itos(c.p) + ".dat");
    fputs(body.c_str(), f);
    fclose(f);
    body.clear();
    for (int kk = 1; kk <= nF; ++kk) body += fi(kk, 9) + fe(F[kk - 1]) + "\n";
    f = fopen(path("idf/idf" + itos(c.p) + ".dat").c_str(), "w");
    if (!f) emergency_stop("ERROR: cannot write idf/idf" + itos(c.p) + ".dat");
    fputs(body.c_str(), f);
    fclose(f);
    append_line("eta_time.dat", fe(c.t) + fe(eta[0]) + fe(eta[1]) + fe(eta[2]));
  }
  if (c.r.save_filter) {
    mkdir(path("proc0000").c_str(), 0755);
    const std::string name = "proc0000/filtered" + itos(c.p) + ".dat";
    std::vector<char> b((size_t)c.P.nx * c.P.ny * c.P.nz * c.esz);
    check(c, gpe_filtered(c.h, 1.0, c.r.filter_kc, b.data(), c.esz == 16 ? GPE_C128 : GPE_C64));
    FILE* f = fopen(path(name).c_str(), "wb");
    if (!f) emergency_stop("ERROR: cannot write " + name);
    wr_real(f, c, c.t);
    for (int v : {c.P.nx, c.P.ny, c.P.nz, 1, 1, 0, c.P.ny - 1, 0, c.P.nz - 1}) wr_int(f, v);
    fwrite(b.data(), 1, b.size(), f);
    for (double v : c.x) wr_real(f, c, v);
    for (double v : c.y) wr_real(f, c, v);
    for (double v : c.z) wr_real(f, c, v);
    fclose(f);
  }
}

}  // namespace

int main(int argc, char** argv) {
  bool parse_only = false;
  for (int a = 1; a < argc; ++a) {
    if (!strcmp(argv[a], "--dir") && a + 1 < argc) g_dir = argv[++a];
    else if (!strcmp(argv[a], "--parse-only")) parse_only = true;
  }
  Ctx c;
  c.r = parse_run_in();
  c.P = parse_parameters_in();
  const gpe_ic ic = parse_ic_in(c.P);
  c.esz = c.P.pr == 8 ? 16 : 8;
  gpe_params& p = c.prm;
  p.nx = c.P.nx;
  p.ny = c.P.ny;
  p.nz = c.P.nz;
  const std::map<std::string, int> schemes = {{"euler", GPE_EULER}, {"rk2", GPE_RK2}, {"rk4", GPE_RK4},
                                              {"rk45", GPE_RK45}};
  if (!schemes.count(c.r.scheme)) emergency_stop("ERROR: Unrecognised time stepping scheme.");
  p.scheme = schemes.at(c.r.scheme);
  p.eqn = c.r.eqn;
  p.bcs = c.r.bcs;
  p.order = c.r.order;
  p.real_time = c.r.real_time ? 1 : 0;
  p.storage = c.P.pr == 8 ? GPE_C128 : GPE_C64;
  p.xr = c.r.xr;
  p.yr = c.r.yr;
  p.zr = c.r.zr;
  p.tau = c.r.tau;
  p.Urhs = c.r.Urhs;
  p.diss_amp = c.r.diss_amp;
  p.scal = c.r.scal;
  p.g = c.r.g;
  p.mu = c.r.mu;
  p.nn = c.r.nn;
  p.omx = c.r.omx;
  p.omy = c.r.omy;
  p.omz = c.r.omz;
  if (parse_only) {
    printf("{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"pr\": %d, \"scheme\": %d, \"eqn\": %d, \"bcs\": %d, "
           "\"order\": %d, \"real_time\": %d, \"tau\": %.17g, \"end_time\": %.17g, \"xr\": %.17g, \"g\": %.17g, "
           "\"mu\": %.17g, \"omz\": %.17g, \"save_rate\": %d, \"ic\": [%d, %d, %d, %d], \"nic\": %d, "
           "\"ring_r0\": %.17g, \"ring_plane\": \"%c%c\", \"line_x0\": %.17g, \"line_dir\": \"%c\", "
           "\"pulse\": [%.17g, %.17g, %.17g, %.17g]}\n",
           p.nx, p.ny, p.nz, c.P.pr, p.scheme, p.eqn, p.bcs, p.order, p.real_time, p.tau, c.r.end_time, p.xr, p.g,
           p.mu, p.omz, c.r.save_rate, ic.factor[0], ic.factor[1], ic.factor[2], ic.factor[3], ic.nfactors,
           ic.ring.r0, ic.ring.plane[0], ic.ring.plane[1], ic.line.x0, ic.line.dir, ic.pulse.x0, ic.pulse.y0,
           ic.pulse.z0, ic.pulse.r0);
    return 0;
  }
  if (c.r.imprint_vl && !c.P.have_vl1) emergency_stop("ERROR: imprint_vl=.true. but parameters.in has no vl1");
  FILE* run = fopen(path("RUNNING").c_str(), "w");
  if (run) fclose(run);
  if (gpe_create(&p, &c.h) != GPE_OK) emergency_stop(std::string("ERROR: ") + gpe_last_error(nullptr));
  c.dt = c.r.real_time ? std::complex<double>(c.r.tau, 0.0) : std::complex<double>(0.0, -c.r.tau);
  c.x.resize(p.nx);
  c.y.resize(p.ny);
  c.z.resize(p.nz);
  double dxyz[3];
  gpe_get_grid(c.h, c.x.data(), c.y.data(), c.z.data(), dxyz);
  if (c.r.restart) state_restart(c, ic);
  else {
    if (exists("end_state0000.dat")) emergency_stop("ERROR: restart=.false. but end_state0000.dat exists.");
    check(c, gpe_set_ic(c.h, &ic));
  }
  if (c.r.save_3d) idl_surface(c);
  double norm = 0, prev_norm = 1.0, relnorm = 0;
  if (c.r.eqn == 4 && !c.r.real_time) {
    check(c, gpe_norm(c.h, &prev_norm));
    if (c.r.renorm) check(c, gpe_renormalise(c.h, prev_norm));
    append_line("norm.dat", fe(c.t) + fe(c.im_t) + fe(prev_norm) + fe(relnorm));
  }
  condensed_particles(c, c.t);  // src/gpe.f90:116
  const double nsites = (double)p.nx * p.ny * p.nz;
  int64_t ps = (int64_t)(c.t / c.r.p_save), n2 = (int64_t)(c.t / c.r.save_rate2);
  int64_t m3 = (int64_t)(c.t / c.r.save_rate3);
  gpe_ic imprint{};
  imprint.nfactors = 1;
  imprint.factor[0] = GPE_IC_LINE;
  imprint.line = c.P.vl1;
  // Fixed-step real-time runs advance in chunks of up to kChunk steps per
  // gpe_step call (one replayed step graph per step, no host round trip in
  // between).  A chunk ends before any step at whose start the reference's
  // loop does something besides stepping (a save or diagnostic whose test
  // fires, the end of the loop), and at every step after which the norm is
  // needed (eqn 4: a norm record after it or after the next step, whose
  // relnorm needs this one).  The clock is advanced here exactly as the
  // library advances it (t += Re dt, im_t += |Im dt|), so the chunk ends are
  // the reference's event steps.  RUNNING and SAVE are polled once per chunk.
  const int64_t kChunk = 100;
  struct Clk {
    double t, im_t;
  };
  const auto advance = [&](Clk k) { return Clk{k.t + c.dt.real(), k.im_t + std::fabs(c.dt.imag())}; };
  const auto save_step = [&](Clk k) {  // modulo(t+im_t, |dt| save_rate) < |dt|
    const double adt = std::abs(c.dt);
    return fmodulo(k.t + k.im_t, adt * c.r.save_rate) < adt;
  };
  const auto pre_event = [&](Clk k) {  // anything at the top of the reference's loop besides stepping
    const double tt = k.t + k.im_t;
    return !(tt <= c.r.end_time) || save_step(k) || tt >= c.r.save_rate3 * m3 || tt >= c.r.save_rate2 * n2 ||
           tt >= c.r.p_save * ps;
  };
  const bool eq4 = c.r.eqn == 4;
  const auto chunk_len = [&]() -> int64_t {
    if (c.r.scheme == "rk45" || !c.r.real_time) return 1;
    Clk k{c.t, c.im_t};
    for (int64_t n = 1; n < kChunk; ++n) {
      const Clk k1 = advance(k), k2 = advance(k1);
      if (eq4 && (save_step(k1) || save_step(k2))) return n;  // the norm after step n-1 is needed
      if (pre_event(k1)) return n;
      k = k1;
    }
    return kChunk;
  };
  while (c.t + c.im_t <= c.r.end_time) {
    if (!exists("RUNNING")) {  // src/gpe.f90:137-161
      printf("\n Stop requested.\n");
      end_state(c, true);
      break;
    }
    const double adt = std::abs(c.dt);
    if (fmodulo(c.t + c.im_t, adt * c.r.save_rate) < adt) {  // src/gpe.f90:179-187
      double E = 0;
      check(c, gpe_energy(c.h, &E));
      append_line("energy.dat", fe(c.t) + fe(c.im_t) + fe(E / nsites));
      save_time(c, c.t);
    }
    if (c.t + c.im_t >= c.r.save_rate3 * m3) {  // src/gpe.f90:189-198
      condensed_particles(c, c.t);
      ++m3;
    }
    if (c.t + c.im_t >= c.r.save_rate2 * n2) {
      if (c.r.save_3d) idl_surface(c);
      ++n2;
    }
    if (c.t + c.im_t >= c.r.p_save * ps) {  // src/gpe.f90:223-227
      end_state(c, false);
      ++ps;
    }
    const int64_t nstep = chunk_len();
    gpe_step_info io;
    memset(&io, 0, sizeof(io));
    io.t = c.t;
    io.im_t = c.im_t;
    io.dt_re = c.dt.real();
    io.dt_im = c.dt.imag();
    io.p = c.p;
    // eqn 4 forms the norm of the new state (src/gpe.f90:243-249): every
    // step in imaginary time and with RKF45; in fixed-step real time only
    // where a record or the next record's relnorm uses it
    io.want_norm = eq4 ? 1 : 0;
    if (eq4 && c.r.real_time && c.r.scheme != "rk45") {
      // the norm of the chunk's last step is needed iff a norm record
      // follows it or the step after it
      Clk k{c.t, c.im_t};
      for (int64_t q = 0; q < nstep; ++q) k = advance(k);
      io.want_norm = (save_step(k) || save_step(advance(k))) ? 1 : 0;
    }
    check(c, gpe_step(c.h, nstep, &io));
    const double norm_before = io.norm;
    c.t = io.t;
    c.im_t = io.im_t;
    c.dt = std::complex<double>(io.dt_re, io.dt_im);
    c.p += nstep - 1;  // the last step's index; incremented at the end of the pass
    if (c.r.scheme == "rk45" && c.p % c.r.save_rate == 0)  // src/solve.f90:234-241
      append_line("timestep.dat", fe(c.t) + fe(c.im_t) + fe(std::abs(c.dt)) + [&] {
        char b[16];
        snprintf(b, sizeof b, "%10lld", (long long)c.p);
        return std::string(b);
      }());
    if (exists("SAVE")) {  // save_run (src/io.f90:1558-1587)
      idl_surface(c);
      unlink(path("SAVE").c_str());
    }
    if (eq4 && io.want_norm) {  // src/gpe.f90:243-249
      norm = norm_before;
      relnorm = std::fabs((norm - prev_norm) / prev_norm);
      if (fmodulo(c.t + c.im_t, std::abs(c.dt) * c.r.save_rate) < std::abs(c.dt))
        append_line("norm.dat", fe(c.t) + fe(c.im_t) + fe(norm) + fe(relnorm));
    }
    if (eq4 && !c.r.real_time) {  // src/gpe.f90:253-273
      if (relnorm < 1e-12) {
        if (c.r.stop_imag) break;  // End run if stop after imaginary time requested
        c.r.real_time = true;
        c.im_t = 0.0;
        ps = (int64_t)(c.t / c.r.p_save);
        n2 = (int64_t)(c.t / c.r.save_rate2);
        m3 = (int64_t)(c.t / c.r.save_rate3);
        if (c.r.save_3d) idl_surface(c);
        c.dt = std::complex<double>(std::fabs(c.dt.imag()), std::fabs(c.dt.real()));
        printf(" Switching to real time\n");
      }
      if (c.r.renorm) check(c, gpe_renormalise(c.h, norm));
      if (c.r.imprint_vl) check(c, gpe_multiply_ic(c.h, &imprint, 1));  // src/gpe.f90:272
    }
    if (eq4 && io.want_norm) prev_norm = norm;
    ++c.p;
  }
  end_state(c, true);
  if (c.r.save_3d) idl_surface(c);
  join_writer(c);
  gpe_destroy(c.h);
  printf(" DONE!\n");
  return 0;
}
