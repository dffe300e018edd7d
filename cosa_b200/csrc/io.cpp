// The reference's case files on the host: input.dat, mesh.dat, restart
// (include/cosa_io.h).  No device code: the readers fill host arrays in the
// library's layouts, which the caller uploads.
#include "../../include/cosa_io.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace {

// ---- gfortran unformatted sequential records ------------------------------------------
constexpr int64_t kMaxSub = 2147483639;  // largest subrecord gfortran writes

bool write_record(FILE *f, const void *data, int64_t bytes) {
  const char *p = static_cast<const char *>(data);
  int64_t left = bytes;
  bool first = true;
  do {
    const int64_t n = std::min(left, kMaxSub);
    const bool more = left > n;
    const int32_t head = more ? -(int32_t)n : (int32_t)n;
    const int32_t tail = first ? (int32_t)n : -(int32_t)n;
    if (fwrite(&head, 4, 1, f) != 1) return false;
    if (n && fwrite(p, 1, (size_t)n, f) != (size_t)n) return false;
    if (fwrite(&tail, 4, 1, f) != 1) return false;
    p += n;
    left -= n;
    first = false;
  } while (left > 0);
  return true;
}

// the next record into `out` (its whole length)
bool read_record(FILE *f, std::vector<char> &out) {
  out.clear();
  for (;;) {
    int32_t head = 0, tail = 0;
    if (fread(&head, 4, 1, f) != 1) return false;
    const int64_t n = head < 0 ? -(int64_t)head : head;
    const size_t at = out.size();
    out.resize(at + (size_t)n);
    if (n && fread(out.data() + at, 1, (size_t)n, f) != (size_t)n) return false;
    if (fread(&tail, 4, 1, f) != 1) return false;
    if ((tail < 0 ? -(int64_t)tail : tail) != n) return false;
    if (head >= 0) return true;
  }
}

struct Offs {
  std::vector<int64_t> p3, p2, p1;
};
Offs offsets(int nb, const int32_t *dims) {
  Offs o;
  int64_t a3 = 0, a2 = 0, a1 = 0;
  for (int b = 0; b < nb; ++b) {
    const int64_t im = dims[3 * b], jm = dims[3 * b + 1], km = dims[3 * b + 2];
    o.p3.push_back(a3); o.p2.push_back(a2); o.p1.push_back(a1);
    a3 += (im + 3) * (jm + 3) * (km + 3);
    a2 += (im + 2) * (jm + 2) * (km + 2);
    a1 += (im + 1) * (jm + 1) * (km + 1);
  }
  return o;
}

bool dims_ok(int nb, const int32_t *dims) {
  if (nb < 1 || !dims) return false;
  for (int i = 0; i < 3 * nb; ++i)
    if (dims[i] < 2) return false;
  return true;
}

// ---- input.dat: the token rules of linarg and list-directed reads ------------------------
std::string lower_d(std::string s) {
  // Fortran D exponents (1.d-3) for strtod
  for (char &c : s)
    if (c == 'd' || c == 'D') c = 'e';
  return s;
}

struct Lines {
  std::vector<std::string> v;
  size_t at = 0;
  bool ok = true;
  std::string next() {
    if (at >= v.size()) { ok = false; return std::string(); }
    return v[at++];
  }
  void skip() { next(); }
  // linarg: the n-th blank-separated word of a line (empty if absent)
  static std::string word(const std::string &line, int n) {
    std::istringstream is(line);
    std::string w;
    for (int i = 0; i < n; ++i)
      if (!(is >> w)) return std::string();
    return w;
  }
  // list-directed read of n values from the next record(s): blanks and
  // commas separate values; a record too short continues on the next
  std::vector<std::string> list(int n) {
    std::vector<std::string> out;
    while ((int)out.size() < n) {
      if (at >= v.size()) { ok = false; break; }
      std::string l = v[at++];
      for (char &c : l)
        if (c == ',') c = ' ';
      std::istringstream is(l);
      std::string w;
      while ((int)out.size() < n && (is >> w)) out.push_back(w);
    }
    return out;
  }
};

bool num(const std::string &s, double &v) {
  if (s.empty()) return false;
  const std::string t = lower_d(s);
  char *end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end && *end == 0;
}
bool inum(const std::string &s, int32_t &v) {
  double d;
  if (!num(s, d) || d != std::floor(d)) return false;
  v = (int32_t)d;
  return true;
}
int yn(const std::string &s, int &v) {
  if (s == "y") { v = 1; return 0; }
  if (s == "n") { v = 0; return 0; }
  return COSA_ERR_ARG;
}

inline int cyc(int idir, int m) {
  static const int t[3][3] = {{1, 2, 3}, {2, 3, 1}, {3, 1, 2}};
  return t[idir - 1][m - 1];
}

// mathb (src/input.f90:5206-5284): D = E^-1 A E on t_n = n 2 pi / (omega S)
void mathb(cosa_params &p) {
  const int nh = p.nharms, S = 2 * nh + 1;
  const double pi = 3.14159265358979323846;
  const double dt = 2 * pi / p.omega / S;
  std::vector<double> zeit(S), ahb(S * S, 0.0), eihb(S * S, 0.0), ehb(S * S, 0.0), t(S * S, 0.0);
  for (int n = 0; n < S; ++n) zeit[n] = n * dt;
  auto A = [&](std::vector<double> &m, int i, int j) -> double & { return m[i * S + j]; };
  for (int i = 1; i <= nh; ++i) {
    A(ahb, 2 * (i - 1) + 1, 2 * (i - 1) + 2) = i;
    A(ahb, 2 * (i - 1) + 2, 2 * (i - 1) + 1) = -i;
  }
  for (int i = 0; i < S; ++i) A(eihb, i, 0) = 1.0;
  for (int j = 1; j <= nh; ++j)
    for (int i = 0; i < S; ++i) {
      A(eihb, i, 2 * (j - 1) + 1) = std::cos(j * p.omega * zeit[i]);
      A(eihb, i, 2 * (j - 1) + 2) = std::sin(j * p.omega * zeit[i]);
    }
  const double fact = 2.0 / S;
  for (int j = 0; j < S; ++j) A(ehb, 0, j) = fact / 2;
  for (int i = 1; i <= nh; ++i)
    for (int j = 0; j < S; ++j) {
      A(ehb, 2 * (i - 1) + 1, j) = fact * std::cos(i * p.omega * zeit[j]);
      A(ehb, 2 * (i - 1) + 2, j) = fact * std::sin(i * p.omega * zeit[j]);
    }
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j) {
      double acc = 0;
      for (int k = 0; k < S; ++k) acc = acc + A(ahb, i, k) * A(ehb, k, j);
      A(t, i, j) = acc;
    }
  for (int i = 0; i < S; ++i)
    for (int j = 0; j < S; ++j) {
      double acc = 0;
      for (int k = 0; k < S; ++k) acc = acc + A(eihb, i, k) * A(t, k, j);
      p.dhb[i * S + j] = acc;
    }
}

// ---- Fortran formatted output of the history and force files -------------------
// A small interpreter of the edit descriptors these files use: Iw, nX, Ew.d,
// Dw.d and '/', with groups expanded beforehand.  Format control ends at the
// first data descriptor left without an item (the record being built is still
// written, as a WRITE statement does); blanks from X editing appear only when
// a field follows them in the same record.
struct FItem {
  char k;     // 'I', 'X', 'E', 'D', '/'
  int w, d;
};

// Ew.d / Dw.d editing of v: [-]0.<d digits>E+ee in w columns, right-justified
// (exponents beyond 99 drop the letter, as Fortran's Ew.d does), asterisks
// when the field is too narrow
std::string fortran_e(double v, int w, int d, char letter) {
  std::string out;
  if (!std::isfinite(v)) {
    out = std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity");
  } else {
    char tmp[64];
    std::snprintf(tmp, sizeof(tmp), "%.*e", d - 1, v);  // d significant digits, d.ddd e+XX
    std::string t(tmp);
    const bool neg = t[0] == '-';
    if (neg) t.erase(0, 1);
    const size_t ep = t.find('e');
    std::string mant = t.substr(0, ep), digits;
    for (char ch : mant)
      if (ch != '.') digits += ch;
    int ex = std::atoi(t.c_str() + ep + 1);
    if (v != 0.0) ex += 1;  // 0.ddd form
    else ex = 0;
    char eb[16];
    if (std::abs(ex) <= 99) std::snprintf(eb, sizeof(eb), "%c%c%02d", letter, ex < 0 ? '-' : '+', std::abs(ex));
    else std::snprintf(eb, sizeof(eb), "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
    out = std::string(neg ? "-" : "") + "0." + digits + eb;
  }
  if ((int)out.size() > w) return std::string((size_t)w, '*');
  return std::string((size_t)(w - (int)out.size()), ' ') + out;
}

std::string fortran_i(long long v, int w) {
  std::string t = std::to_string(v);
  if ((int)t.size() > w) return std::string((size_t)w, '*');
  return std::string((size_t)(w - (int)t.size()), ' ') + t;
}

// one WRITE of the integer and real items through the expanded format
std::string fortran_write(const std::vector<FItem> &fmt, const std::vector<long long> &ints,
                          const std::vector<double> &reals) {
  std::string out, rec;
  int pend = 0;
  size_t ii = 0, ri = 0;
  for (const FItem &f : fmt) {
    if (f.k == '/') { out += rec + "\n"; rec.clear(); pend = 0; continue; }
    if (f.k == 'X') { pend += f.w; continue; }
    if (f.k == 'I') {
      if (ii >= ints.size()) break;
      rec += std::string((size_t)pend, ' ') + fortran_i(ints[ii++], f.w);
    } else {
      if (ri >= reals.size()) break;
      rec += std::string((size_t)pend, ' ') + fortran_e(reals[ri++], f.w, f.d, f.k);
    }
    pend = 0;
  }
  return out + rec + "\n";
}

void push_n(std::vector<FItem> &v, int n, FItem a, FItem b) {
  for (int i = 0; i < n; ++i) { v.push_back(a); v.push_back(b); }
}

// (i8,1x,[(1x,d12.5)],4(/12(1x,d12.5)),[/(1x,d12.5)]) and the itime form
// 2(i8,1x) of formats 212-220 (src/output.f90:4376-4380)
std::vector<FItem> force_format(bool two_ints, bool time, bool alpha) {
  std::vector<FItem> f;
  f.push_back({'I', 8, 0}); f.push_back({'X', 1, 0});
  if (two_ints) { f.push_back({'I', 8, 0}); f.push_back({'X', 1, 0}); }
  if (time) push_n(f, 1, {'X', 1, 0}, {'D', 12, 5});
  for (int g = 0; g < 4; ++g) {
    f.push_back({'/', 0, 0});
    push_n(f, 12, {'X', 1, 0}, {'D', 12, 5});
  }
  if (alpha) { f.push_back({'/', 0, 0}); push_n(f, 1, {'X', 1, 0}, {'D', 12, 5}); }
  return f;
}

int copy_out(const std::string &t, char *buf, int64_t cap) {
  if (!buf || cap < (int64_t)t.size() + 1) return COSA_ERR_ARG;
  std::memcpy(buf, t.c_str(), t.size() + 1);
  return COSA_OK;
}

// variable names of one surface block of the force files
std::string force_names(int isurf, int nsurface) {
  static const char *base[6] = {"Cl", "Cd", "Cz", "Cmx", "Cmy", "Cm"};
  std::string s;
  for (int c = 0; c < 6; ++c)
    for (int pv = 0; pv < 2; ++pv) {
      std::string nm = std::string(base[c]) + (nsurface > 1 ? std::to_string(isurf) : "") + (pv ? "_v" : "_p");
      s += ",\"" + nm + "\"";
    }
  return s;
}

}  // namespace

struct cosa_input {
  std::vector<int32_t> dims, nbcs, bct, cut;
  int32_t nblocks = 0, ncuts = 0;
};

extern "C" {

int cosa_io_default_params(cosa_params *p) {
  if (!p) return COSA_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->gamma = 1.4; p->pranl = 0.72; p->prant = 0.9; p->stemp = 110.4 / 288.15;
  p->rhoinf = 1.0; p->ainf = 1.0; p->tinf = 1.0; p->pinf = 1.0 / p->gamma;
  p->rkap = 1.0 / 3.0; p->epslimf = 1.0e-6; p->epslimt = 1.0e-6; p->ilimf = 1; p->ilimt = 1;
  p->nl_crs = 99;
  p->cfl = 2.0; p->cflt = 2.0; p->cdff = 1.0; p->rat = 1.0; p->ratt = 1.0;
  p->iupdt = 1; p->nstage = 4;
  const double ar4[5] = {0.25, 0.333333, 0.5, 1.0, 0.0};
  for (int i = 0; i < 5; ++i) p->alphas[i] = ar4[i];
  p->npde = 5; p->lmet = 4; p->nlevel = 1; p->aircraft = 1;
  const double qmin[7] = {1.0e-8, 1.0, 1.0, 1.0, 1.0e-8, 1.0e-12, 1.0e-8};
  for (int i = 0; i < 7; ++i) p->qmin[i] = qmin[i];
  p->epst = 1.0e-12; p->kappa = 0.41; p->cmu = 1.0; p->sigk = 0.5; p->sigw = 0.5;
  p->bkw = 3.0 / 40.0; p->bstrkw = 0.09;
  p->gkw = p->bkw / p->bstrkw - p->sigw * p->kappa * p->kappa / std::sqrt(p->bstrkw);
  p->inlet_t0 = 1.008; p->inlet_p0 = 0.734486515085076; p->inlet_dir[0] = 1.0;
  for (int i = 0; i < 3; ++i) p->outlet_p[i] = 0.714285714285714;
  p->precision = COSA_PREC_FP64;
  p->nstart = p->npre = p->npost = p->ncrs = 1;
  p->bln_prol = 1;
  p->bdf1 = 1;
  p->cutoff_type = 1;
  return COSA_OK;
}

// input() (src/input.f90:2540-4392), line by line in its order
int cosa_io_read_input(const char *path, cosa_params *pp, cosa_run_opts *rr, cosa_input **out) {
  if (!path || !pp || !rr || !out) return COSA_ERR_ARG;
  *out = nullptr;
  std::ifstream fs(path);
  if (!fs) return COSA_ERR_ARG;
  Lines L;
  for (std::string l; std::getline(fs, l);) {
    if (!l.empty() && l.back() == '\r') l.pop_back();
    L.v.push_back(l);
  }
  cosa_params p;
  cosa_io_default_params(&p);
  p.aircraft = 0;
  cosa_run_opts r;
  std::memset(&r, 0, sizeof(r));
  double vcfl3 = 0, vcfli3 = 0, vcflt3 = 0, vcflit3 = 0, mutfar = 0;
  int e = 0;
  auto W = Lines::word;
  std::string line;

  L.skip();
  line = L.next();
  if (W(line, 1) == "cgns") return COSA_ERR_UNSUPPORTED;
  line = L.next();
  if ((e = yn(W(line, 1), r.debug))) return e;
  const std::string eqs = W(line, 2);
  if (eqs == "euler") { p.npde = 5; }
  else if (eqs == "laminar") { p.npde = 5; p.viscous = 1; }
  else if (eqs == "komega") { p.npde = 7; p.viscous = 1; p.kom = 1; }
  else if (eqs == "bsl") { p.npde = 7; p.viscous = 1; p.kom_bsl = 1; }
  else if (eqs == "sst") { p.npde = 7; p.viscous = 1; p.kom_sst = 1; }
  else return COSA_ERR_ARG;
  const std::string ext = W(line, 3);
  if (ext == "external") r.exter = 1;
  else if (ext == "internal") r.exter = 0;
  else return COSA_ERR_ARG;
  const std::string kind = W(line, 4);
  std::snprintf(r.flow_kind, sizeof(r.flow_kind), "%s", kind.c_str());
  if (kind == "aircraft") p.aircraft = 1;
  else if (kind == "saircraft" || kind == "vawt" || kind == "rhawt" || kind == "shawt") return COSA_ERR_UNSUPPORTED;
  else return COSA_ERR_ARG;

  // flow
  L.skip();
  line = L.next();
  double alpha = 0, beta = 0;
  if (!num(W(line, 1), p.gamma)) return COSA_ERR_ARG;
  if (p.viscous) {
    if (!num(W(line, 2), p.reyno) || !num(W(line, 3), p.pranl) || !num(W(line, 4), p.machfs)) return COSA_ERR_ARG;
    if (r.exter && (!num(W(line, 5), alpha) || !num(W(line, 6), beta))) return COSA_ERR_ARG;
  } else if (r.exter) {
    if (!num(W(line, 2), p.machfs) || !num(W(line, 3), alpha) || !num(W(line, 4), beta)) return COSA_ERR_ARG;
  }
  const double pi = 3.14159265358979323846;
  p.alpha = alpha / 180 * pi;
  p.beta = beta / 180 * pi;
  p.pinf = 1.0 / p.gamma;

  const bool turb = p.kom || p.kom_bsl || p.kom_sst;
  if (turb) {
    L.skip();
    line = L.next();
    if (!num(W(line, 1), p.prant) || !num(W(line, 2), p.tkefar) || !num(W(line, 3), mutfar)) return COSA_ERR_ARG;
    const std::string wall = W(line, 4);
    if (wall == "wilcox") {
      p.wallwilc = 1;
      if (!num(W(line, 5), p.roughk)) return COSA_ERR_ARG;
    } else if (wall == "menter") {
      p.wallwilc = 0;
    }
    p.tkefar = p.tkefar * p.machfs * p.machfs;
    p.omefar = p.cmu * p.rhoinf * p.tkefar / mutfar * p.reyno / p.machfs;
    p.mutfar = mutfar;
    L.skip();
    line = L.next();
    int v;
    if ((e = yn(W(line, 1), v))) return e;
    p.turcmp = v;
    if ((e = yn(W(line, 2), p.lim_prodtke))) return e;
    if (!num(W(line, 3), p.prdlim)) return COSA_ERR_ARG;
    if ((e = yn(W(line, 4), p.lim_prodomega))) return e;
    if (p.lim_prodomega && !p.lim_prodtke) return COSA_ERR_ARG;
    const std::string fx = W(line, 5);
    if (fx == "none") p.ifixq = 0;
    else if (fx == "minimum") p.ifixq = 1;
    else return COSA_ERR_ARG;
    const std::string fo = W(line, 6);
    if (fo == "second") p.foturb = 0;
    else if (fo == "first") p.foturb = 1;
    else return COSA_ERR_ARG;
  }

  // steady / unsteady
  L.skip();
  line = L.next();
  bool unsteady = false;
  const std::string st = W(line, 1);
  if (st == "unsteady") {
    unsteady = true;
    const std::string how = W(line, 2);
    if (how == "rgkun") {
      p.rgkuns = 1;
      if (!num(W(line, 3), r.dt)) return COSA_ERR_ARG;
    } else if (how == "dual") {
      p.dualt = 1;
      if (!num(W(line, 3), r.dt) || !inum(W(line, 4), r.ntime) || !inum(W(line, 5), r.nsave)) return COSA_ERR_ARG;
      if (W(line, 6) != "second") return COSA_ERR_UNSUPPORTED;
      const std::string rk = W(line, 7);
      if (rk == "rkex") p.rkimp = 0;
      else if (rk == "rkim") p.rkimp = 1;
      else return COSA_ERR_ARG;
    } else if (how == "hb") {
      p.harbal = 1;
      const std::string rk = W(line, 3);
      if (rk == "rkex") p.rkimp = 0;
      else if (rk == "rkim") p.rkimp = 1;
      else return COSA_ERR_ARG;
      if (!inum(W(line, 4), p.nharms) || p.nharms < 0 || 2 * p.nharms + 1 > COSA_MAX_SNAP) return COSA_ERR_ARG;
    } else {
      return COSA_ERR_ARG;
    }
  } else if (st != "steady") {
    return COSA_ERR_ARG;
  }
  if (unsteady) {
    L.skip();
    line = L.next();
    const std::string mv = W(line, 1);
    if (mv == "pitch") {
      p.moving = 1;
      double f = 0, dth = 0;
      if (!num(W(line, 2), f) || !num(W(line, 3), p.xh) || !num(W(line, 4), p.yh) || !num(W(line, 5), dth))
        return COSA_ERR_ARG;
      p.omegas = 2 * pi * f;
      p.dtheta0 = dth / 180.0 * pi;
    } else if (mv == "fixed") {
      if (p.harbal) return COSA_ERR_ARG;
    } else {
      return COSA_ERR_UNSUPPORTED;  // plunge, plupit, rotating
    }
  }
  if (p.harbal) {
    if (p.nharms > 0) {
      p.omega = std::fabs(p.omegas);
      if (p.omega <= 0) return COSA_ERR_ARG;
      r.dt = 2 * pi / p.omega / (2 * p.nharms + 1);
      mathb(p);
      if (p.moving) p.hbmove = 1;  // one grid per snapshot
    } else {
      p.moving = 0;
    }
  }
  if (p.dualt) {
    L.skip();
    line = L.next();
    for (int i = 0; i < 3; ++i)
      if (!inum(W(line, i + 1), r.wrifl[i])) return COSA_ERR_ARG;
    if (r.wrifl[0] <= 0 || r.wrifl[1] < r.wrifl[0] ||
        (r.wrifl[2] > r.wrifl[1] - r.wrifl[0] && r.wrifl[1] != r.wrifl[0]))
      return COSA_ERR_ARG;
  }

  // iteration controls (list-directed)
  L.skip();
  {
    std::vector<std::string> t = L.list(p.viscous ? 7 : 6);
    if (!L.ok) return COSA_ERR_ARG;
    int k = 0;
    if (!inum(t[k++], r.irest) || !inum(t[k++], r.srest) || !num(t[k++], vcfl3)) return COSA_ERR_ARG;
    if (p.viscous && !num(t[k++], p.cdff)) return COSA_ERR_ARG;
    if (!inum(t[k++], r.lmax) || !inum(t[k++], p.iupdt) || !num(t[k++], r.toler)) return COSA_ERR_ARG;
    if (r.irest != 0 && r.irest != 1) return COSA_ERR_ARG;
  }
  // MUSCL kappa and implicit residual smoothing
  L.skip();
  line = L.next();
  if (!num(W(line, 1), p.rkap)) return COSA_ERR_ARG;
  {
    const std::string irs = W(line, 2);
    if (irs == "cirs_v2v") p.irsop = 6;
    else if (irs == "cirs_v1v") p.irsop = 5;
    else if (irs == "cirs_v2") p.irsop = 3;
    else if (irs == "cirs_v1") p.irsop = 2;
    else if (irs == "cirs_c") p.irsop = 1;
    else if (irs == "no_irs") p.irsop = 0;
    else return COSA_ERR_ARG;
    if (p.irsop > 0) {
      if (!num(W(line, 3), vcfli3) || !inum(W(line, 4), p.cutcirs) || (p.cutcirs != 0 && p.cutcirs != 1))
        return COSA_ERR_ARG;
      if ((p.irsop == 3 || p.irsop == 6) && !num(W(line, 5), p.psirs)) return COSA_ERR_ARG;
    }
  }
  if (turb) {
    L.skip();
    line = L.next();
    if (!num(W(line, 1), vcflt3) || !num(W(line, 2), vcflit3)) return COSA_ERR_ARG;
    if (W(line, 3).compare(0, 7, "ramping") == 0) return COSA_ERR_UNSUPPORTED;  // ramps live in the driver
  }
  // mean-flow limiter and entropy fix
  L.skip();
  line = L.next();
  {
    int v;
    if (!inum(W(line, 1), p.ilimf) || !num(W(line, 2), p.epslimf)) return COSA_ERR_ARG;
    if ((e = yn(W(line, 3), p.efx_setup_f))) return e;
    if (p.efx_setup_f) {
      int typ;
      if (!num(W(line, 4), p.cntrpy_f) || p.cntrpy_f < 0 || p.cntrpy_f > 1 || !inum(W(line, 5), typ) ||
          typ < 0 || typ > 2 || !num(W(line, 6), p.entfxctf_f))
        return COSA_ERR_ARG;
      p.entfx_f_w[typ] = 1;
      if ((e = yn(W(line, 7), v))) return e;
      p.efx_all_f = v;
    }
    L.skip();
    line = L.next();
    if ((e = yn(W(line, 1), p.eig_limit_f))) return e;
    if (p.eig_limit_f) {
      if (!num(W(line, 2), p.eig_cutoff_f) || p.eig_cutoff_f < 0 || p.eig_cutoff_f > 1) return COSA_ERR_ARG;
      if ((e = yn(W(line, 3), p.eig_lim_all_f))) return e;
    }
    // turbulence limiter and entropy fix; the reference sets entfx_t_w(2:3)
    // from the mean-flow type (src/input.f90:3444-3446), kept
    int typf = p.efx_setup_f ? (p.entfx_f_w[0] ? 0 : (p.entfx_f_w[1] ? 1 : 2)) : -1;
    L.skip();
    line = L.next();
    if (!inum(W(line, 1), p.ilimt) || !num(W(line, 2), p.epslimt)) return COSA_ERR_ARG;
    if ((e = yn(W(line, 3), p.efx_setup_t))) return e;
    if (p.efx_setup_t) {
      int typ;
      if (!num(W(line, 4), p.cntrpy_t) || p.cntrpy_t < 0 || p.cntrpy_t > 1 || !inum(W(line, 5), typ) ||
          typ < 0 || typ > 2 || !num(W(line, 6), p.entfxctf_t))
        return COSA_ERR_ARG;
      if (typ == 0) p.entfx_t_w[0] = 1;
      if (typf == 1) p.entfx_t_w[1] = 1;
      if (typf == 2) p.entfx_t_w[2] = 1;
      if ((e = yn(W(line, 7), v))) return e;
      p.efx_all_t = v;
    }
    L.skip();
    line = L.next();
    if ((e = yn(W(line, 1), p.eig_limit_t))) return e;
    if (p.eig_limit_t) {
      if (!num(W(line, 2), p.eig_cutoff_t) || p.eig_cutoff_t < 0 || p.eig_cutoff_t > 1) return COSA_ERR_ARG;
      if ((e = yn(W(line, 3), p.eig_lim_all_t))) return e;
    }
  }
  // multigrid
  L.skip();
  {
    std::vector<std::string> t = L.list(7);
    if (!L.ok) return COSA_ERR_ARG;
    if (!inum(t[0], p.nlevel) || !inum(t[1], p.nl_crs) || !inum(t[2], r.nl_fmg) || !inum(t[3], p.nstart) ||
        !inum(t[4], p.npre) || !inum(t[5], p.npost) || !inum(t[6], p.ncrs))
      return COSA_ERR_ARG;
    if (p.nlevel < 1 || p.nlevel > COSA_MAX_LEVELS) return COSA_ERR_ARG;
  }
  if (p.nlevel > 1) {
    L.skip();
    line = L.next();
    const std::string pr = W(line, 1);
    if (pr == "linear") p.bln_prol = 0;
    else if (pr == "bilinear") p.bln_prol = 1;
    else return COSA_ERR_ARG;
    if (turb) {
      const std::string ho = W(line, 2);
      if (ho == "ho_rest") p.ho_rest = 1;
      else if (ho == "lo_rest") p.ho_rest = 0;
      else return COSA_ERR_ARG;
      const std::string lc = W(line, 3);
      if (lc == "lim_corr1") p.lim_corr = 1;
      else if (lc == "lim_corr2") p.lim_corr = 2;
      else if (lc == "lim_corr3") p.lim_corr = 3;
      else return COSA_ERR_ARG;
      if ((e = yn(W(line, 4), p.prd_all_lvls))) return e;
    }
  }
  // low-speed preconditioning control parameters (src/input.f90:3582-3700)
  L.skip();
  line = L.next();
  if (W(line, 1) == "lomach") {
    p.lomach = 1;
    if (!inum(W(line, 2), p.cutoff_type) || p.cutoff_type < 1 || p.cutoff_type > 3) return COSA_ERR_ARG;
    const std::string vp = W(line, 3);
    if (vp == "viscous") {
      if (!p.viscous) return COSA_ERR_ARG;
      p.visprec = 1;
    } else if (vp == "inviscid") {
      p.visprec = 0;
    } else {
      return COSA_ERR_ARG;
    }
    int lsp_vfr = 0;
    if (p.moving && !unsteady && (!inum(W(line, 4), lsp_vfr) || lsp_vfr < 0 || lsp_vfr > 1)) return COSA_ERR_ARG;
    if (unsteady) {
      const std::string mx = W(line, 4);
      if (mx == "standard") p.mixpi = 0;
      else if (mx == "mixed") p.mixpi = 1;
      else return COSA_ERR_ARG;
      double lx = 0, ly = 0;
      if (!num(W(line, 5), lx) || !num(W(line, 6), ly)) return COSA_ERR_ARG;
      // the unsteady reference velocity
      p.uprv = std::max(lx / (pi * r.dt), ly / (pi * r.dt));
      if (p.moving && (!inum(W(line, 7), lsp_vfr) || lsp_vfr < 0 || lsp_vfr > 1)) return COSA_ERR_ARG;
    }
    // the preconditioner's Mach number in the frame of a moving grid is not built
    if (lsp_vfr == 1) return COSA_ERR_UNSUPPORTED;
    // entropy fix type 1 is inadmissible with preconditioning
    if (p.entfx_f_w[1] == 1 || p.entfx_t_w[1] == 1) return COSA_ERR_ARG;
    // the constant cut-off of every multigrid level
    L.skip();
    line = L.next();
    for (int l = 0; l < p.nlevel; ++l)
      if (!num(W(line, l + 1), p.epsp[l])) return COSA_ERR_ARG;
  }
  if (p.viscous) {
    L.skip();
    line = L.next();
    if (!num(W(line, 1), r.tref) || r.tref <= 0) return COSA_ERR_ARG;
    p.stemp = 1.104e2 / r.tref;
  }
  // degenerate cells, restart and tecplot output
  L.skip();
  line = L.next();
  if ((e = yn(W(line, 1), r.dgn_cell)) || (e = yn(W(line, 2), r.wri_res)) || (e = yn(W(line, 3), r.wri_tec)))
    return e;
  L.skip();
  line = L.next();
  {
    const std::string fmt = W(line, 1);
    if (fmt != "cgns" && fmt != "plt" && fmt != "szplt" && fmt != "bin") return COSA_ERR_ARG;
    std::snprintf(r.out_format, sizeof(r.out_format), "%s", fmt.c_str());
  }
  // forces
  L.skip();
  line = L.next();
  {
    const std::string fo = W(line, 1);
    if (fo == "default") {
      r.calfor = 1;
      for (int i = 0; i < 3; ++i)
        if (!num(W(line, 2 + i), r.xmom[i])) return COSA_ERR_ARG;
      L.skip();
      line = L.next();
      for (int i = 0; i < 3; ++i)
        if (!num(W(line, 1 + i), r.lngth[i])) return COSA_ERR_ARG;
      line = L.next();
      if (!inum(W(line, 1), r.nsurface) || r.nsurface < 0 || r.nsurface > 8) return COSA_ERR_ARG;
      for (int s = 0; s < r.nsurface; ++s) {
        line = L.next();
        if (!inum(W(line, 1), r.n_surblo[s]) || r.n_surblo[s] < 0 || r.n_surblo[s] > 64) return COSA_ERR_ARG;
        for (int b = 0; b < r.n_surblo[s]; ++b)
          if (!inum(W(line, 2 + b), r.i_surbl[s][b])) return COSA_ERR_ARG;
      }
    } else if (fo != "none") {
      return COSA_ERR_ARG;
    }
  }
  // blocks and their boundary patches (bcdata, src/input.f90:3795-3840)
  auto *in = new cosa_input;
  auto fail = [&](int code) { delete in; return code; };
  {
    std::vector<std::string> t = L.list(1);
    if (!L.ok || !inum(t[0], in->nblocks) || in->nblocks < 1) return fail(COSA_ERR_ARG);
  }
  for (int b = 0; b < in->nblocks; ++b) {
    line = L.next();
    int32_t im, jm, km, nb;
    if (!inum(W(line, 1), im) || !inum(W(line, 2), jm) || !inum(W(line, 3), km) || !inum(W(line, 4), nb) ||
        im < 2 || jm < 2 || km < 2 || nb < 0)
      return fail(COSA_ERR_ARG);
    in->dims.insert(in->dims.end(), {im, jm, km});
    in->nbcs.push_back(nb);
    for (int ibc = 0; ibc < nb; ++ibc) {
      std::vector<std::string> t = L.list(7);
      int32_t v[7];
      for (int i = 0; i < 7; ++i)
        if (!L.ok || !inum(t[i], v[i])) return fail(COSA_ERR_ARG);
      int istrt[4] = {0, v[0], v[1], v[2]}, iend[4] = {0, v[3], v[4], v[5]};
      int idir = 0;
      for (int i = 1; i <= 3; ++i)
        if (istrt[i] == iend[i]) idir = i;
      if (idir < 1) return fail(COSA_ERR_ARG);
      for (int i = 1; i <= 3; ++i)
        if (i != idir) iend[i] = iend[i] - 1;
      const int32_t rec[10] = {v[6], idir, istrt[idir], istrt[1], iend[1], istrt[2], iend[2], istrt[3], iend[3], 0};
      in->bct.insert(in->bct.end(), rec, rec + 10);
    }
  }
  // cuts (cutdata, src/input.f90:3850-4045): each input cut gives two records
  {
    std::vector<std::string> t = L.list(1);
    int32_t nc;
    if (!L.ok || !inum(t[0], nc) || nc < 0) return fail(COSA_ERR_ARG);
    for (int icut = 0; icut < nc; ++icut) {
      int32_t c1[21] = {0}, c2[21] = {0};
      for (int side = 0; side < 2; ++side) {
        std::vector<std::string> w = L.list(side ? 10 : 7);
        int32_t v[10];
        for (int i = 0; i < (side ? 10 : 7); ++i)
          if (!L.ok || !inum(w[i], v[i])) return fail(COSA_ERR_ARG);
        const int iblk = v[0];
        int istrt[4] = {0, v[1], v[2], v[3]}, iend[4] = {0, v[4], v[5], v[6]};
        int idir = 0;
        for (int l = 1; l <= 3; ++l)
          if (istrt[l] == iend[l]) idir = l;
        if (idir < 1) return fail(COSA_ERR_ARG);
        for (int l = 1; l <= 3; ++l)
          if (l != idir) {
            if (iend[l] > istrt[l]) iend[l] = iend[l] - 1;
            else istrt[l] = istrt[l] - 1;
          }
        const int32_t f9[9] = {iblk, idir, istrt[idir], istrt[1], iend[1], istrt[2], iend[2], istrt[3], iend[3]};
        if (side == 0) {
          std::copy(f9, f9 + 9, c1);
          std::copy(f9, f9 + 9, c2 + 9);
        } else {
          const int iord[4] = {0, v[7], v[8], v[9]};
          for (int l = 1; l <= 3; ++l)
            if (iord[l] < 1 || iord[l] > 3) return fail(COSA_ERR_ARG);
          std::copy(f9, f9 + 9, c1 + 9);
          c1[18] = iord[1]; c1[19] = iord[2]; c1[20] = iord[3];
          std::copy(f9, f9 + 9, c2);
          int m = 1;
          if (iord[1] == 2 && iord[2] == 3) m = 2;
          else if (iord[1] == 3 && iord[2] == 1) m = 3;
          c2[18] = cyc(iord[1], m); c2[19] = cyc(iord[2], m); c2[20] = cyc(iord[3], m);
        }
      }
      in->cut.insert(in->cut.end(), c1, c1 + 21);
      in->cut.insert(in->cut.end(), c2, c2 + 21);
    }
    in->ncuts = 2 * nc;
  }
  // compatibility tests (src/input.f90:4235-4275)
  if ((p.machfs < 1e-14 && p.viscous) || (p.rgkuns && p.nlevel > 1) || (p.rgkuns && p.lomach))
    return fail(COSA_ERR_ARG);
  // IRS for the removal of the diffusion limit is not available with preconditioning
  if (p.lomach && (p.irsop == 5 || p.irsop == 6)) return fail(COSA_ERR_ARG);
  if (turb && p.nlevel > 1 && (!p.bln_prol || (!p.prd_all_lvls && p.lim_prodtke && !p.lim_prodomega)))
    return fail(COSA_ERR_ARG);
  // derived CFL values (src/input.f90:4205-4221)
  if (p.irsop > 0) {
    p.rat = vcfli3 / vcfl3;
    if (turb) p.ratt = vcflit3 / vcflt3;
    p.cfl = vcfli3;
    if (turb) p.cflt = vcflit3;
  } else {
    p.cfl = vcfl3;
    if (turb) p.cflt = vcflt3;
  }
  if (p.dualt || p.rgkuns) p.dt = r.dt;
  // first-order first step unless a dual-time restart holds two states
  // (zeit.dat key 9992999, src/input.f90:5614-5620), which the caller knows
  p.bdf1 = 1;
  *pp = p;
  *rr = r;
  *out = in;
  return COSA_OK;
}

int cosa_io_input_level(const cosa_input *in, cosa_level_desc *d) {
  if (!in || !d) return COSA_ERR_ARG;
  d->nblocks = in->nblocks;
  d->dims = in->dims.data();
  d->nbcs = in->nbcs.data();
  d->bctopo = in->bct.data();
  d->ncuts = in->ncuts;
  d->cutopo = in->cut.data();
  return COSA_OK;
}

int cosa_io_free_input(cosa_input *in) {
  delete in;
  return COSA_OK;
}

int cosa_io_write_input(const char *path, const cosa_params *pp, const cosa_run_opts *rr, const cosa_level_desc *d) {
  if (!path || !pp || !rr || !d || !dims_ok(d->nblocks, d->dims)) return COSA_ERR_ARG;
  const cosa_params &p = *pp;
  const cosa_run_opts &r = *rr;
  const double pi = 3.14159265358979323846;
  const bool turb = p.kom || p.kom_bsl || p.kom_sst;
  if (turb && p.nlevel > 1 && (p.lim_corr < 1 || p.lim_corr > 3)) return COSA_ERR_ARG;  // not expressible
  const char *eqs = p.kom ? "komega" : (p.kom_bsl ? "bsl" : (p.kom_sst ? "sst" : (p.viscous ? "laminar" : "euler")));
  FILE *f = std::fopen(path, "w");
  if (!f) return COSA_ERR_ARG;
  std::fprintf(f, "input.dat\n");
  std::fprintf(f, "mesh\n");
  std::fprintf(f, "%s %s %s aircraft\n", r.debug ? "y" : "n", eqs, r.exter ? "external" : "internal");
  std::fprintf(f, "gamma [reyno pranl] machfs [alpha beta]\n");
  const double ad = p.alpha * 180 / pi, bd = p.beta * 180 / pi;
  if (p.viscous) {
    std::fprintf(f, "%.17g %.17g %.17g %.17g", p.gamma, p.reyno, p.pranl, p.machfs);
    if (r.exter) std::fprintf(f, " %.17g %.17g", ad, bd);
    std::fprintf(f, "\n");
  } else if (r.exter) {
    std::fprintf(f, "%.17g %.17g %.17g %.17g\n", p.gamma, p.machfs, ad, bd);
  } else {
    std::fprintf(f, "%.17g\n", p.gamma);
  }
  if (turb) {
    const double tke = p.tkefar / (p.machfs * p.machfs);
    std::fprintf(f, "prant tkefar mutfar wall\n%.17g %.17g %.17g %s", p.prant, tke, p.mutfar,
                 p.wallwilc ? "wilcox" : "menter");
    if (p.wallwilc) std::fprintf(f, " %.17g", p.roughk);
    std::fprintf(f, "\nturcmp lim_prodtke prdlim lim_prodomega fixq order\n%s %s %.17g %s %s %s\n",
                 p.turcmp != 0 ? "y" : "n", p.lim_prodtke ? "y" : "n", p.prdlim, p.lim_prodomega ? "y" : "n",
                 p.ifixq ? "minimum" : "none", p.foturb ? "first" : "second");
  }
  std::fprintf(f, "time\n");
  if (p.harbal) std::fprintf(f, "unsteady hb %s %d\n", p.rkimp ? "rkim" : "rkex", p.nharms);
  else if (p.rgkuns) std::fprintf(f, "unsteady rgkun %.17g\n", r.dt);
  else if (p.dualt) std::fprintf(f, "unsteady dual %.17g %d %d second %s\n", r.dt, r.ntime, r.nsave,
                                 p.rkimp ? "rkim" : "rkex");
  else std::fprintf(f, "steady\n");
  if (p.harbal || p.rgkuns || p.dualt) {
    std::fprintf(f, "motion\n");
    if (p.moving) std::fprintf(f, "pitch %.17g %.17g %.17g %.17g\n", p.omegas / (2 * pi), p.xh, p.yh,
                               p.dtheta0 * 180 / pi);
    else std::fprintf(f, "fixed\n");
  }
  if (p.dualt) std::fprintf(f, "wrifl\n%d %d %d\n", r.wrifl[0], r.wrifl[1], r.wrifl[2]);
  const double vcfl = p.irsop > 0 ? p.cfl / p.rat : p.cfl;
  std::fprintf(f, "irest srest cfl [cdff] lmax iupdt toler\n%d %d %.17g", r.irest, r.srest, vcfl);
  if (p.viscous) std::fprintf(f, " %.17g", p.cdff);
  std::fprintf(f, " %d %d %.17g\n", r.lmax, p.iupdt, r.toler);
  static const char *irs[7] = {"no_irs", "cirs_c", "cirs_v1", "cirs_v2", "", "cirs_v1v", "cirs_v2v"};
  std::fprintf(f, "rkap irs\n%.17g %s", p.rkap, irs[std::min(std::max(p.irsop, 0), 6)]);
  if (p.irsop > 0) {
    std::fprintf(f, " %.17g %d", p.cfl, p.cutcirs);
    if (p.irsop == 3 || p.irsop == 6) std::fprintf(f, " %.17g", p.psirs);
  }
  std::fprintf(f, "\n");
  if (turb) {
    const double vt = p.irsop > 0 ? p.cflt / p.ratt : p.cflt;
    std::fprintf(f, "cflt cflit\n%.17g %.17g\n", vt, p.cflt);
  }
  auto typ_of = [](const int32_t *w) { return w[0] ? 0 : (w[1] ? 1 : 2); };
  std::fprintf(f, "ilimf epslimf efx\n%d %.17g %s", p.ilimf, p.epslimf, p.efx_setup_f ? "y" : "n");
  if (p.efx_setup_f)
    std::fprintf(f, " %.17g %d %.17g %s", p.cntrpy_f, typ_of(p.entfx_f_w), p.entfxctf_f, p.efx_all_f ? "y" : "n");
  std::fprintf(f, "\neig_limit_f\n%s", p.eig_limit_f ? "y" : "n");
  if (p.eig_limit_f) std::fprintf(f, " %.17g %s", p.eig_cutoff_f, p.eig_lim_all_f ? "y" : "n");
  std::fprintf(f, "\nilimt epslimt efx\n%d %.17g %s", p.ilimt, p.epslimt, p.efx_setup_t ? "y" : "n");
  if (p.efx_setup_t)
    std::fprintf(f, " %.17g %d %.17g %s", p.cntrpy_t, typ_of(p.entfx_t_w), p.entfxctf_t, p.efx_all_t ? "y" : "n");
  std::fprintf(f, "\neig_limit_t\n%s", p.eig_limit_t ? "y" : "n");
  if (p.eig_limit_t) std::fprintf(f, " %.17g %s", p.eig_cutoff_t, p.eig_lim_all_t ? "y" : "n");
  std::fprintf(f, "\nnlevel nl_crs nl_fmg nstart npre npost ncrs\n%d %d %d %d %d %d %d\n", p.nlevel, p.nl_crs,
               r.nl_fmg, p.nstart, p.npre, p.npost, p.ncrs);
  if (p.nlevel > 1) {
    std::fprintf(f, "prolongation\n%s", p.bln_prol ? "bilinear" : "linear");
    if (turb) std::fprintf(f, " %s lim_corr%d %s", p.ho_rest ? "ho_rest" : "lo_rest", p.lim_corr,
                           p.prd_all_lvls ? "y" : "n");
    std::fprintf(f, "\n");
  }
  if (p.lomach) {
    std::fprintf(f, "preconditioning\nlomach %d %s", p.cutoff_type, p.visprec ? "viscous" : "inviscid");
    if (p.harbal || p.dualt || p.rgkuns) {
      const double l = p.uprv * pi * r.dt;
      std::fprintf(f, " %s %.17g %.17g", p.mixpi ? "mixed" : "standard", l, l);
    }
    std::fprintf(f, "\nepsp\n");
    for (int l = 0; l < p.nlevel; ++l) std::fprintf(f, "%s%.17g", l ? " " : "", p.epsp[l]);
    std::fprintf(f, "\n");
  } else {
    std::fprintf(f, "preconditioning\nnone\n");
  }
  if (p.viscous) std::fprintf(f, "tref\n%.17g\n", 110.4 / p.stemp);
  std::fprintf(f, "dgn_cell wri_res wri_tec\n%s %s %s\n", r.dgn_cell ? "y" : "n", r.wri_res ? "y" : "n",
               r.wri_tec ? "y" : "n");
  std::fprintf(f, "output\n%s\n", r.out_format[0] ? r.out_format : "bin");
  if (r.calfor) {
    std::fprintf(f, "forces\ndefault %.17g %.17g %.17g\nlengths\n%.17g %.17g %.17g\n%d\n", r.xmom[0], r.xmom[1],
                 r.xmom[2], r.lngth[0], r.lngth[1], r.lngth[2], r.nsurface);
    for (int s = 0; s < r.nsurface; ++s) {
      std::fprintf(f, "%d", r.n_surblo[s]);
      for (int b = 0; b < r.n_surblo[s]; ++b) std::fprintf(f, " %d", r.i_surbl[s][b]);
      std::fprintf(f, "\n");
    }
  } else {
    std::fprintf(f, "forces\nnone\n");
  }
  // blocks: the input file gives node ranges; bcdata stores cell ranges
  std::fprintf(f, "%d\n", d->nblocks);
  int64_t ob = 0;
  for (int b = 0; b < d->nblocks; ++b) {
    std::fprintf(f, "%d %d %d %d\n", d->dims[3 * b], d->dims[3 * b + 1], d->dims[3 * b + 2], d->nbcs[b]);
    for (int ibc = 0; ibc < d->nbcs[b]; ++ibc, ob += 10) {
      const int32_t *t = d->bctopo + ob;
      const int idir = t[1];
      int lo[4] = {0, t[3], t[5], t[7]}, hi[4] = {0, t[4], t[6], t[8]};
      for (int i = 1; i <= 3; ++i)
        if (i != idir) hi[i] = hi[i] + 1;
      std::fprintf(f, "%d %d %d %d %d %d %d\n", lo[1], lo[2], lo[3], hi[1], hi[2], hi[3], t[0]);
    }
  }
  // cuts: the first record of each pair holds both sides with iord
  std::fprintf(f, "%d\n", d->ncuts / 2);
  for (int ic = 0; ic + 1 < d->ncuts; ic += 2) {
    const int32_t *c = d->cutopo + 21 * (int64_t)ic;
    for (int side = 0; side < 2; ++side) {
      const int32_t *s = c + 9 * side;
      const int idir = s[1];
      int lo[4] = {0, s[3], s[5], s[7]}, hi[4] = {0, s[4], s[6], s[8]};
      for (int l = 1; l <= 3; ++l)
        if (l != idir) {
          if (hi[l] >= lo[l]) hi[l] = hi[l] + 1;
          else lo[l] = lo[l] + 1;
        }
      std::fprintf(f, "%d %d %d %d %d %d %d", s[0], lo[1], lo[2], lo[3], hi[1], hi[2], hi[3]);
      if (side == 1) std::fprintf(f, " %d %d %d", c[18], c[19], c[20]);
      std::fprintf(f, "\n");
    }
  }
  const bool ok = std::fclose(f) == 0;
  return ok ? COSA_OK : COSA_ERR_ARG;
}

int cosa_io_read_mesh(const char *path, int32_t nb, const int32_t *dims, int32_t with_disp, double *x, double *y,
                      double *z, double *dx, double *dy, double *dz) {
  if (!path || !dims_ok(nb, dims) || !x || !y || !z || (with_disp && (!dx || !dy || !dz))) return COSA_ERR_ARG;
  FILE *f = std::fopen(path, "rb");
  if (!f) return COSA_ERR_ARG;
  const Offs o = offsets(nb, dims);
  std::vector<char> rec;
  int status = COSA_OK;
  for (int b = 0; b < nb && !status; ++b) {
    const int64_t im = dims[3 * b], jm = dims[3 * b + 1], km = dims[3 * b + 2], n = im * jm * km;
    double *xyz[3] = {x, y, z}, *dxyz[3] = {dx, dy, dz};
    for (int part = 0; part < (with_disp ? 2 : 1) && !status; ++part) {
      if (!read_record(f, rec) || (int64_t)rec.size() != 3 * n * 8) { status = COSA_ERR_ARG; break; }
      const double *v = reinterpret_cast<const double *>(rec.data());
      for (int c = 0; c < 3; ++c)
        for (int64_t k = 1; k <= km; ++k)
          for (int64_t j = 1; j <= jm; ++j)
            for (int64_t i = 1; i <= im; ++i) {
              const double val = v[c * n + (i - 1) + im * ((j - 1) + jm * (k - 1))];
              if (part == 0) xyz[c][o.p2[b] + i + (im + 2) * (j + (jm + 2) * k)] = val;
              else dxyz[c][o.p1[b] + i + (im + 1) * (j + (jm + 1) * k)] = val;
            }
    }
  }
  std::fclose(f);
  return status;
}

int cosa_io_write_mesh(const char *path, int32_t nb, const int32_t *dims, int32_t with_disp, const double *x,
                       const double *y, const double *z, const double *dx, const double *dy, const double *dz) {
  if (!path || !dims_ok(nb, dims) || !x || !y || !z || (with_disp && (!dx || !dy || !dz))) return COSA_ERR_ARG;
  FILE *f = std::fopen(path, "wb");
  if (!f) return COSA_ERR_ARG;
  const Offs o = offsets(nb, dims);
  bool ok = true;
  for (int b = 0; b < nb && ok; ++b) {
    const int64_t im = dims[3 * b], jm = dims[3 * b + 1], km = dims[3 * b + 2], n = im * jm * km;
    const double *xyz[3] = {x, y, z}, *dxyz[3] = {dx, dy, dz};
    std::vector<double> buf(3 * n);
    for (int part = 0; part < (with_disp ? 2 : 1) && ok; ++part) {
      for (int c = 0; c < 3; ++c)
        for (int64_t k = 1; k <= km; ++k)
          for (int64_t j = 1; j <= jm; ++j)
            for (int64_t i = 1; i <= im; ++i)
              buf[c * n + (i - 1) + im * ((j - 1) + jm * (k - 1))] =
                  part == 0 ? xyz[c][o.p2[b] + i + (im + 2) * (j + (jm + 2) * k)]
                            : dxyz[c][o.p1[b] + i + (im + 1) * (j + (jm + 1) * k)];
      ok = write_record(f, buf.data(), 3 * n * 8);
    }
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? COSA_OK : COSA_ERR_ARG;
}

int cosa_io_read_restart(const char *path, int32_t nb, const int32_t *dims, int32_t npde, int32_t nharms,
                         int32_t with_q1, int32_t with_mut, double *q, double *q1, double *mut) {
  // q1 (dual time) has no snapshots: with_q1 needs nharms = 0
  if (!path || !dims_ok(nb, dims) || npde < 1 || nharms < 0 || !q || (with_q1 && (!q1 || nharms)) ||
      (with_mut && !mut))
    return COSA_ERR_ARG;
  FILE *f = std::fopen(path, "rb");
  if (!f) return COSA_ERR_ARG;
  const Offs o = offsets(nb, dims);
  const int64_t S = 2 * nharms + 1;
  std::vector<char> rec;
  int status = COSA_OK;
  for (int b = 0; b < nb && !status; ++b) {
    const int64_t P3 = (int64_t)(dims[3 * b] + 3) * (dims[3 * b + 1] + 3) * (dims[3 * b + 2] + 3);
    struct Part { double *dst; int64_t n; bool on; };
    const Part parts[3] = {{q + o.p3[b] * npde * S, P3 * npde * S, true},
                           {q1 ? q1 + o.p3[b] * npde : nullptr, P3 * npde, with_q1 != 0},
                           {mut ? mut + o.p3[b] * S : nullptr, P3 * S, with_mut != 0}};
    for (const Part &pt : parts) {
      if (!pt.on) continue;
      if (!read_record(f, rec) || (int64_t)rec.size() != pt.n * 8) { status = COSA_ERR_ARG; break; }
      std::memcpy(pt.dst, rec.data(), rec.size());
    }
  }
  std::fclose(f);
  return status;
}

int cosa_io_write_restart(const char *path, int32_t nb, const int32_t *dims, int32_t npde, int32_t nharms,
                          int32_t with_q1, int32_t with_mut, const double *q, const double *q1, const double *mut) {
  // q1 (dual time) has no snapshots: with_q1 needs nharms = 0
  if (!path || !dims_ok(nb, dims) || npde < 1 || nharms < 0 || !q || (with_q1 && (!q1 || nharms)) ||
      (with_mut && !mut))
    return COSA_ERR_ARG;
  FILE *f = std::fopen(path, "wb");
  if (!f) return COSA_ERR_ARG;
  const Offs o = offsets(nb, dims);
  const int64_t S = 2 * nharms + 1;
  bool ok = true;
  for (int b = 0; b < nb && ok; ++b) {
    const int64_t P3 = (int64_t)(dims[3 * b] + 3) * (dims[3 * b + 1] + 3) * (dims[3 * b + 2] + 3);
    ok = write_record(f, q + o.p3[b] * npde * S, P3 * npde * S * 8);
    if (ok && with_q1) ok = write_record(f, q1 + o.p3[b] * npde, P3 * npde * 8);
    if (ok && with_mut) ok = write_record(f, mut + o.p3[b] * S, P3 * S * 8);
  }
  ok = (std::fclose(f) == 0) && ok;
  return ok ? COSA_OK : COSA_ERR_ARG;
}

// history files of output() (src/output.f90:4941-4965): hist.dat holds
// resrms(1:5), histur.dat resrms(6:npde) of k-omega runs, histg.dat the last
// cycle's line; format (i7,2x,i7,5(1x,e13.5))
int cosa_io_hist_record(int32_t itime, int32_t it, const double *res, int32_t n, char *buf, int64_t cap) {
  if (!res || n < 0 || n > 5) return COSA_ERR_ARG;
  std::vector<FItem> f = {{'I', 7, 0}, {'X', 2, 0}, {'I', 7, 0}};
  push_n(f, 5, {'X', 1, 0}, {'E', 13, 5});
  return copy_out(fortran_write(f, {itime, it}, std::vector<double>(res, res + n)), buf, cap);
}

// the header force() writes when it creates the force file of snapshot n
// (src/output.f90:4100-4240): forces_tec.dat for steady and time-accurate
// runs, forces_hb_<nnn>.dat per snapshot for harmonic balance.  The variable
// lists keep the reference's spellings, among them the second "it" of the
// two- and four-surface time-accurate fixed-grid lists, "Cm2_v" for "Cm1_v"
// in the three-surface steady list and "Cm_p","Cm_v" for surface 1 of the
// two-surface moving harmonic-balance list; the harmonic-balance title is
// a 72-character line (trailing blanks kept)
int cosa_io_force_header(const cosa_params *p, int32_t nsurface, int32_t n, char *buf, int64_t cap) {
  if (!p || nsurface < 1 || nsurface > 4 || n < 0 || n > 999) return COSA_ERR_ARG;
  const bool unsteady_t = p->dualt || p->rgkuns;
  std::string names;
  for (int is = 1; is <= nsurface; ++is) names += force_names(is, nsurface);
  std::string t;
  if (!p->harbal) {
    t = " TITLE=\"Force coefficients\"\n";
    std::string head;
    if (unsteady_t) {
      head = "\"itime\",\"it\",\"time\"";
      if (!p->moving && (nsurface == 2 || nsurface == 4)) head += ",\"it\"";
    } else {
      head = "\"it\"";
      if (nsurface == 3) {
        const size_t at = names.find("\"Cm1_v\"");
        if (at != std::string::npos) names.replace(at, 7, "\"Cm2_v\"");
      }
    }
    t += " VARIABLES=" + head + names + (unsteady_t && p->moving ? ",\"alpha\"" : "") + "\n";
  } else {
    char line[80];
    std::snprintf(line, sizeof(line), " TITLE=\"Force coefficients, Harmonic %2d\"", n);
    std::string l(line);
    l.resize(72, ' ');
    t = l + "\n";
    if (p->moving) {
      if (nsurface == 2) {
        const size_t at = names.find("\"Cm1_p\",\"Cm1_v\"");
        if (at != std::string::npos) names.replace(at, 15, "\"Cm_p\",\"Cm_v\"");
      }
      t += " VARIABLES=\"it\",\"time\"" + names + ",\"alpha\"\n";
    } else {
      t += " VARIABLES=\"it\",\"time\",\"Cl\",\"Cd\",\"Cz\"\n";
    }
  }
  return copy_out(t, buf, cap);
}

// one record of the force file of snapshot n (src/output.f90:4310-4360,
// formats 212-220): coef holds per surface cl_p, cl_v, cd_p, cd_v, cz_p, cz_v,
// cmx_p, cmx_v, cmy_p, cmy_v, cm_p, cm_v; time the physical time of a
// time-accurate run, zeit the snapshot's time of harmonic balance, alpha_deg
// the effective incidence of a moving grid
int cosa_io_force_record(const cosa_params *p, int32_t nsurface, int32_t itime, int32_t it, double time,
                         double zeit, const double *coef, double alpha_deg, char *buf, int64_t cap) {
  if (!p || !coef || nsurface < 1 || nsurface > 4) return COSA_ERR_ARG;
  std::vector<double> v;
  std::vector<long long> ints;
  std::vector<FItem> f;
  if (p->dualt || p->rgkuns) {
    ints = {itime, it};
    v.push_back(time);
    f = force_format(true, true, p->moving);
  } else if (!p->harbal) {
    ints = {it};
    f = force_format(false, false, false);
  } else {
    ints = {it};
    v.push_back(zeit);
    f = force_format(false, true, p->moving);
  }
  v.insert(v.end(), coef, coef + 12 * nsurface);
  if ((p->dualt || p->rgkuns || p->harbal) && p->moving) v.push_back(alpha_deg);
  return copy_out(fortran_write(f, ints, v), buf, cap);
}

}  // extern "C"
