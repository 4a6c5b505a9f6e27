// mesh_io.cpp -- the ADCIRC text files at this path's edges: the fort.14
// mesh (read14, mesh.F:319-581) and the full-domain ASCII output files
// fort.63/fort.64 (header63/64, globalio.F:1005-1085; writeFullFormat and
// storeOne/storeTwo, globalio.F:544-643, 802-930).  They let the same mesh
// and results pass between this library and a reference build.
//
// fort.14 node numbers may be any labels; as read14 does, they are mapped
// to 1..NP in file order and element and boundary references go through
// that map.  Boundary segments of the types the 2DDI hot path handles
// (one node per line: IBTYPE 0, 1, 2, 10, 11, 12, 20, 21, 22, 30, 32, 40,
// 41, 52, 102, 112, 122, 152; external barriers 3, 13, 23 with the crest
// height BARLANHT and discharge coefficient BARLANCFSP after the node,
// mesh.F:460-473; internal barriers 4, 24 with the paired node IBCONN,
// BARINHT, BARINCFSB and BARINCFSP, mesh.F:479-495, and 5, 25 with the
// pipe's PIPEHT, PIPECOEF and PIPEDIAM after them, mesh.F:506-524; their
// pairs count twice in NVEL, mesh.F:260-268) are returned; periodic
// segments (94) return ADC_ERR_UNSUPPORTED.
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/adcgpu.h"

namespace adc {
void set_error(const char *fmt, ...);
}
using adc::set_error;

namespace {

// Whitespace/comma-separated numeric reader over a whole text file, with
// line tracking for messages (Fortran list-directed input accepts either).
struct Reader {
  std::string buf;
  size_t pos = 0;
  int line = 1;
  bool open(const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    return true;
  }
  std::string read_line() {   // the rest of the current line
    size_t e = buf.find('\n', pos);
    if (e == std::string::npos) e = buf.size();
    std::string s = buf.substr(pos, e - pos);
    pos = e < buf.size() ? e + 1 : e;
    ++line;
    if (!s.empty() && s.back() == '\r') s.pop_back();
    return s;
  }
  void skip_ws() {
    while (pos < buf.size() && (buf[pos] == ' ' || buf[pos] == '\t' || buf[pos] == ',' ||
                                buf[pos] == '\r' || buf[pos] == '\n')) {
      if (buf[pos] == '\n') ++line;
      ++pos;
    }
  }
  bool num(double &v) {
    skip_ws();
    if (pos >= buf.size()) return false;
    const char *s = buf.c_str() + pos;
    char *end = nullptr;
    // Fortran exponents may use D
    std::string tok;
    size_t k = pos;
    while (k < buf.size() && !std::strchr(" \t,\r\n", buf[k])) ++k;
    tok = buf.substr(pos, k - pos);
    for (char &ch : tok)
      if (ch == 'd' || ch == 'D') ch = 'e';
    errno = 0;
    v = std::strtod(tok.c_str(), &end);
    (void)s;
    if (end == tok.c_str() || *end != '\0' || errno == ERANGE) return false;
    pos = k;
    return true;
  }
  bool inum(long long &v) {
    double d;
    if (!num(d) || d != std::floor(d)) return false;
    v = (long long)d;
    return true;
  }
  // drop what is left of the current line (trailing comments)
  void end_line() {
    size_t e = buf.find('\n', pos);
    if (e == std::string::npos) {
      pos = buf.size();
    } else {
      pos = e + 1;
      ++line;
    }
  }
};

bool simple_flux_type(long long t) {
  switch (t) {
    case 0: case 1: case 2: case 10: case 11: case 12: case 20: case 21: case 22: case 30:
    case 32: case 40: case 41: case 52: case 102: case 112: case 122: case 152:
    case 3: case 13: case 23: case 4: case 24: case 5: case 25:
      return true;
    default:
      return false;
  }
}

struct Mesh14 {
  std::string title;
  std::vector<double> x, y, dp;
  std::vector<int> nm;                 // NM(NE,3), 1-based
  std::vector<int> nvdll, nbdv, nvell, ibtype, nbvv;
  std::vector<double> barlanht, barlancfsp;   // per nbvv entry, 0 off external barriers
  std::vector<int> ibconn;                     // per nbvv entry, 0 off internal barriers
  std::vector<double> barinht, barincfsb, barincfsp;
  std::vector<double> pipeht, pipecoef, pipediam;
};

bool external_barrier(long long t) { return t == 3 || t == 13 || t == 23; }
bool pipe_barrier(long long t) { return t == 5 || t == 25; }
bool internal_barrier(long long t) { return t == 4 || t == 24 || pipe_barrier(t); }

int parse14(const char *path, Mesh14 &m) {
  Reader r;
  if (!r.open(path)) { set_error("fort.14: cannot open %s", path); return ADC_ERR_ARG; }
  m.title = r.read_line();
  long long ne, np;
  auto bad = [&](const char *what) {
    set_error("fort.14 %s: %s near line %d", path, what, r.line);
    return ADC_ERR_MESH;
  };
  if (!r.inum(ne) || !r.inum(np) || ne < 1 || np < 3) return bad("NE NP");
  r.end_line();
  m.x.resize(np); m.y.resize(np); m.dp.resize(np);
  std::unordered_map<long long, int> label;
  label.reserve(np * 2);
  for (long long k = 0; k < np; ++k) {
    long long lab;
    if (!r.inum(lab) || !r.num(m.x[k]) || !r.num(m.y[k]) || !r.num(m.dp[k])) return bad("node table");
    r.end_line();
    if (!label.emplace(lab, (int)k + 1).second) return bad("repeated node label");
  }
  auto find = [&](long long lab, int &out) {
    auto it = label.find(lab);
    if (it == label.end()) return false;
    out = it->second;
    return true;
  };
  m.nm.assign(3 * ne, 0);
  for (long long e = 0; e < ne; ++e) {
    long long je, nhy, n[3];
    if (!r.inum(je) || !r.inum(nhy) || !r.inum(n[0]) || !r.inum(n[1]) || !r.inum(n[2]))
      return bad("element table");
    r.end_line();
    if (nhy != 3) return bad("element with NHY != 3");
    for (int k = 0; k < 3; ++k)
      if (!find(n[k], m.nm[e + ne * k])) return bad("element refers to an unknown node");
  }
  long long nope, neta;
  if (!r.inum(nope)) return bad("NOPE");
  r.end_line();
  if (!r.inum(neta)) return bad("NETA");
  r.end_line();
  for (long long k = 0; k < nope; ++k) {
    long long nv;
    if (!r.inum(nv)) return bad("NVDLL");
    r.end_line();   // an IBTYPEE may follow on the line
    m.nvdll.push_back((int)nv);
    for (long long j = 0; j < nv; ++j) {
      long long lab;
      int id;
      if (!r.inum(lab) || !find(lab, id)) return bad("elevation boundary node");
      r.end_line();
      m.nbdv.push_back(id);
    }
  }
  if ((long long)m.nbdv.size() != neta) return bad("NETA does not match the segment lengths");
  long long nbou, nvel, nvel_count = 0;
  if (!r.inum(nbou)) return bad("NBOU");
  r.end_line();
  if (!r.inum(nvel)) return bad("NVEL");
  r.end_line();
  for (long long k = 0; k < nbou; ++k) {
    long long nv, t;
    if (!r.inum(nv) || !r.inum(t)) return bad("NVELL IBTYPE");
    r.end_line();
    if (!simple_flux_type(t)) {
      set_error("fort.14 %s: boundary segment %lld has IBTYPE %lld (barrier or periodic), which "
                "this path does not implement", path, k + 1, t);
      return ADC_ERR_UNSUPPORTED;
    }
    m.nvell.push_back((int)nv);
    m.ibtype.push_back((int)t);
    for (long long j = 0; j < nv; ++j) {
      long long lab;
      int id;
      if (!r.inum(lab) || !find(lab, id)) return bad("flux boundary node");
      double ht = 0.0, cf = 0.0, iht = 0.0, icb = 0.0, icp = 0.0, pht = 0.0, pcf = 0.0, pdm = 0.0;
      int across = 0;
      if (external_barrier(t) && (!r.num(ht) || !r.num(cf)))
        return bad("external barrier node (NBVV BARLANHT BARLANCFSP)");
      if (internal_barrier(t)) {
        long long lab2;
        if (!r.inum(lab2) || !find(lab2, across) || !r.num(iht) || !r.num(icb) || !r.num(icp))
          return bad("internal barrier node (NBVV IBCONN BARINHT BARINCFSB BARINCFSP)");
        if (pipe_barrier(t) && (!r.num(pht) || !r.num(pcf) || !r.num(pdm)))
          return bad("barrier pipe (PIPEHT PIPECOEF PIPEDIAM)");
      }
      r.end_line();
      m.nbvv.push_back(id);
      m.barlanht.push_back(ht);
      m.barlancfsp.push_back(cf);
      m.ibconn.push_back(across);
      m.barinht.push_back(iht);
      m.barincfsb.push_back(icb);
      m.barincfsp.push_back(icp);
      m.pipeht.push_back(pht);
      m.pipecoef.push_back(pcf);
      m.pipediam.push_back(pdm);
      nvel_count += internal_barrier(t) ? 2 : 1;
    }
  }
  if (nvel_count != nvel) return bad("NVEL does not match the segment lengths");
  return ADC_OK;
}

// Fortran 1PE20.10E3 (one digit before the point, 10 after, a 3-digit
// exponent field) right-justified in 20 columns.
void fmt_1pe(char *out, double v, int width, int digits) {
  if (std::isnan(v) || std::isinf(v)) {
    std::snprintf(out, width + 1, "%*s", width, std::isnan(v) ? "NaN" : (v > 0 ? "Infinity" : "-Infinity"));
    return;
  }
  char m[64];
  std::snprintf(m, sizeof(m), "%.*E", digits, v);
  char *e = std::strchr(m, 'E');
  int ex = std::atoi(e + 1);
  *e = '\0';
  char full[80];
  std::snprintf(full, sizeof(full), "%sE%c%03d", m, ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
  std::snprintf(out, width + 1, "%*s", width, full);
}

// Fortran E15.7E3 without a scale factor: 0.ddddddd E+eee.
void fmt_e0(char *out, double v, int width, int digits) {
  if (v == 0.0) {
    char full[64];
    std::snprintf(full, sizeof(full), "0.%0*dE+000", digits, 0);
    std::snprintf(out, width + 1, "%*s", width, full);
    return;
  }
  char m[64];
  std::snprintf(m, sizeof(m), "%.*E", digits - 1, v);   // d.dddddd E x
  char *e = std::strchr(m, 'E');
  int ex = std::atoi(e + 1) + 1;
  *e = '\0';
  std::string mant(m);
  bool neg = mant[0] == '-';
  if (neg) mant.erase(0, 1);
  mant.erase(1, 1);   // drop the point: ddddddd
  char full[80];
  std::snprintf(full, sizeof(full), "%s0.%sE%c%03d", neg ? "-" : "", mant.c_str(), ex < 0 ? '-' : '+',
                ex < 0 ? -ex : ex);
  std::snprintf(out, width + 1, "%*s", width, full);
}

}  // namespace

extern "C" int adc_fort14_dims(const char *path, int dims[6]) {
  if (!path || !dims) { set_error("adc_fort14_dims: null argument"); return ADC_ERR_ARG; }
  Mesh14 m;
  int rc = parse14(path, m);
  if (rc) return rc;
  dims[0] = (int)m.x.size();
  dims[1] = (int)(m.nm.size() / 3);
  dims[2] = (int)m.nvdll.size();
  dims[3] = (int)m.nbdv.size();
  dims[4] = (int)m.nvell.size();
  dims[5] = (int)m.nbvv.size();
  return ADC_OK;
}

extern "C" int adc_fort14_read(const char *path, char *title, double *x, double *y, double *dp,
                               int *nm, int *nvdll, int *nbdv, int *nvell, int *ibtype, int *nbvv) {
  if (!path || !x || !y || !dp || !nm) { set_error("adc_fort14_read: null argument"); return ADC_ERR_ARG; }
  Mesh14 m;
  int rc = parse14(path, m);
  if (rc) return rc;
  if (title) {
    std::strncpy(title, m.title.c_str(), 80);
    title[80] = '\0';
  }
  std::memcpy(x, m.x.data(), m.x.size() * sizeof(double));
  std::memcpy(y, m.y.data(), m.y.size() * sizeof(double));
  std::memcpy(dp, m.dp.data(), m.dp.size() * sizeof(double));
  std::memcpy(nm, m.nm.data(), m.nm.size() * sizeof(int));
  if (nvdll && !m.nvdll.empty()) std::memcpy(nvdll, m.nvdll.data(), m.nvdll.size() * sizeof(int));
  if (nbdv && !m.nbdv.empty()) std::memcpy(nbdv, m.nbdv.data(), m.nbdv.size() * sizeof(int));
  if (nvell && !m.nvell.empty()) std::memcpy(nvell, m.nvell.data(), m.nvell.size() * sizeof(int));
  if (ibtype && !m.ibtype.empty()) std::memcpy(ibtype, m.ibtype.data(), m.ibtype.size() * sizeof(int));
  if (nbvv && !m.nbvv.empty()) std::memcpy(nbvv, m.nbvv.data(), m.nbvv.size() * sizeof(int));
  return ADC_OK;
}

extern "C" int adc_fort14_barriers(const char *path, double *barlanht, double *barlancfsp) {
  if (!path || !barlanht || !barlancfsp) {
    set_error("adc_fort14_barriers: null argument");
    return ADC_ERR_ARG;
  }
  Mesh14 m;
  int rc = parse14(path, m);
  if (rc) return rc;
  if (!m.barlanht.empty()) {
    std::memcpy(barlanht, m.barlanht.data(), m.barlanht.size() * sizeof(double));
    std::memcpy(barlancfsp, m.barlancfsp.data(), m.barlancfsp.size() * sizeof(double));
  }
  return ADC_OK;
}

extern "C" int adc_fort14_internal_barriers(const char *path, int *ibconn, double *barinht,
                                            double *barincfsb, double *barincfsp, double *pipeht,
                                            double *pipecoef, double *pipediam) {
  if (!path || !ibconn || !barinht || !barincfsb || !barincfsp) {
    set_error("adc_fort14_internal_barriers: null argument");
    return ADC_ERR_ARG;
  }
  Mesh14 m;
  int rc = parse14(path, m);
  if (rc) return rc;
  const size_t n = m.nbvv.size();
  if (n) {
    std::memcpy(ibconn, m.ibconn.data(), n * sizeof(int));
    std::memcpy(barinht, m.barinht.data(), n * sizeof(double));
    std::memcpy(barincfsb, m.barincfsb.data(), n * sizeof(double));
    std::memcpy(barincfsp, m.barincfsp.data(), n * sizeof(double));
    if (pipeht) std::memcpy(pipeht, m.pipeht.data(), n * sizeof(double));
    if (pipecoef) std::memcpy(pipecoef, m.pipecoef.data(), n * sizeof(double));
    if (pipediam) std::memcpy(pipediam, m.pipediam.data(), n * sizeof(double));
  }
  return ADC_OK;
}

extern "C" int adc_fort14_write(const char *path, const char *title, int np, int ne, const double *x,
                                const double *y, const double *dp, const int *nm, int nope,
                                const int *nvdll, const int *nbdv, int nbou, const int *nvell,
                                const int *ibtype, const int *nbvv) {
  return adc_fort14_write_barriers(path, title, np, ne, x, y, dp, nm, nope, nvdll, nbdv, nbou,
                                   nvell, ibtype, nbvv, nullptr, nullptr, nullptr, nullptr, nullptr,
                                   nullptr, nullptr, nullptr, nullptr);
}

extern "C" int adc_fort14_write_barriers(const char *path, const char *title, int np, int ne,
                                         const double *x, const double *y, const double *dp,
                                         const int *nm, int nope, const int *nvdll,
                                         const int *nbdv, int nbou, const int *nvell,
                                         const int *ibtype, const int *nbvv,
                                         const double *barlanht, const double *barlancfsp,
                                         const int *ibconn, const double *barinht,
                                         const double *barincfsb, const double *barincfsp,
                                         const double *pipeht, const double *pipecoef,
                                         const double *pipediam) {
  if (!path || !x || !y || !dp || !nm || np < 3 || ne < 1 || nope < 0 || nbou < 0) {
    set_error("adc_fort14_write: bad arguments");
    return ADC_ERR_ARG;
  }
  FILE *f = std::fopen(path, "w");
  if (!f) { set_error("adc_fort14_write: cannot open %s", path); return ADC_ERR_ARG; }
  std::fprintf(f, "%s\n", title ? title : "adcirc_b200 mesh");
  std::fprintf(f, "%d %d\n", ne, np);
  // %.17g round-trips every double
  for (int i = 0; i < np; ++i) std::fprintf(f, "%d %.17g %.17g %.17g\n", i + 1, x[i], y[i], dp[i]);
  for (int e = 0; e < ne; ++e)
    std::fprintf(f, "%d 3 %d %d %d\n", e + 1, nm[e], nm[e + (size_t)ne], nm[e + 2 * (size_t)ne]);
  long long neta = 0;
  for (int k = 0; k < nope; ++k) neta += nvdll[k];
  std::fprintf(f, "%d\n%lld\n", nope, neta);
  long long q = 0;
  for (int k = 0; k < nope; ++k) {
    std::fprintf(f, "%d 0\n", nvdll[k]);
    for (int j = 0; j < nvdll[k]; ++j) std::fprintf(f, "%d\n", nbdv[q++]);
  }
  long long nvel = 0;
  for (int k = 0; k < nbou; ++k) nvel += internal_barrier(ibtype[k]) ? 2 * nvell[k] : nvell[k];
  std::fprintf(f, "%d\n%lld\n", nbou, nvel);
  q = 0;
  for (int k = 0; k < nbou; ++k) {
    std::fprintf(f, "%d %d\n", nvell[k], ibtype[k]);
    const bool bar = external_barrier(ibtype[k]), ibar = internal_barrier(ibtype[k]);
    const bool pipe = pipe_barrier(ibtype[k]);
    if ((bar && (!barlanht || !barlancfsp)) ||
        (ibar && (!ibconn || !barinht || !barincfsb || !barincfsp)) ||
        (pipe && (!pipeht || !pipecoef || !pipediam))) {
      std::fclose(f);
      set_error("adc_fort14_write: segment %d is a barrier; its pairs, heights and "
                "coefficients are required", k + 1);
      return ADC_ERR_ARG;
    }
    for (int j = 0; j < nvell[k]; ++j, ++q) {
      if (bar)
        std::fprintf(f, "%d %.17g %.17g\n", nbvv[q], barlanht[q], barlancfsp[q]);
      else if (pipe)
        std::fprintf(f, "%d %d %.17g %.17g %.17g %.17g %.17g %.17g\n", nbvv[q], ibconn[q], barinht[q],
                     barincfsb[q], barincfsp[q], pipeht[q], pipecoef[q], pipediam[q]);
      else if (ibar)
        std::fprintf(f, "%d %d %.17g %.17g %.17g\n", nbvv[q], ibconn[q], barinht[q], barincfsb[q],
                     barincfsp[q]);
      else
        std::fprintf(f, "%d\n", nbvv[q]);
    }
  }
  if (std::fclose(f) != 0) { set_error("adc_fort14_write: write to %s failed", path); return ADC_ERR_ARG; }
  return ADC_OK;
}

extern "C" int adc_fort6x_header(const char *path, const char *rundes, const char *runid,
                                 const char *agrid, int ndsets, int np, double dt_out, int nspool,
                                 int irtype) {
  if (!path || np < 1 || (irtype != 1 && irtype != 2)) {
    set_error("adc_fort6x_header: bad arguments");
    return ADC_ERR_ARG;
  }
  FILE *f = std::fopen(path, "w");
  if (!f) { set_error("adc_fort6x_header: cannot open %s", path); return ADC_ERR_ARG; }
  // (1X,A32,2X,A24,2X,A24)
  std::fprintf(f, " %-32.32s  %-24.24s  %-24.24s\n", rundes ? rundes : "", runid ? runid : "",
               agrid ? agrid : "");
  // (1X,I10,1X,I10,1X,E15.7E3,1X,I8,1X,I5,1X,'FileFmtVersion: ',I10)
  char dt[32];
  fmt_e0(dt, dt_out, 15, 7);
  const int ffv = (1 << 20) | (2 << 10) | 0;   // VERSION_NUMBER(1, 2, 0), global.F:1295
  std::fprintf(f, " %10d %10d %s %8d %5d FileFmtVersion: %10d\n", ndsets, np, dt, nspool, irtype, ffv);
  if (std::fclose(f) != 0) { set_error("adc_fort6x_header: write failed"); return ADC_ERR_ARG; }
  return ADC_OK;
}

extern "C" int adc_fort6x_append(const char *path, double timeloc, int it, int np, const double *v1,
                                 const double *v2, const int *nodecode, double alternate) {
  if (!path || !v1 || np < 1) { set_error("adc_fort6x_append: bad arguments"); return ADC_ERR_ARG; }
  FILE *f = std::fopen(path, "a");
  if (!f) { set_error("adc_fort6x_append: cannot open %s", path); return ADC_ERR_ARG; }
  char a[32], b[32];
  fmt_1pe(a, timeloc, 20, 10);
  std::fprintf(f, "  %s     %10d\n", a, it);   // (2x,1pE20.10E3,5X,I10)
  for (int i = 0; i < np; ++i) {
    const bool dry = nodecode && nodecode[i] == 0;
    fmt_1pe(a, dry ? alternate : v1[i], 20, 10);
    if (v2) {
      fmt_1pe(b, dry ? alternate : v2[i], 20, 10);
      std::fprintf(f, "  %8d  %s%s\n", i + 1, a, b);   // (2x, i8, 2x, 1pE20.10E3, 1pE20.10E3)
    } else {
      std::fprintf(f, "  %8d  %s\n", i + 1, a);
    }
  }
  if (std::fclose(f) != 0) { set_error("adc_fort6x_append: write failed"); return ADC_ERR_ARG; }
  return ADC_OK;
}
