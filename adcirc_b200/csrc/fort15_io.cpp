// fort15_io.cpp -- the fort.15 model parameter file of a 2DDI run
// (READ_INPUT, read_input.F:949-4566): the positional records in the order
// read_input reads them, plus the two namelists whose values this path
// uses (&wetDryControl slim, read_input.F:242-246, 623; &metControl
// WindDragLimit, read_input.F:238, 485).
//
// Each READ(15,*) starts on a new record and takes its items from it,
// continuing on the next records if the record holds too few (Fortran
// list-directed input); what follows the last item of a record (the usual
// "! NAME" annotations) is skipped.  Character records (RUNDES, RUNID,
// constituent tags) are taken whole.  Angles the reference converts to
// radians on reading (FACE, EFA, FFACE, QNPH, ENPH, FACET) are returned in
// radians; everything else as read.
//
// Supported: IM = 0, 10 and 111111 (2DDI), NWS = 0 or +-8 without wave
// radiation stress or ice (the wind record of NWS = 8 is IREFYR, IREFMO,
// IREFDAY, IREFHR, StormNumber, BLAdj, read_input.F:2603-2621).  3D and
// baroclinic runs, other NWS values and station files (negative station
// counts) return ADC_ERR_UNSUPPORTED.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/adcgpu.h"

namespace adc {
void set_error(const char *fmt, ...);
}
using adc::set_error;

namespace {

const double kDeg2Rad = 3.141592653589793 / 180.0;   // constants.F90 DEG2RAD

struct Records {
  std::vector<std::string> rec;
  size_t next = 0;
  const char *path = "";

  bool open(const char *p) {
    path = p;
    FILE *f = std::fopen(p, "rb");
    if (!f) return false;
    std::string buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, n);
    std::fclose(f);
    size_t s = 0;
    while (s <= buf.size()) {
      size_t e = buf.find('\n', s);
      if (e == std::string::npos) e = buf.size();
      std::string line = buf.substr(s, e - s);
      if (!line.empty() && line.back() == '\r') line.pop_back();
      if (e == buf.size() && line.empty()) break;
      rec.push_back(line);
      s = e + 1;
    }
    return true;
  }
  int line() const { return (int)next; }   // 1-based number of the last record taken

  // a whole character record, trailing blanks removed, cut to `width`
  bool text(std::string &out, size_t width) {
    if (next >= rec.size()) return false;
    out = rec[next++].substr(0, width);
    while (!out.empty() && std::isspace((unsigned char)out.back())) out.pop_back();
    return true;
  }

  // the items of one list-directed READ: tokens separated by blanks or
  // commas, from the next record on
  bool items(size_t n, std::vector<std::string> &tok) {
    tok.clear();
    while (tok.size() < n) {
      if (next >= rec.size()) return false;
      const std::string &r = rec[next++];
      size_t k = 0;
      while (k < r.size() && tok.size() < n) {
        while (k < r.size() && (r[k] == ' ' || r[k] == '\t' || r[k] == ',')) ++k;
        if (k >= r.size() || r[k] == '!') break;
        size_t e = k;
        while (e < r.size() && r[e] != ' ' && r[e] != '\t' && r[e] != ',') ++e;
        tok.push_back(r.substr(k, e - k));
        k = e;
      }
    }
    return true;
  }
};

bool to_real(const std::string &s, double &v) {
  std::string t = s;
  for (char &c : t)
    if (c == 'd' || c == 'D') c = 'e';
  char *end = nullptr;
  errno = 0;
  v = std::strtod(t.c_str(), &end);
  return end != t.c_str() && *end == '\0' && errno != ERANGE;
}

bool to_int(const std::string &s, int &v) {
  char *end = nullptr;
  errno = 0;
  long x = std::strtol(s.c_str(), &end, 10);
  if (end == s.c_str() || *end != '\0' || errno == ERANGE || x < -2147483647L || x > 2147483647L)
    return false;
  v = (int)x;
  return true;
}

// A typed READ(15,*) of a mix of integers ('i') and reals ('r').
struct Item {
  char kind;
  void *dst;
};

struct Parser {
  Records r;
  std::vector<std::string> tok;
  int rc = ADC_OK;

  int fail(const char *what) {
    set_error("fort.15 %s: %s (record %d)", r.path, what, r.line());
    return rc = ADC_ERR_ARG;
  }
  int unsupported(const char *what) {
    set_error("fort.15 %s: %s (record %d)", r.path, what, r.line());
    return rc = ADC_ERR_UNSUPPORTED;
  }
  bool read(const char *what, std::initializer_list<Item> it) {
    if (rc) return false;
    if (!r.items(it.size(), tok)) {
      fail(what);
      return false;
    }
    size_t k = 0;
    for (const Item &x : it) {
      bool ok = x.kind == 'i' ? to_int(tok[k], *(int *)x.dst) : to_real(tok[k], *(double *)x.dst);
      if (!ok) {
        fail(what);
        return false;
      }
      ++k;
    }
    return true;
  }
  bool text(const char *what, std::string &s, size_t width) {
    if (rc) return false;
    if (!r.text(s, width)) {
      fail(what);
      return false;
    }
    return true;
  }
};

void put_tag(char *tags, int k, const std::string &s) {
  if (!tags) return;
  char *d = tags + 16 * (size_t)k;
  std::memset(d, 0, 16);
  size_t b = 0;
  while (b < s.size() && std::isspace((unsigned char)s[b])) ++b;
  std::strncpy(d, s.c_str() + b, 15);
}

// case-insensitive search for `name` = value inside namelist group `grp`
bool namelist_real(const Records &r, const char *grp, const char *name, double &v) {
  std::string all;
  for (const std::string &s : r.rec) {
    all += s;
    all += '\n';
  }
  std::string low = all;
  for (char &c : low) c = (char)std::tolower((unsigned char)c);
  std::string g = std::string("&") + grp;
  for (char &c : g) c = (char)std::tolower((unsigned char)c);
  size_t at = low.find(g);
  if (at == std::string::npos) return false;
  size_t end = low.find('/', at);
  if (end == std::string::npos) end = low.size();
  std::string nm = name;
  for (char &c : nm) c = (char)std::tolower((unsigned char)c);
  size_t p = at + g.size();
  while (true) {
    p = low.find(nm, p);
    if (p == std::string::npos || p >= end) return false;
    const bool left_ok = !(std::isalnum((unsigned char)low[p - 1]) || low[p - 1] == '_');
    size_t q = p + nm.size();
    while (q < end && std::isspace((unsigned char)low[q])) ++q;
    if (left_ok && q < end && low[q] == '=') {
      ++q;
      while (q < end && std::isspace((unsigned char)low[q])) ++q;
      size_t e = q;
      while (e < end && !std::isspace((unsigned char)low[e]) && low[e] != ',' && low[e] != '/') ++e;
      return to_real(all.substr(q, e - q), v);
    }
    p += nm.size();
  }
}

// the raw text of `name` = value inside namelist group `grp` (quotes and
// surrounding blanks removed), lower-cased
bool namelist_text(const Records &r, const char *grp, const char *name, std::string &out) {
  std::string all;
  for (const std::string &s : r.rec) {
    all += s;
    all += '\n';
  }
  for (char &c : all) c = (char)std::tolower((unsigned char)c);
  std::string g = std::string("&") + grp, nm = name;
  for (char &c : g) c = (char)std::tolower((unsigned char)c);
  for (char &c : nm) c = (char)std::tolower((unsigned char)c);
  size_t at = all.find(g);
  if (at == std::string::npos) return false;
  size_t end = all.find('/', at);
  if (end == std::string::npos) end = all.size();
  for (size_t p = all.find(nm, at + g.size()); p != std::string::npos && p < end;
       p = all.find(nm, p + nm.size())) {
    if (std::isalnum((unsigned char)all[p - 1]) || all[p - 1] == '_') continue;
    size_t q = p + nm.size();
    while (q < end && std::isspace((unsigned char)all[q])) ++q;
    if (q >= end || all[q] != '=') continue;
    ++q;
    while (q < end && std::isspace((unsigned char)all[q])) ++q;
    size_t e = q;
    if (q < end && (all[q] == '\'' || all[q] == '"')) {
      const char quote = all[q];
      e = all.find(quote, q + 1);
      if (e == std::string::npos || e > end) return false;
      out = all.substr(q + 1, e - q - 1);
      return true;
    }
    while (e < end && !std::isspace((unsigned char)all[e]) && all[e] != ',') ++e;
    out = all.substr(q, e - q);
    return true;
  }
  return false;
}

// a Fortran logical value: .true./.false./t/f
bool fortran_true(const std::string &v) {
  size_t k = 0;
  while (k < v.size() && v[k] == '.') ++k;
  return k < v.size() && v[k] == 't';
}

bool flux_code(int c) { return c == 2 || c == 12 || c == 22 || c == 52; }

}  // namespace

extern "C" int adc_fort15_read(const char *path, int neta, int nvel, const int *lbcodei,
                               adc_fort15_t *o, const adc_fort15_tables_t *t) {
  if (!path || !o || neta < 0 || nvel < 0 || (nvel > 0 && !lbcodei)) {
    set_error("adc_fort15_read: invalid arguments");
    return ADC_ERR_ARG;
  }
  Parser P;
  if (!P.r.open(path)) {
    set_error("fort.15: cannot open %s", path);
    return ADC_ERR_ARG;
  }
  std::memset(o, 0, sizeof(*o));
  o->slim = 1.0e9;                 // global.F:796
  o->wind_drag_limit = 0.0035;     // wind.F:122
  std::string s;
  if (!P.text("RUNDES", s, 80)) return P.rc;
  std::strncpy(o->rundes, s.c_str(), sizeof(o->rundes) - 1);
  if (!P.text("RUNID", s, 80)) return P.rc;
  std::strncpy(o->runid, s.c_str(), sizeof(o->runid) - 1);
  P.read("NFOVER", {{'i', &o->nfover}});
  P.read("NABOUT", {{'i', &o->nabout}});
  P.read("NSCREEN", {{'i', &o->nscreen}});
  P.read("IHOT", {{'i', &o->ihot}});
  P.read("ICS", {{'i', &o->ics}});
  if (!P.read("IM", {{'i', &o->im}})) return P.rc;
  if (o->im != 0 && o->im != 10 && o->im != 111111)
    return P.unsupported("IM other than 0, 10 or 111111 (3D, baroclinic or non-default 2DDI "
                         "formulations) is not read");
  P.read("NOLIBF", {{'i', &o->nolibf}});
  P.read("NOLIFA", {{'i', &o->nolifa}});
  P.read("NOLICA", {{'i', &o->nolica}});
  P.read("NOLICAT", {{'i', &o->nolicat}});
  if (!P.read("NWP", {{'i', &o->nwp}})) return P.rc;
  for (int k = 0; k < o->nwp; ++k)
    if (!P.text("AttrName", s, 80)) return P.rc;   // nodal attribute names (fort.13)
  P.read("NCOR", {{'i', &o->ncor}});
  P.read("NTIP", {{'i', &o->ntip}});
  if (!P.read("NWS", {{'i', &o->nws}})) return P.rc;
  if (o->nws != 0 && std::abs(o->nws) != 8)
    return P.unsupported("NWS other than 0 and 8 (and wave radiation stress or ice flags) "
                         "is not read");
  if (!P.read("NRAMP", {{'i', &o->nramp}})) return P.rc;
  P.read("G", {{'r', &o->g}});
  if (!P.read("TAU0", {{'r', &o->tau0}})) return P.rc;
  if (o->tau0 == -5.0) P.read("Tau0FullDomainMin/Max", {{'r', &o->tau0_min}, {'r', &o->tau0_max}});
  P.read("DTDP", {{'r', &o->dtdp}});
  P.read("STATIM", {{'r', &o->statim}});
  P.read("REFTIM", {{'r', &o->reftim}});
  if (std::abs(o->nws) == 8)
    P.read("IREFYR IREFMO IREFDAY IREFHR StormNumber BLAdj",
           {{'i', &o->irefyr}, {'i', &o->irefmo}, {'i', &o->irefday}, {'i', &o->irefhr},
            {'i', &o->storm_number}, {'r', &o->bladj}});
  P.read("RNDAY", {{'r', &o->rnday}});
  // DRAMP record by NRAMP (read_input.F:2893-2955): DRAMP, DRampExtFlux,
  // FluxSettlingTime, DRampIntFlux, DRampElev, DRampTip, DRampMete,
  // DRampWRad, DUnRampMete; the ramps a record does not give take DRAMP
  if (o->nramp < 0 || o->nramp > 8) return P.unsupported("NRAMP outside 0..8");
  const int nd = o->nramp <= 1 ? 1 : o->nramp + 1;
  double dr[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  {
    if (!P.r.items(nd, P.tok)) return P.fail("DRAMP record");
    for (int k = 0; k < nd; ++k)
      if (!to_real(P.tok[k], dr[k])) return P.fail("DRAMP record");
    for (int k = nd; k < 8; ++k)
      if (k != 2) dr[k] = dr[0];
  }
  o->dramp = dr[0];
  o->dramp_extflux = dr[1];
  o->flux_settling_time = dr[2];
  o->dramp_intflux = dr[3];
  o->dramp_elev = dr[4];
  o->dramp_tip = dr[5];
  o->dramp_mete = dr[6];
  o->dramp_wrad = dr[7];
  o->dunramp_mete = dr[8];
  P.read("A00 B00 C00", {{'r', &o->a00}, {'r', &o->b00}, {'r', &o->c00}});
  if (o->nolifa == 2)
    P.read("H0 NODEDRYMIN NODEWETMIN VELMIN",
           {{'r', &o->h0}, {'i', &o->nodedrymin}, {'i', &o->nodewetmin}, {'r', &o->velmin}});
  else
    P.read("H0", {{'r', &o->h0}});
  P.read("SLAM0 SFEA0", {{'r', &o->slam0}, {'r', &o->sfea0}});
  if (o->nolibf == 0) P.read("TAU", {{'r', &o->tau}});
  else if (o->nolibf == 1) P.read("CF", {{'r', &o->cf}});
  else if (o->nolibf == 2)
    P.read("CF HBREAK FTHETA FGAMMA", {{'r', &o->cf}, {'r', &o->hbreak}, {'r', &o->ftheta}, {'r', &o->fgamma}});
  else if (o->nolibf == 3)
    P.read("CF HBREAK FTHETA", {{'r', &o->cf}, {'r', &o->hbreak}, {'r', &o->ftheta}});
  else
    return P.unsupported("NOLIBF outside 0..3");
  if (o->im == 10) P.read("ESLM ESLC", {{'r', &o->eslm}, {'r', &o->eslc}});
  else P.read("ESLM", {{'r', &o->eslm}});
  P.read("CORI", {{'r', &o->cori}});
  if (!P.read("NTIF", {{'i', &o->ntif}})) return P.rc;
  for (int k = 0; k < o->ntif; ++k) {
    if (!P.text("TIPOTAG", s, 5)) return P.rc;
    put_tag(t ? t->tiptag : nullptr, k, s);
    double v[5];
    if (!P.read("TPK AMIGT ETRF FFT FACET", {{'r', v}, {'r', v + 1}, {'r', v + 2}, {'r', v + 3}, {'r', v + 4}}))
      return P.rc;
    if (t && t->tpk) {
      t->tpk[k] = v[0];
      t->amigt[k] = v[1];
      t->etrf[k] = v[2];
      t->fft[k] = v[3];
      t->facet[k] = v[4] * kDeg2Rad;
    }
  }
  if (!P.read("NBFR", {{'i', &o->nbfr}})) return P.rc;
  for (int k = 0; k < o->nbfr; ++k) {
    if (!P.text("BOUNTAG", s, 5)) return P.rc;
    put_tag(t ? t->bountag : nullptr, k, s);
    double v[3];
    if (!P.read("AMIG FF FACE", {{'r', v}, {'r', v + 1}, {'r', v + 2}})) return P.rc;
    if (t && t->amig) {
      t->amig[k] = v[0];
      t->ff[k] = v[1];
      t->face[k] = v[2] * kDeg2Rad;
    }
  }
  for (int k = 0; k < o->nbfr; ++k) {
    if (!P.text("ALPHAE", s, 10)) return P.rc;
    for (int j = 0; j < neta; ++j) {
      double a, p;
      if (!P.read("EMO EFA", {{'r', &a}, {'r', &p}})) return P.rc;
      if (t && t->emo) {
        t->emo[k + (size_t)o->nbfr * j] = a;            // EMO(NBFR,NETA)
        t->efa[k + (size_t)o->nbfr * j] = p * kDeg2Rad;
      }
    }
  }
  P.read("ANGINN", {{'r', &o->anginn}});
  bool nfluxf = false;
  for (int j = 0; j < nvel; ++j) nfluxf = nfluxf || flux_code(lbcodei[j]) || lbcodei[j] == 32;
  if (nfluxf) {
    if (!P.read("NFFR", {{'i', &o->nffr}})) return P.rc;
    if (o->nffr > 0) {
      for (int k = 0; k < o->nffr; ++k) {
        if (!P.text("FBOUNTAG", s, 5)) return P.rc;
        put_tag(t ? t->fbountag : nullptr, k, s);
        double v[3];
        if (!P.read("FAMIG FFF FFACE", {{'r', v}, {'r', v + 1}, {'r', v + 2}})) return P.rc;
        if (t && t->famig) {
          t->famig[k] = v[0];
          t->fff[k] = v[1];
          t->fface[k] = v[2] * kDeg2Rad;
        }
      }
      for (int k = 0; k < o->nffr; ++k) {
        if (!P.text("ALPHA", s, 10)) return P.rc;
        for (int j = 0; j < nvel; ++j) {
          const size_t q = k + (size_t)o->nffr * j;       // QNAM(NFFR,NVEL)
          if (flux_code(lbcodei[j])) {
            double a, p;
            if (!P.read("QNAM QNPH", {{'r', &a}, {'r', &p}})) return P.rc;
            if (t && t->qnam) {
              t->qnam[q] = a;
              t->qnph[q] = p * kDeg2Rad;
            }
          } else if (lbcodei[j] == 32) {
            double a, p, e, f;
            if (!P.read("QNAM QNPH ENAM ENPH", {{'r', &a}, {'r', &p}, {'r', &e}, {'r', &f}})) return P.rc;
            if (t && t->qnam) {
              t->qnam[q] = a;
              t->qnph[q] = p * kDeg2Rad;
              if (t->enam) {
                t->enam[q] = e;
                t->enph[q] = f * kDeg2Rad;
              }
            }
          }
        }
      }
    }
  }
  // output controls and stations (read_input.F:3606-4360)
  auto out4 = [&](const char *what, adc_output_spec_t &sp) {
    return P.read(what, {{'i', &sp.nout}, {'r', &sp.touts}, {'r', &sp.toutf}, {'i', &sp.nspool}});
  };
  auto stations = [&](const char *what, int &nsta, double *xs, double *ys) {
    if (!P.read(what, {{'i', &nsta}})) return false;
    if (nsta < 0) {
      P.unsupported("station coordinates in an external .151 file are not read");
      return false;
    }
    for (int k = 0; k < nsta; ++k) {
      double x, y;
      if (!P.read("station coordinates", {{'r', &x}, {'r', &y}})) return false;
      if (xs) xs[k] = x;
      if (ys) ys[k] = y;
    }
    return true;
  };
  if (!out4("NOUTE TOUTSE TOUTFE NSPOOLE", o->oute)) return P.rc;
  if (!stations("NSTAE", o->nstae, t ? t->xel : nullptr, t ? t->yel : nullptr)) return P.rc;
  if (!out4("NOUTV TOUTSV TOUTFV NSPOOLV", o->outv)) return P.rc;
  if (!stations("NSTAV", o->nstav, t ? t->xev : nullptr, t ? t->yev : nullptr)) return P.rc;
  if (o->im == 10) {
    if (!out4("NOUTC TOUTSC TOUTFC NSPOOLC", o->outc)) return P.rc;
    if (!stations("NSTAC", o->nstac, nullptr, nullptr)) return P.rc;
  }
  if (o->nws != 0) {
    if (!out4("NOUTM TOUTSM TOUTFM NSPOOLM", o->outm)) return P.rc;
    if (!stations("NSTAM", o->nstam, t ? t->xem : nullptr, t ? t->yem : nullptr)) return P.rc;
  }
  if (!out4("NOUTGE TOUTSGE TOUTFGE NSPOOLGE", o->outge)) return P.rc;
  if (!out4("NOUTGV TOUTSGV TOUTFGV NSPOOLGV", o->outgv)) return P.rc;
  if (o->im == 10 && !out4("NOUTGC TOUTSGC TOUTFGC NSPOOLGC", o->outgc)) return P.rc;
  if (o->nws != 0 && !out4("NOUTGW TOUTSGW TOUTFGW NSPOOLGW", o->outgw)) return P.rc;
  // harmonic analysis (read_input.F:4420-4507)
  if (!P.read("NFREQ", {{'i', &o->nfreq}})) return P.rc;
  if (o->nfreq < 0) return P.fail("NFREQ < 0");
  for (int k = 0; k < o->nfreq; ++k) {
    if (!P.text("NAMEFR", s, 10)) return P.rc;
    put_tag(t ? t->namefr : nullptr, k, s);
    double v[3];
    if (!P.read("HAFREQ HAFF HAFACE", {{'r', v}, {'r', v + 1}, {'r', v + 2}})) return P.rc;
    if (t && t->hafreq) {
      t->hafreq[k] = v[0];
      t->haff[k] = v[1];
      t->haface[k] = v[2];
    }
  }
  P.read("THAS THAF NHAINC FMV", {{'r', &o->thas}, {'r', &o->thaf}, {'i', &o->nhainc}, {'r', &o->fmv}});
  P.read("NHASE NHASV NHAGE NHAGV", {{'i', &o->nhase}, {'i', &o->nhasv}, {'i', &o->nhage}, {'i', &o->nhagv}});
  P.read("NHSTAR NHSINC", {{'i', &o->nhstar}, {'i', &o->nhsinc}});
  P.read("ITITER ISLDIA CONVCR ITMAX",
         {{'i', &o->ititer}, {'i', &o->isldia}, {'r', &o->convcr}, {'i', &o->itmax}});
  if (P.rc) return P.rc;
  double v;
  if (namelist_real(P.r, "wetDryControl", "slim", v)) {
    o->slim = v;
    o->has_slim = 1;
  }
  if (namelist_real(P.r, "metControl", "WindDragLimit", v)) {
    o->wind_drag_limit = v;
    o->has_wind_drag_limit = 1;
  }
  // &nws08Control (nws08.F90:318-413): defaults, then what the group sets
  o->windspeed_averaging_minute = 1;
  o->wind_multiplier = 1.0;
  {
    std::string t;
    const bool any = namelist_text(P.r, "nws08Control", "vortexModel", t) |
                     namelist_text(P.r, "nws08Control", "backgroundWindModel", t) |
                     namelist_text(P.r, "nws08Control", "BCalc", t) |
                     namelist_text(P.r, "nws08Control", "windspeed_averaging_minute", t) |
                     namelist_text(P.r, "nws08Control", "WindMultiplier", t) |
                     namelist_text(P.r, "nws08Control", "useInflow", t) |
                     namelist_text(P.r, "nws08Control", "thetaLatDep", t);
    o->has_nws08 = any ? 1 : 0;
    struct Want {
      const char *name, *value;
    };
    for (const Want &w : {Want{"vortexModel", "holland"},
                          Want{"backgroundWindModel", "radialvelocityweighted"},
                          Want{"BCalc", "limited"}})
      if (namelist_text(P.r, "nws08Control", w.name, t) && t != w.value) {
        set_error("fort.15 %s: &nws08Control %s = '%s' is not implemented (only '%s')", path,
                  w.name, t.c_str(), w.value);
        return ADC_ERR_UNSUPPORTED;
      }
    for (const char *flag : {"useInflow", "thetaLatDep"})
      if (namelist_text(P.r, "nws08Control", flag, t) && fortran_true(t)) {
        set_error("fort.15 %s: &nws08Control %s = .true. is not implemented", path, flag);
        return ADC_ERR_UNSUPPORTED;
      }
    if (namelist_real(P.r, "nws08Control", "WindMultiplier", v)) o->wind_multiplier = v;
    if (namelist_real(P.r, "nws08Control", "windspeed_averaging_minute", v))
      o->windspeed_averaging_minute = (int)v;
  }
  return ADC_OK;
}

// The writer: the same records in the same order, every real to 17
// significant digits (so a read gives back the same doubles; angles are
// written in degrees as the file holds them), each record annotated with
// its variable names after "!".
namespace {
struct Writer {
  FILE *f;
  void rec(const char *names, std::initializer_list<Item> it) {
    bool first = true;
    for (const Item &x : it) {
      if (!first) std::fputc(' ', f);
      first = false;
      if (x.kind == 'i') std::fprintf(f, "%d", *(const int *)x.dst);
      else std::fprintf(f, "%.17g", *(const double *)x.dst);
    }
    std::fprintf(f, "   ! %s\n", names);
  }
  void text(const char *s) { std::fprintf(f, "%s\n", s); }
};

std::string tag_of(const char *tags, int k, const char *dflt) {
  if (!tags) return dflt;
  std::string s(tags + 16 * (size_t)k, strnlen(tags + 16 * (size_t)k, 16));
  return s.empty() ? std::string(dflt) : s;
}
}  // namespace

extern "C" int adc_fort15_write(const char *path, const adc_fort15_t *o, int neta, int nvel,
                                const int *lbcodei, const adc_fort15_tables_t *t) {
  if (!path || !o || !t || neta < 0 || nvel < 0 || (nvel > 0 && !lbcodei) ||
      (o->nbfr > 0 && (!t->amig || !t->ff || !t->face || (neta > 0 && (!t->emo || !t->efa)))) ||
      (o->ntif > 0 && (!t->tpk || !t->amigt || !t->etrf || !t->fft || !t->facet)) ||
      (o->nffr > 0 && (!t->famig || !t->fff || !t->fface || !t->qnam || !t->qnph)) ||
      (o->nfreq > 0 && (!t->hafreq || !t->haff || !t->haface)) || o->nstae < 0 || o->nstav < 0 ||
      o->nstac < 0 || o->nstam < 0 || (o->nstae > 0 && (!t->xel || !t->yel)) ||
      (o->nstav > 0 && (!t->xev || !t->yev)) || (o->nstam > 0 && (!t->xem || !t->yem))) {
    set_error("adc_fort15_write: invalid arguments");
    return ADC_ERR_ARG;
  }
  if (o->nstac > 0) {
    set_error("adc_fort15_write: concentration stations are not written");
    return ADC_ERR_UNSUPPORTED;
  }
  FILE *f = std::fopen(path, "w");
  if (!f) {
    set_error("fort.15: cannot create %s", path);
    return ADC_ERR_ARG;
  }
  Writer w{f};
  const double r2d = 1.0 / kDeg2Rad;
  char rundes[89], runid[89];
  std::snprintf(rundes, sizeof(rundes), "%.80s", o->rundes);
  std::snprintf(runid, sizeof(runid), "%.80s", o->runid);
  w.text(rundes);
  w.text(runid);
  w.rec("NFOVER", {{'i', (void *)&o->nfover}});
  w.rec("NABOUT", {{'i', (void *)&o->nabout}});
  w.rec("NSCREEN", {{'i', (void *)&o->nscreen}});
  w.rec("IHOT", {{'i', (void *)&o->ihot}});
  w.rec("ICS", {{'i', (void *)&o->ics}});
  w.rec("IM", {{'i', (void *)&o->im}});
  w.rec("NOLIBF", {{'i', (void *)&o->nolibf}});
  w.rec("NOLIFA", {{'i', (void *)&o->nolifa}});
  w.rec("NOLICA", {{'i', (void *)&o->nolica}});
  w.rec("NOLICAT", {{'i', (void *)&o->nolicat}});
  const int nwp = 0;   // no fort.13 attributes
  w.rec("NWP", {{'i', (void *)&nwp}});
  w.rec("NCOR", {{'i', (void *)&o->ncor}});
  w.rec("NTIP", {{'i', (void *)&o->ntip}});
  w.rec("NWS", {{'i', (void *)&o->nws}});
  w.rec("NRAMP", {{'i', (void *)&o->nramp}});
  w.rec("G", {{'r', (void *)&o->g}});
  w.rec("TAU0", {{'r', (void *)&o->tau0}});
  if (o->tau0 == -5.0)
    w.rec("Tau0FullDomainMin, Tau0FullDomainMax", {{'r', (void *)&o->tau0_min}, {'r', (void *)&o->tau0_max}});
  w.rec("DTDP", {{'r', (void *)&o->dtdp}});
  w.rec("STATIM", {{'r', (void *)&o->statim}});
  w.rec("REFTIM", {{'r', (void *)&o->reftim}});
  if (std::abs(o->nws) == 8)
    w.rec("IREFYR, IREFMO, IREFDAY, IREFHR, StormNumber, BLAdj",
          {{'i', (void *)&o->irefyr}, {'i', (void *)&o->irefmo}, {'i', (void *)&o->irefday},
           {'i', (void *)&o->irefhr}, {'i', (void *)&o->storm_number}, {'r', (void *)&o->bladj}});
  w.rec("RNDAY", {{'r', (void *)&o->rnday}});
  const double dr[9] = {o->dramp, o->dramp_extflux, o->flux_settling_time, o->dramp_intflux,
                        o->dramp_elev, o->dramp_tip, o->dramp_mete, o->dramp_wrad, o->dunramp_mete};
  const int nd = o->nramp <= 1 ? 1 : std::min(o->nramp + 1, 9);
  for (int k = 0; k < nd; ++k) std::fprintf(f, k ? " %.17g" : "%.17g", dr[k]);
  std::fprintf(f, "   ! DRAMP record (NRAMP = %d)\n", o->nramp);
  w.rec("A00, B00, C00", {{'r', (void *)&o->a00}, {'r', (void *)&o->b00}, {'r', (void *)&o->c00}});
  if (o->nolifa == 2)
    w.rec("H0, NODEDRYMIN, NODEWETMIN, VELMIN",
          {{'r', (void *)&o->h0}, {'i', (void *)&o->nodedrymin}, {'i', (void *)&o->nodewetmin},
           {'r', (void *)&o->velmin}});
  else
    w.rec("H0", {{'r', (void *)&o->h0}});
  w.rec("SLAM0, SFEA0", {{'r', (void *)&o->slam0}, {'r', (void *)&o->sfea0}});
  if (o->nolibf == 0) w.rec("TAU", {{'r', (void *)&o->tau}});
  else if (o->nolibf == 1) w.rec("CF", {{'r', (void *)&o->cf}});
  else if (o->nolibf == 2)
    w.rec("CF, HBREAK, FTHETA, FGAMMA", {{'r', (void *)&o->cf}, {'r', (void *)&o->hbreak},
                                         {'r', (void *)&o->ftheta}, {'r', (void *)&o->fgamma}});
  else
    w.rec("CF, HBREAK, FTHETA", {{'r', (void *)&o->cf}, {'r', (void *)&o->hbreak}, {'r', (void *)&o->ftheta}});
  if (o->im == 10) w.rec("ESLM, ESLC", {{'r', (void *)&o->eslm}, {'r', (void *)&o->eslc}});
  else w.rec("ESLM", {{'r', (void *)&o->eslm}});
  w.rec("CORI", {{'r', (void *)&o->cori}});
  w.rec("NTIF", {{'i', (void *)&o->ntif}});
  for (int k = 0; k < o->ntif; ++k) {
    w.text(tag_of(t->tiptag, k, "TIP").c_str());
    const double facet = t->facet[k] * r2d;
    w.rec("TPK, AMIGT, ETRF, FFT, FACET", {{'r', &t->tpk[k]}, {'r', &t->amigt[k]}, {'r', &t->etrf[k]},
                                            {'r', &t->fft[k]}, {'r', (void *)&facet}});
  }
  w.rec("NBFR", {{'i', (void *)&o->nbfr}});
  for (int k = 0; k < o->nbfr; ++k) {
    w.text(tag_of(t->bountag, k, "CONST").c_str());
    const double face = t->face[k] * r2d;
    w.rec("AMIG, FF, FACE", {{'r', &t->amig[k]}, {'r', &t->ff[k]}, {'r', (void *)&face}});
  }
  for (int k = 0; k < o->nbfr; ++k) {
    w.text(tag_of(t->bountag, k, "CONST").c_str());
    for (int j = 0; j < neta; ++j) {
      const size_t q = k + (size_t)o->nbfr * j;
      const double efa = t->efa[q] * r2d;
      std::fprintf(f, "%.17g %.17g\n", t->emo[q], efa);
    }
  }
  w.rec("ANGINN", {{'r', (void *)&o->anginn}});
  bool nfluxf = false;
  for (int j = 0; j < nvel; ++j) nfluxf = nfluxf || flux_code(lbcodei[j]) || lbcodei[j] == 32;
  if (nfluxf) {
    w.rec("NFFR", {{'i', (void *)&o->nffr}});
    for (int k = 0; k < o->nffr; ++k) {
      w.text(tag_of(t->fbountag, k, "FLUX").c_str());
      const double fface = t->fface[k] * r2d;
      w.rec("FAMIG, FFF, FFACE", {{'r', &t->famig[k]}, {'r', &t->fff[k]}, {'r', (void *)&fface}});
    }
    for (int k = 0; k < o->nffr; ++k) {
      w.text(tag_of(t->fbountag, k, "FLUX").c_str());
      for (int j = 0; j < nvel; ++j) {
        const size_t q = k + (size_t)o->nffr * j;
        if (flux_code(lbcodei[j])) {
          std::fprintf(f, "%.17g %.17g\n", t->qnam[q], t->qnph[q] * r2d);
        } else if (lbcodei[j] == 32) {
          const double ea = t->enam ? t->enam[q] : 0.0, ep = t->enph ? t->enph[q] * r2d : 0.0;
          std::fprintf(f, "%.17g %.17g %.17g %.17g\n", t->qnam[q], t->qnph[q] * r2d, ea, ep);
        }
      }
    }
  }
  auto out4 = [&](const char *names, const adc_output_spec_t &sp) {
    w.rec(names, {{'i', (void *)&sp.nout}, {'r', (void *)&sp.touts}, {'r', (void *)&sp.toutf},
                  {'i', (void *)&sp.nspool}});
  };
  auto stations = [&](const char *name, int n, const double *xs, const double *ys) {
    w.rec(name, {{'i', (void *)&n}});
    for (int k = 0; k < n; ++k) std::fprintf(f, "%.17g %.17g\n", xs[k], ys[k]);
  };
  out4("NOUTE, TOUTSE, TOUTFE, NSPOOLE", o->oute);
  stations("NSTAE", o->nstae, t->xel, t->yel);
  out4("NOUTV, TOUTSV, TOUTFV, NSPOOLV", o->outv);
  stations("NSTAV", o->nstav, t->xev, t->yev);
  if (o->im == 10) {
    out4("NOUTC, TOUTSC, TOUTFC, NSPOOLC", o->outc);
    stations("NSTAC", 0, nullptr, nullptr);
  }
  if (o->nws != 0) {
    out4("NOUTM, TOUTSM, TOUTFM, NSPOOLM", o->outm);
    stations("NSTAM", o->nstam, t->xem, t->yem);
  }
  out4("NOUTGE, TOUTSGE, TOUTFGE, NSPOOLGE", o->outge);
  out4("NOUTGV, TOUTSGV, TOUTFGV, NSPOOLGV", o->outgv);
  if (o->im == 10) out4("NOUTGC, TOUTSGC, TOUTFGC, NSPOOLGC", o->outgc);
  if (o->nws != 0) out4("NOUTGW, TOUTSGW, TOUTFGW, NSPOOLGW", o->outgw);
  w.rec("NFREQ", {{'i', (void *)&o->nfreq}});
  for (int k = 0; k < o->nfreq; ++k) {
    w.text(tag_of(t->namefr, k, "HA").c_str());
    w.rec("HAFREQ, HAFF, HAFACE", {{'r', &t->hafreq[k]}, {'r', &t->haff[k]}, {'r', &t->haface[k]}});
  }
  w.rec("THAS, THAF, NHAINC, FMV", {{'r', (void *)&o->thas}, {'r', (void *)&o->thaf},
                                    {'i', (void *)&o->nhainc}, {'r', (void *)&o->fmv}});
  w.rec("NHASE, NHASV, NHAGE, NHAGV", {{'i', (void *)&o->nhase}, {'i', (void *)&o->nhasv},
                                       {'i', (void *)&o->nhage}, {'i', (void *)&o->nhagv}});
  w.rec("NHSTAR, NHSINC", {{'i', (void *)&o->nhstar}, {'i', (void *)&o->nhsinc}});
  w.rec("ITITER, ISLDIA, CONVCR, ITMAX", {{'i', (void *)&o->ititer}, {'i', (void *)&o->isldia},
                                          {'r', (void *)&o->convcr}, {'i', (void *)&o->itmax}});
  if (o->has_slim) std::fprintf(f, "&wetDryControl slim=%.17g /\n", o->slim);
  if (o->has_wind_drag_limit) std::fprintf(f, "&metControl WindDragLimit=%.17g /\n", o->wind_drag_limit);
  if (o->has_nws08)
    std::fprintf(f, "&nws08Control windspeed_averaging_minute=%d, WindMultiplier=%.17g /\n",
                 o->windspeed_averaging_minute, o->wind_multiplier);
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  if (!ok) {
    set_error("fort.15: write error on %s", path);
    return ADC_ERR_ARG;
  }
  return ADC_OK;
}

// ---------------------------------------------------------------------------
// fort.19 / fort.20: non-periodic elevation and normal-flux boundary series.
// The interval, then records as the reference's READ(19,*)/READ(20,*) take
// them (cstart.F:207-216, 227-256; gwce.F:1664-1666; timestep.F:886-897).

namespace {

// Reads the interval line and every full record of `per` values; a record
// takes `items(j)` values for its j-th READ.  Returns the record count or a
// negative status.
template <class ItemsOf, class Store>
int read_series(const char *path, const char *which, int nreads, ItemsOf items, Store store,
                double *interval) {
  Records r;
  if (!r.open(path)) {
    set_error("%s %s: cannot open", which, path);
    return ADC_ERR_ARG;
  }
  std::vector<std::string> tok;
  double inc = 0.0;
  if (!r.items(1, tok) || !to_real(tok[0], inc) || !(inc > 0.0)) {
    set_error("%s %s: the first record must hold a positive time increment", which, path);
    return ADC_ERR_ARG;
  }
  *interval = inc;
  int nrec = 0;
  for (;;) {
    // the end of the file (blank records aside) ends the series
    size_t q0 = r.next;
    while (q0 < r.rec.size() && r.rec[q0].find_first_not_of(" \t") == std::string::npos) ++q0;
    if (q0 >= r.rec.size()) break;
    std::vector<double> vals;
    for (int j = 0; j < nreads; ++j) {
      const int k = items(j);
      if (k == 0) continue;
      if (!r.items((size_t)k, tok)) {
        set_error("%s %s: record %d is incomplete", which, path, nrec + 1);
        return ADC_ERR_ARG;
      }
      for (int q = 0; q < k; ++q) {
        double v;
        if (!to_real(tok[q], v)) {
          set_error("%s %s: '%s' is not a number (line %d)", which, path, tok[q].c_str(), r.line());
          return ADC_ERR_ARG;
        }
        vals.push_back(v);
      }
    }
    store(nrec, vals);
    ++nrec;
  }
  return nrec;
}

}  // namespace

extern "C" int adc_fort19_read(const char *path, int neta, int *nrec, double *interval,
                               double *esbin) {
  if (!path || neta < 1 || !nrec || !interval) {
    set_error("adc_fort19_read: a path, NETA >= 1 and the count outputs are required");
    return ADC_ERR_ARG;
  }
  const int cap = esbin ? *nrec : 0;
  int n = read_series(
      path, "fort.19", neta, [](int) { return 1; },
      [&](int k, const std::vector<double> &v) {
        if (esbin && k < cap)
          for (int j = 0; j < neta; ++j) esbin[(size_t)k * neta + j] = v[j];
      },
      interval);
  if (n < 0) return n;
  if (n < 2) {
    set_error("adc_fort19_read %s: fewer than two records of %d values", path, neta);
    return ADC_ERR_ARG;
  }
  *nrec = esbin ? (n < cap ? n : cap) : n;
  return ADC_OK;
}

extern "C" int adc_fort20_read(const char *path, int nvel, const int *lbcodei, int *nrec,
                               double *interval, double *qnin, double *enin) {
  if (!path || nvel < 1 || !lbcodei || !nrec || !interval) {
    set_error("adc_fort20_read: a path, NVEL >= 1, LBCODEI and the count outputs are required");
    return ADC_ERR_ARG;
  }
  auto items = [&](int j) {
    const int lb = lbcodei[j];
    return (lb == 2 || lb == 12 || lb == 22) ? 1 : lb == 32 ? 2 : 0;
  };
  int any = 0;
  for (int j = 0; j < nvel; ++j) any |= items(j);
  if (!any) {
    set_error("adc_fort20_read: no boundary entry of code 2, 12, 22 or 32 takes a fort.20 record");
    return ADC_ERR_ARG;
  }
  const int cap = qnin ? *nrec : 0;
  int n = read_series(
      path, "fort.20", nvel, items,
      [&](int k, const std::vector<double> &v) {
        if (!qnin || k >= cap) return;
        size_t q = 0;
        for (int j = 0; j < nvel; ++j) {
          const size_t o = (size_t)k * nvel + j;
          const int m = items(j);
          qnin[o] = m ? v[q] : 0.0;   // ICS = 1: the flux is not rotated
          if (enin) enin[o] = m == 2 ? v[q + 1] : 0.0;
          q += m;
        }
      },
      interval);
  if (n < 0) return n;
  if (n < 2) {
    set_error("adc_fort20_read %s: fewer than two records", path);
    return ADC_ERR_ARG;
  }
  *nrec = qnin ? (n < cap ? n : cap) : n;
  return ADC_OK;
}
