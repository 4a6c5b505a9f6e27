// fort22_io.cpp -- the NWS = 8 storm track file (fort.22, ATCF best-track /
// objective-aid lines) as readBestTrackData reads it (nws08.F90:884-1098),
// turned into the track fixes of adc_vortex_t.
//
// Each line is read with the fixed columns of the reference's FORMAT 228
// (nws08.F90:962): year, month, day, hour at columns 9-18, the line type at
// 25-28 (BEST, OFCL or CALM), the forecast hour at 31-33, latitude and its
// hemisphere at 35-39, longitude and E/W at 42-46, Vmax (kt) at 49-51,
// central pressure (mb) at 54-57, the radius of the last closed isobar (nm)
// at 105-107 and the radius to maximum winds (nm) at 110-112.  Integer
// fields follow Fortran formatted input: blanks are ignored and a blank
// field reads 0.
//
// Repeated times are dropped as the reference drops them; times are seconds
// since the wind reference time (TIMECONV, global.F:1556-1583); BEST lines
// and OFCL/CALM lines of forecast hour 0 take their date, later forecast
// lines the previous time plus the change of the forecast increment.  Units
// are converted as nws08.F90:1055-1066 converts them, and the translation
// velocity of each fix comes from the move since the previous fix (uvtrans,
// wind/vortex.F:1174-1200, haversine distances), the first fix taking the
// second's.  CALM lines become fixes with a negative central pressure,
// which the vortex step treats as the reference treats a CALM neighbour
// (zero wind, background pressure; GetHollandStormData nws08.F90:858-872).
//
// The centre goes into mesh coordinates with the CPP projection about
// (SLAM0, SFEA0) that INVCP inverts for ICS = 1 meshes (mesh.F:3409-3418):
// x = R cos(SFEA0) (lon - SLAM0), y = R lat, angles in radians.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/adcgpu.h"

namespace adc {
void set_error(const char *fmt, ...);
}
using adc::set_error;

namespace {

const double kPi = 3.141592653589793;          // constants.F90 PI
const double kDeg2Rad = kPi / 180.0;           // constants.F90 DEG2RAD
const double kRearth = 6378206.4;              // constants.F90 Rearth
const double kNm2Km = 1.852000003180799;       // nws08.F90:1063-1064
const double kKt2Ms = 0.51444444;              // nws08.F90:1065

// TIMECONV (global.F:1556-1583): seconds since the start of the year, with
// the reference's leap-year test (divisible by 4).
double timeconv(int iyr, int imo, int iday, int ihr, int imin, double sec) {
  double t = (iday - 1) * 86400.0 + ihr * 3600.0 + imin * 60.0 + sec;
  // days of March..October, added from April..November on
  static const int mdays[8] = {31, 30, 31, 30, 31, 31, 30, 31};
  if (imo >= 2) t += 31 * 86400.0;
  const bool leap = (iyr / 4) * 4 == iyr;
  if (imo >= 3) t += (leap ? 29 : 28) * 86400.0;
  for (int m = 4; m <= 11 && m <= imo; ++m) t += mdays[m - 4] * 86400.0;
  if (imo == 12) t += 30 * 86400.0;
  if (imo > 12) t += 30 * 86400.0;   // the reference logs an error and goes on
  return t;
}

// sphericalDistance (global.F:830-848): haversine distance, dx and dy in
// radians, latitudes in degrees.
double spherical_distance(double dx, double dy, double y1, double y2) {
  const double sy = std::sin(dy / 2.0), sx = std::sin(dx / 2.0);
  return kRearth * (2.0 * std::asin(std::sqrt(sy * sy + std::cos(y1 * kDeg2Rad) *
                                                            std::cos(y2 * kDeg2Rad) * sx * sx)));
}

// A formatted integer field (columns a..b, 1-based, inclusive).
bool int_field(const std::string &line, int a, int b, int &v) {
  std::string digits;
  for (int c = a; c <= b; ++c) {
    const char ch = c - 1 < (int)line.size() ? line[c - 1] : ' ';
    if (ch == ' ' || ch == '\t') continue;
    digits.push_back(ch);
  }
  if (digits.empty()) {
    v = 0;
    return true;
  }
  size_t k = 0;
  bool neg = false;
  if (digits[0] == '+' || digits[0] == '-') {
    neg = digits[0] == '-';
    k = 1;
  }
  if (k >= digits.size()) return false;
  long x = 0;
  for (; k < digits.size(); ++k) {
    if (digits[k] < '0' || digits[k] > '9') return false;
    x = x * 10 + (digits[k] - '0');
    if (x > 2147483647L) return false;
  }
  v = (int)(neg ? -x : x);
  return true;
}

std::string text_field(const std::string &line, int a, int b) {
  std::string s;
  for (int c = a; c <= b; ++c) s.push_back(c - 1 < (int)line.size() ? line[c - 1] : ' ');
  while (!s.empty() && s.back() == ' ') s.pop_back();
  while (!s.empty() && s.front() == ' ') s.erase(s.begin());
  return s;
}

struct Line {
  int yr, mo, dy, hr, inc, lat, lon, spd, cp, rrp, rmw;
  char ns, ew;
  std::string type;
};

}  // namespace

extern "C" int adc_fort22_read(const char *path, const adc_fort22_opts_t *o, int *nfix,
                               adc_vortex_fix_t *fix) {
  if (!path || !o || !nfix) {
    set_error("adc_fort22_read: a path, the options and the count output are required");
    return ADC_ERR_ARG;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    set_error("fort.22 %s: cannot open", path);
    return ADC_ERR_ARG;
  }
  std::string buf;
  char tmp[1 << 16];
  size_t nr;
  while ((nr = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.append(tmp, nr);
  std::fclose(f);

  const double wind_ref = timeconv(o->irefyr, o->irefmo, o->irefday, o->irefhr, 0, 0.0);
  std::vector<Line> kept;
  std::vector<double> cast_time, fcst_inc;
  size_t s = 0;
  int lineno = 0;
  while (s < buf.size()) {
    size_t e = buf.find('\n', s);
    if (e == std::string::npos) e = buf.size();
    std::string line = buf.substr(s, e - s);
    s = e + 1;
    ++lineno;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.find_first_not_of(" \t") == std::string::npos) continue;
    Line L;
    const bool ok = int_field(line, 9, 12, L.yr) && int_field(line, 13, 14, L.mo) &&
                    int_field(line, 15, 16, L.dy) && int_field(line, 17, 18, L.hr) &&
                    int_field(line, 31, 33, L.inc) && int_field(line, 35, 38, L.lat) &&
                    int_field(line, 42, 45, L.lon) && int_field(line, 49, 51, L.spd) &&
                    int_field(line, 54, 57, L.cp) && int_field(line, 105, 107, L.rrp) &&
                    int_field(line, 110, 112, L.rmw);
    if (!ok) {
      set_error("fort.22 %s: line %d does not hold the best-track fields", path, lineno);
      return ADC_ERR_ARG;
    }
    L.type = text_field(line, 25, 28);
    L.ns = line.size() >= 39 ? line[38] : ' ';
    L.ew = line.size() >= 46 ? line[45] : ' ';
    const Line *prev = kept.empty() ? nullptr : &kept.back();
    const bool same_time = prev && L.yr == prev->yr && L.mo == prev->mo && L.dy == prev->dy &&
                           L.hr == prev->hr;
    double ct, fi;
    if (L.type == "BEST") {   // nws08.F90:978-1001
      if (same_time) continue;
      ct = timeconv(L.yr, L.mo, L.dy, L.hr, 0, 0.0) - wind_ref;
      fi = (double)L.inc;
    } else if (L.type == "OFCL" || L.type == "CALM") {   // nws08.F90:1003-1046
      if (prev && ((L.inc == 0 && same_time) || (L.inc != 0 && L.inc == prev->inc))) continue;
      fi = (double)L.inc;
      if (L.inc == 0) {
        ct = timeconv(L.yr, L.mo, L.dy, L.hr, 0, 0.0) - wind_ref;
      } else {
        if (!prev) {
          set_error("fort.22 %s: line %d is a forecast with no earlier line", path, lineno);
          return ADC_ERR_ARG;
        }
        fi = fi * 3600.0;
        ct = cast_time.back() + (fi - fcst_inc.back());
      }
      if (L.type == "OFCL" && (L.cp == 0 || L.rmw == 0)) {
        set_error("fort.22 %s: line %d has no central pressure or Rmax (forecast lines need both)",
                  path, lineno);
        return ADC_ERR_ARG;
      }
    } else {
      set_error("fort.22 %s: line %d: only BEST, OFCL or CALM lines are allowed, not '%s'", path,
                lineno, L.type.c_str());
      return ADC_ERR_ARG;
    }
    kept.push_back(L);
    cast_time.push_back(ct);
    fcst_inc.push_back(fi);
  }
  const int pl = (int)kept.size();
  if (pl < 2) {
    set_error("fort.22 %s: fewer than two track times", path);
    return ADC_ERR_ARG;
  }
  if (o->rnday > 0.0 && cast_time[pl - 1] < o->rnday * 86400.0) {
    set_error("fort.22 %s: the track ends at %g s, before RNDAY", path, cast_time[pl - 1]);
    return ADC_ERR_ARG;
  }
  for (int i = 1; i < pl; ++i)
    if (!(cast_time[i] > cast_time[i - 1])) {
      set_error("fort.22 %s: track time %d does not follow the one before", path, i + 1);
      return ADC_ERR_ARG;
    }
  if (!fix) {
    *nfix = pl;
    return ADC_OK;
  }
  if (*nfix < pl) {
    set_error("adc_fort22_read: room for %d fixes, the track has %d", *nfix, pl);
    return ADC_ERR_ARG;
  }
  std::vector<double> lat(pl), lon(pl);
  for (int i = 0; i < pl; ++i) {
    lat[i] = kept[i].lat / 10.0;
    lon[i] = kept[i].lon / 10.0;
    if (kept[i].ew == 'W') lon[i] = -1.0 * lon[i];
    if (kept[i].ns == 'S') lat[i] = -1.0 * lat[i];
  }
  const double lam0 = o->slam0 * kDeg2Rad, phi0 = o->sfea0 * kDeg2Rad;
  for (int i = 0; i < pl; ++i) {
    adc_vortex_fix_t &x = fix[i];
    x.time = cast_time[i];
    x.x = kRearth * std::cos(phi0) * (lon[i] * kDeg2Rad - lam0);
    x.y = kRearth * (lat[i] * kDeg2Rad);
    x.cpress = kept[i].type == "CALM" ? -99999.0 : kept[i].cp * 100.0;
    x.vmax = kept[i].spd * kKt2Ms;
    x.rmw = kept[i].rmw * kNm2Km;
    x.tvx = x.tvy = 0.0;
  }
  for (int i = 1; i < pl; ++i) {   // uvtrans, wind/vortex.F:1174-1200
    const double avg = (lat[i - 1] + lat[i]) / 2.0;
    const double dx = spherical_distance((lon[i] - lon[i - 1]) * kDeg2Rad, 0.0, avg, avg);
    const double dy = spherical_distance(0.0, (lat[i] - lat[i - 1]) * kDeg2Rad, lat[i - 1], lat[i]);
    const double dt = cast_time[i] - cast_time[i - 1];
    fix[i].tvx = std::copysign(std::fabs(dx / dt), lon[i] - lon[i - 1]);
    fix[i].tvy = std::copysign(std::fabs(dy / dt), lat[i] - lat[i - 1]);
  }
  fix[0].tvx = fix[1].tvx;
  fix[0].tvy = fix[1].tvy;
  *nfix = pl;
  return ADC_OK;
}
