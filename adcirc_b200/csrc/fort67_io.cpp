// fort67_io.cpp -- the reference's own binary hotstart file (fort.67 /
// fort.68) for a serial 2DDI run, so a run can start from a reference
// hotstart and a reference run from this library's state.
//
// Layout (writeHotstart, write_output.F:4900-5154, the non-portable binary
// branch; read back by hstart.F:500-560): a direct-access file of 8-byte
// records.  An INTEGER record holds the 4-byte value in the first half of
// its record, a REAL(8) record fills it.  Records in order:
//   FileFmtVersion, IM, TimeLoc, IT, NP, NE, NP, NE,
//   ETA1(NP), ETA2(NP), EtaDisc(NP), UU2(NP), VV2(NP), CH1(NP) if IM = 10,
//   NNODECODE(NP), NOFF(NE),
//   4 NP wave radiation stress records and 4 NP SWAN records (zeros when
//   NRS = 0, as the writer pads them),
//   18 output-counter records (0 and the NSCOU* counters, written 0 here).
// Harmonic-analysis sections (written only while harmonic analysis runs)
// are not produced and are ignored on reading.  FileFmtVersion is
// VERSION_NUMBER(1, 2, 0) (global.F:1295-1303, adcirc_version.py); a file
// whose major or minor number differs is refused, as CMP_VERSION_NUMBERS
// (global.F:1307-1311) refuses it.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/adcgpu.h"

namespace adc {
void set_error(const char *fmt, ...);
}
using adc::set_error;

namespace {

constexpr int32_t kFileFmtVersion = (1 << 20) | (2 << 10) | 0;

struct Out {
  FILE *f;
  bool ok = true;
  void rec_i(int32_t v) {
    unsigned char b[8] = {0};
    std::memcpy(b, &v, 4);
    ok = ok && std::fwrite(b, 8, 1, f) == 1;
  }
  void rec_d(double v) { ok = ok && std::fwrite(&v, 8, 1, f) == 1; }
};

struct In {
  std::vector<unsigned char> buf;
  size_t rec = 0;   // next record, 0-based
  bool has(size_t n) const { return (rec + n) * 8 <= buf.size(); }
  int32_t rec_i() {
    int32_t v;
    std::memcpy(&v, buf.data() + 8 * rec++, 4);
    return v;
  }
  double rec_d() {
    double v;
    std::memcpy(&v, buf.data() + 8 * rec++, 8);
    return v;
  }
};

}  // namespace

extern "C" int adc_fort67_write(const char *path, const adc_fort67_t *h) {
  if (!path || !h || h->np < 1 || h->ne < 1 || !h->eta1 || !h->eta2 || !h->uu2 || !h->vv2 ||
      !h->nodecode || !h->noff || (h->im == 10 && !h->ch1)) {
    set_error("adc_fort67_write: sizes and the state arrays are required");
    return ADC_ERR_ARG;
  }
  Out o{std::fopen(path, "wb")};
  if (!o.f) {
    set_error("adc_fort67_write: cannot open %s", path);
    return ADC_ERR_ARG;
  }
  o.rec_i(kFileFmtVersion);
  o.rec_i(h->im);
  o.rec_d(h->timeloc);
  o.rec_i(h->it);
  o.rec_i(h->np);
  o.rec_i(h->ne);
  o.rec_i(h->np);
  o.rec_i(h->ne);
  for (const double *a : {h->eta1, h->eta2})
    for (int i = 0; i < h->np; ++i) o.rec_d(a[i]);
  for (int i = 0; i < h->np; ++i) o.rec_d(h->etadisc ? h->etadisc[i] : 0.0);
  for (const double *a : {h->uu2, h->vv2})
    for (int i = 0; i < h->np; ++i) o.rec_d(a[i]);
  if (h->im == 10)
    for (int i = 0; i < h->np; ++i) o.rec_d(h->ch1[i]);
  for (int i = 0; i < h->np; ++i) o.rec_i(h->nodecode[i]);
  for (int e = 0; e < h->ne; ++e) o.rec_i(h->noff[e]);
  for (long long k = 0; k < 8LL * h->np; ++k) o.rec_i(0);   // NRS = 0 and SWAN pads
  for (int k = 0; k < 18; ++k) o.rec_i(0);                  // output counters
  const bool closed = std::fclose(o.f) == 0;
  if (!o.ok || !closed) {
    set_error("adc_fort67_write: write to %s failed", path);
    return ADC_ERR_ARG;
  }
  return ADC_OK;
}

extern "C" int adc_fort67_read(const char *path, adc_fort67_t *h) {
  if (!path || !h) {
    set_error("adc_fort67_read: null argument");
    return ADC_ERR_ARG;
  }
  FILE *f = std::fopen(path, "rb");
  if (!f) {
    set_error("adc_fort67_read: cannot open %s", path);
    return ADC_ERR_ARG;
  }
  In in;
  unsigned char tmp[1 << 16];
  size_t n;
  while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) in.buf.insert(in.buf.end(), tmp, tmp + n);
  std::fclose(f);
  if (!in.has(8)) {
    set_error("adc_fort67_read: %s is too short for a hotstart header", path);
    return ADC_ERR_ARG;
  }
  const int32_t vn = in.rec_i();
  if ((vn >> 10) != (kFileFmtVersion >> 10)) {
    set_error("adc_fort67_read: %s has file format version %d.%d, this reader %d.%d", path,
              vn >> 20, (vn >> 10) & 1023, kFileFmtVersion >> 20, (kFileFmtVersion >> 10) & 1023);
    return ADC_ERR_ARG;
  }
  const int im = in.rec_i();
  const double timeloc = in.rec_d();
  const int it = in.rec_i();
  const int np = in.rec_i(), ne = in.rec_i();
  in.rec_i();
  in.rec_i();
  if (h->np == 0 && h->ne == 0) {   // size query
    h->im = im;
    h->timeloc = timeloc;
    h->it = it;
    h->np = np;
    h->ne = ne;
    return ADC_OK;
  }
  if (np != h->np || ne != h->ne) {
    set_error("adc_fort67_read: %s holds NP %d NE %d, the caller expects NP %d NE %d", path, np, ne,
              h->np, h->ne);
    return ADC_ERR_ARG;
  }
  const size_t need = 5 * (size_t)np + (im == 10 ? np : 0) + np + ne;
  if (!in.has(need)) {
    set_error("adc_fort67_read: %s is truncated", path);
    return ADC_ERR_ARG;
  }
  if (!h->eta1 || !h->eta2 || !h->uu2 || !h->vv2 || !h->nodecode || !h->noff) {
    set_error("adc_fort67_read: the state arrays are required");
    return ADC_ERR_ARG;
  }
  h->im = im;
  h->timeloc = timeloc;
  h->it = it;
  for (double *a : {h->eta1, h->eta2})
    for (int i = 0; i < np; ++i) a[i] = in.rec_d();
  for (int i = 0; i < np; ++i) {
    const double v = in.rec_d();
    if (h->etadisc) h->etadisc[i] = v;
  }
  for (double *a : {h->uu2, h->vv2})
    for (int i = 0; i < np; ++i) a[i] = in.rec_d();
  if (im == 10)
    for (int i = 0; i < np; ++i) {
      const double v = in.rec_d();
      if (h->ch1) h->ch1[i] = v;
    }
  for (int i = 0; i < np; ++i) h->nodecode[i] = in.rec_i();
  for (int e = 0; e < ne; ++e) h->noff[e] = in.rec_i();
  return ADC_OK;
}
