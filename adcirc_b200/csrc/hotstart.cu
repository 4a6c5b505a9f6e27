// hotstart.cu -- hotstart dump and load of the device-resident state.
//
// The reference writes fort.67/68 (write_output.F:4429-5582) and reads them
// back at start-up (hstart.F:47-2048); a restarted reference run rebuilds
// its GWCE matrix and restarts ITPACK's saved state.  This file format is
// this library's own: it holds every array and scalar the device step
// carries from one step to the next (state fields, the GWCE matrix and EP,
// ITPACK's persistent scalars, the pending unscal drift, the vortex track
// state, the specified boundary fluxes of the last two steps, the position
// in non-periodic boundary series and the warm-start history), so N steps equal N/2 steps, a dump, a
// load into a freshly bound context of the same mesh and mode, and N/2
// more steps, bit for bit.
//
// Layout: "ADCB2HS\0", u32 version, then i64 np, ne, nnz_pad, n_obc, mode,
// record count; then per record a 32-byte zero-padded name, u64 byte count
// and the bytes (host byte order).
#include "adc_internal.cuh"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace adc {

constexpr char kHsMagic[8] = {'A', 'D', 'C', 'B', '2', 'H', 'S', '\0'};
constexpr uint32_t kHsVersion = 1;

struct HsRec {
  const char *name;
  void *dev;
  size_t bytes;
};

static std::vector<HsRec> hs_records(adc_ctx *c) {
  const size_t np = c->np, ne = c->ne;
  const size_t d = sizeof(double), i4 = sizeof(int);
  std::vector<HsRec> r = {
      {"eta1", c->eta1, np * d},        {"eta2", c->eta2, np * d},
      {"etas", c->etas, np * d},        {"uu1", c->uu1, np * d},
      {"vv1", c->vv1, np * d},          {"uu2", c->uu2, np * d},
      {"vv2", c->vv2, np * d},          {"qx1", c->qx1, np * d},
      {"qy1", c->qy1, np * d},          {"qx2", c->qx2, np * d},
      {"qy2", c->qy2, np * d},          {"h1", c->h1, np * d},
      {"h2", c->h2, np * d},            {"tk", c->tk, np * d},
      {"tkm", c->tkm, 3 * np * d},      {"totalarea", c->totalarea, np * d},
      {"wsx1", c->wsx1, np * d},        {"wsy1", c->wsy1, np * d},
      {"wsx2", c->wsx2, np * d},        {"wsy2", c->wsy2, np * d},
      {"pr1", c->pr1, np * d},          {"pr2", c->pr2, np * d},
      {"gwce_lv", c->gwce_lv, np * d},  {"mom_lv_x", c->mom_x, np * d},
      {"mom_lv_y", c->mom_y, np * d},   {"nodecode", c->nodecode, np * i4},
      {"nnodecode", c->nnodecode, np * i4}, {"mju", c->mju, np * i4},
      {"noff", c->noff, ne * i4},       {"noffold", c->noffold, ne * i4},
      {"alphal", c->alphal, ne * d},    {"coef_diag", c->diag, np * d},
      {"coef_offd", c->offd, (size_t)c->nnz_pad * d},
      {"obccoef", c->obccoef, (size_t)c->n_obc * d},
      {"jcg_w", c->jw, np * d},         // the w of the last solve (pending drift)
      {"flags", c->flags, sizeof(Flags)},
      {"lhs_words", c->flags + 1, 3 * i4},   // rebuild decision, drift pending/apply
      {"itpack", c->itp, sizeof(Itp)},
  };
  if (c->vortex_on) r.push_back({"vortex", c->vstate, sizeof(VortexState)});
  if (c->nfluxf || c->nfluxrbc || c->nfluxgbc || c->nfluxb || c->nfluxib) {
    r.push_back({"flux_qn", c->qn, 3 * (size_t)c->nvel * d});
    r.push_back({"flux_en", c->en, 3 * (size_t)c->nvel * d});
    r.push_back({"flux_elevdisc", c->elevdisc, (size_t)c->nvel * d});   // river radiation
    r.push_back({"flux_etadisc", c->etadisc_b, (size_t)c->nvel * d});
  }
  // fort.19 / fort.20 record pair, read-ahead times and ratio
  if (c->eser_on || c->fser_on) r.push_back({"series", c->sstate, 2 * sizeof(SeriesState)});
  if (c->prec & ADC_WARM_START) {
    r.push_back({"etas_prev", c->etas_prev, np * d});
    r.push_back({"warm", c->warm, sizeof(WarmState)});
  }
  return r;
}

struct HsHeader {
  char magic[8];
  uint32_t version, pad_;
  int64_t np, ne, nnz_pad, n_obc, mode, nrec;
};

}  // namespace adc

using namespace adc;

extern "C" int adc_hotstart_write(adc_ctx *c, const char *path) {
  if (!c || !path) { set_error("adc_hotstart_write: null argument"); return ADC_ERR_ARG; }
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  const std::vector<HsRec> recs = hs_records(c);
  FILE *f = std::fopen(path, "wb");
  if (!f) { set_error("adc_hotstart_write: cannot open %s", path); return ADC_ERR_ARG; }
  HsHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kHsMagic, 8);
  h.version = kHsVersion;
  h.np = c->np; h.ne = c->ne; h.nnz_pad = c->nnz_pad; h.n_obc = c->n_obc; h.mode = c->prec;
  h.nrec = (int64_t)recs.size();
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
  std::vector<char> buf;
  for (const HsRec &r : recs) {
    if (!ok) break;
    char name[32];
    memset(name, 0, sizeof(name));
    std::strncpy(name, r.name, sizeof(name) - 1);
    const uint64_t nb = r.bytes;
    buf.resize(r.bytes > 0 ? r.bytes : 1);
    if (r.bytes > 0 && cudaMemcpy(buf.data(), r.dev, r.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
      std::fclose(f);
      return cuda_fail(cudaGetLastError(), "adc_hotstart_write: device copy");
    }
    ok = std::fwrite(name, sizeof(name), 1, f) == 1 && std::fwrite(&nb, sizeof(nb), 1, f) == 1 &&
         (r.bytes == 0 || std::fwrite(buf.data(), r.bytes, 1, f) == 1);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) { set_error("adc_hotstart_write: write to %s failed", path); return ADC_ERR_ARG; }
  return ADC_OK;
}

extern "C" int adc_hotstart_read(adc_ctx *c, const char *path) {
  if (!c || !path) { set_error("adc_hotstart_read: null argument"); return ADC_ERR_ARG; }
  FILE *f = std::fopen(path, "rb");
  if (!f) { set_error("adc_hotstart_read: cannot open %s", path); return ADC_ERR_ARG; }
  HsHeader h;
  if (std::fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, kHsMagic, 8) != 0 ||
      h.version != kHsVersion) {
    std::fclose(f);
    set_error("adc_hotstart_read: %s is not a hotstart file of this library (version %u)", path,
              kHsVersion);
    return ADC_ERR_ARG;
  }
  if (h.np != c->np || h.ne != c->ne || h.nnz_pad != c->nnz_pad || h.n_obc != c->n_obc ||
      h.mode != c->prec) {
    std::fclose(f);
    set_error("adc_hotstart_read: %s holds np %lld ne %lld mode %lld, the context np %d ne %d mode %d",
              path, (long long)h.np, (long long)h.ne, (long long)h.mode, c->np, c->ne, c->prec);
    return ADC_ERR_ARG;
  }
  const std::vector<HsRec> recs = hs_records(c);
  if (h.nrec != (int64_t)recs.size()) {
    std::fclose(f);
    set_error("adc_hotstart_read: %s has %lld records, the context needs %zu (vortex, flux, "
              "boundary-series or warm-start state differs)", path, (long long)h.nrec, recs.size());
    return ADC_ERR_ARG;
  }
  ADC_CUDA(cudaStreamSynchronize(c->stream));
  std::vector<char> buf;
  std::vector<bool> seen(recs.size(), false);
  for (int64_t k = 0; k < h.nrec; ++k) {
    char name[32];
    uint64_t nb = 0;
    if (std::fread(name, sizeof(name), 1, f) != 1 || std::fread(&nb, sizeof(nb), 1, f) != 1) {
      std::fclose(f);
      set_error("adc_hotstart_read: %s is truncated", path);
      return ADC_ERR_ARG;
    }
    name[31] = '\0';
    size_t j = 0;
    while (j < recs.size() && std::strcmp(recs[j].name, name) != 0) ++j;
    if (j == recs.size() || seen[j] || nb != recs[j].bytes) {
      std::fclose(f);
      set_error("adc_hotstart_read: record '%s' (%llu bytes) does not fit this context", name,
                (unsigned long long)nb);
      return ADC_ERR_ARG;
    }
    buf.resize(nb > 0 ? nb : 1);
    if (nb > 0 && std::fread(buf.data(), nb, 1, f) != 1) {
      std::fclose(f);
      set_error("adc_hotstart_read: %s is truncated", path);
      return ADC_ERR_ARG;
    }
    if (nb > 0 && cudaMemcpy(recs[j].dev, buf.data(), nb, cudaMemcpyHostToDevice) != cudaSuccess) {
      std::fclose(f);
      return cuda_fail(cudaGetLastError(), "adc_hotstart_read: device copy");
    }
    seen[j] = true;
  }
  std::fclose(f);
  c->met_pending = 0;
  // the cached GWCE element entries describe the old state: rebuild in full
  {
    int *w = (int *)(c->flags + 1);
    int all = 1;
    ADC_CUDA(cudaMemcpy(w + 3, &all, sizeof(int), cudaMemcpyHostToDevice));
    ADC_CUDA(cudaMemset(c->lhs_nc, 0xff, (size_t)c->ne * sizeof(int)));
  }
  return ADC_OK;
}
