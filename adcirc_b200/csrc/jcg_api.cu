// jcg_api.cu -- the ITPACK entry points jcg / dfault (itpackv.F:63, 1070)
// with the reference's argument list, running the device JCG kernel.
//
// The host part mirrors what jcg does before iterating: echall
// (itpackv.F:1212-1255), the zeta floor (:223-232), and the structural half
// of scal (:2281-2391: diagonal moved to column 1, negative rows negated,
// zero diagonal -> ier 401, empty jcoef slots -> the row itself).  The
// system is then staged once in HBM in sliced-ELL form and solved by the
// persistent kernel of jcg.cu, which performs the numerical scal/unscal,
// the iteration and peror; the scaled-then-unscaled coefficients are
// copied back as the reference leaves them.
#include "adc_internal.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>
#include <algorithm>

namespace adc {
int jcg_setup_grid(adc_ctx *c, const JcgHostSell *h);
int launch_jcg_impl(adc_ctx *c, int eta_update, int do_peror, int run_init, int defer_drift);

// ITPACK state that survives between jcg calls: itjcg's SAVEd q1 flag.
static int g_q1 = 0;
int jcg_q1_get() { return g_q1; }
void jcg_q1_set(int v) { g_q1 = v; }

struct Stage {
  adc_ctx c;
  Stage() { memset((void *)&c, 0, sizeof(c)); }
  ~Stage() {
    void *ptrs[] = {c.sl_ptr, c.sl_w, c.col, c.rlen, c.offd, c.soff, c.diag, c.gwce_lv,
                    c.etas, c.ju1, c.jp[0], c.jp[1], c.jw, c.jexp, c.jlcol, c.jhalo_ptr, c.jhalo_ids,
                    c.jpart, c.jtri, c.itp, c.bar, c.flags, c.jlines};
    for (void *p : ptrs)
      if (p) cudaFree(p);
    if (c.stream) cudaStreamDestroy(c.stream);
  }
};

template <class T>
static cudaError_t alloc_up(T **d, const T *h, size_t n) {
  cudaError_t e = cudaMalloc((void **)d, std::max<size_t>(n, 1) * sizeof(T));
  if (e != cudaSuccess || !h || n == 0) return e;
  return cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice);
}

static int jcg_solve(int n, int ndim, int maxnz, int *jcoef, double *coef, double *rhs,
                     double *u, int itmax, int *iparm, double *rparm, int &ier, int &in_out,
                     double &stptst, double &cme, double &bnrm, double &rnrm) {
  // sliced ELL of the slots that take part in pjac: every j >= 2 except the
  // empty ones (jcoef == i and coef == 0, i.e. 0*u(i) terms)
  const int nslices = (n + kSlice - 1) / kSlice;
  std::vector<int> rlen(n, 0), sl_w(nslices, 0), sl_ptr(nslices + 1, 0);
  std::vector<std::vector<int>> rows(n);
  for (int i = 0; i < n; ++i) {
    for (int j = 1; j < maxnz; ++j) {
      size_t k = i + (size_t)ndim * j;
      if (jcoef[k] == i + 1 && coef[k] == 0.0) continue;
      rows[i].push_back(j);
    }
    rlen[i] = (int)rows[i].size();
    sl_w[i / kSlice] = std::max(sl_w[i / kSlice], rlen[i]);
  }
  for (int s = 0; s < nslices; ++s) sl_ptr[s + 1] = sl_ptr[s] + sl_w[s] * kSlice;
  const int nnz = sl_ptr[nslices];
  std::vector<int> col(std::max(nnz, 1), 0), src(std::max(nnz, 1), -1);
  std::vector<double> off(std::max(nnz, 1), 0.0), diag(n);
  for (int i = 0; i < n; ++i) {
    diag[i] = coef[i];
    int s = i / kSlice, lane = i % kSlice;
    for (int k = 0; k < sl_w[s]; ++k) {
      int idx = sl_ptr[s] + k * kSlice + lane;
      if (k < rlen[i]) {
        size_t e = i + (size_t)ndim * rows[i][k];
        col[idx] = jcoef[e] - 1;
        off[idx] = coef[e];
        src[idx] = (int)e;
      } else {
        col[idx] = i;
      }
    }
  }
  Stage st;
  adc_ctx &c = st.c;
  c.np = n;
  c.nslices = nslices;
  c.nnz_pad = nnz;
  c.itmax = itmax;
  if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return ADC_ERR_CUDA;
  ADC_CUDA(alloc_up(&c.sl_ptr, sl_ptr.data(), sl_ptr.size()));
  ADC_CUDA(alloc_up(&c.sl_w, sl_w.data(), sl_w.size()));
  ADC_CUDA(alloc_up(&c.col, col.data(), col.size()));
  rlen.resize((size_t)nslices * kSlice, 0);
  ADC_CUDA(alloc_up(&c.rlen, rlen.data(), rlen.size()));
  ADC_CUDA(alloc_up(&c.offd, off.data(), off.size()));
  ADC_CUDA(alloc_up<double>(&c.soff, nullptr, off.size()));
  ADC_CUDA(alloc_up(&c.diag, diag.data(), n));
  ADC_CUDA(alloc_up(&c.gwce_lv, rhs, n));
  const size_t npad = (size_t)nslices * kSlice;
  ADC_CUDA(alloc_up<double>(&c.etas, nullptr, npad));
  ADC_CUDA(cudaMemset(c.etas, 0, npad * sizeof(double)));
  ADC_CUDA(cudaMemcpy(c.etas, u, n * sizeof(double), cudaMemcpyHostToDevice));
  double **vec[] = {&c.ju1, &c.jw};
  for (double **v : vec) {
    ADC_CUDA(alloc_up<double>(v, nullptr, npad));
    ADC_CUDA(cudaMemset(*v, 0, npad * sizeof(double)));
  }
  ADC_CUDA(alloc_up<double4>(&c.jp[0], nullptr, npad));
  ADC_CUDA(alloc_up<double4>(&c.jp[1], nullptr, npad));
  ADC_CUDA(cudaMemset(c.jp[0], 0, npad * sizeof(double4)));
  ADC_CUDA(cudaMemset(c.jp[1], 0, npad * sizeof(double4)));
  const JcgHostSell hs{sl_ptr.data(), sl_w.data(), col.data(), rlen.data()};
  int rc = jcg_setup_grid(&c, &hs);
  if (rc) return rc;
  ADC_CUDA(alloc_up<double>(&c.jpart, nullptr, 4 * (size_t)c.jcg_grid));
  ADC_CUDA(alloc_up<double>(&c.jtri, nullptr, 4 * (size_t)std::max(itmax, 2)));
  ADC_CUDA(alloc_up<char>((char **)&c.jlines, nullptr, 2 * 128 * (size_t)c.jcg_rows_blocks));
  Itp it;
  memset(&it, 0, sizeof(it));
  it.zeta = rparm[0];
  it.rparm1 = rparm[0];
  it.cme = rparm[1];
  it.sme = (rparm[2] == 0.0) ? -1.0 : rparm[2];
  it.itmax = itmax;
  it.adapt = (iparm[5] == 1 || iparm[5] == 3) ? 1 : 0;
  it.q1 = g_q1;
  it.srelpr = DBL_EPSILON;
  double temp = 512.0 * DBL_EPSILON;
  if (it.zeta < temp) it.zeta = temp;
  it.rec.need_unorm = !it.q1;
  ADC_CUDA(alloc_up(&c.itp, &it, 1));
  Bar bar = {0, 0};
  ADC_CUDA(alloc_up(&c.bar, &bar, 1));
  Flags fl;
  memset(&fl, 0, sizeof(fl));
  ADC_CUDA(alloc_up(&c.flags, &fl, 1));
  rc = launch_jcg_impl(&c, 0, iparm[11] >= 0 ? 1 : 0, 0, 0);
  if (rc) return rc;
  ADC_CUDA(cudaStreamSynchronize(c.stream));
  ADC_CUDA(cudaMemcpy(&fl, c.flags, sizeof(fl), cudaMemcpyDeviceToHost));
  if (fl.timeout) { set_error("JCG barrier wait expired"); return ADC_ERR_TIMEOUT; }
  ADC_CUDA(cudaMemcpy(&it, c.itp, sizeof(it), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(u, c.etas, n * sizeof(double), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(rhs, c.gwce_lv, n * sizeof(double), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(diag.data(), c.diag, n * sizeof(double), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(off.data(), c.offd, nnz * sizeof(double), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) coef[i] = diag[i];
  for (int idx = 0; idx < nnz; ++idx)
    if (src[idx] >= 0) coef[src[idx]] = off[idx];
  g_q1 = it.q1;
  ier = fl.ier;
  in_out = it.in;
  stptst = it.stptst;
  cme = it.cme;
  bnrm = it.dtnrm;
  rnrm = it.unorm;
  return ADC_OK;
}

}  // namespace adc

using namespace adc;

extern "C" {

void adc_dfault(int *iparm, double *rparm) {
  // dfault, itpackv.F:1070-1170 (srelpr = 2**-52 for IEEE double)
  const double srelpr = DBL_EPSILON;
  const int ip[12] = {100, -1, 0, 6, 0, 1, 1, 0, -2, 0, 0, 3};
  for (int k = 0; k < 12; ++k) iparm[k] = ip[k];
  rparm[0] = 5.0e-6; rparm[1] = 0.0; rparm[2] = 0.0; rparm[3] = 0.75; rparm[4] = 1.0;
  rparm[5] = 0.0; rparm[6] = 0.25; rparm[7] = 128.0 * srelpr; rparm[8] = 0.0;
  rparm[9] = 0.0; rparm[10] = 0.0; rparm[11] = 0.0;
}

void adc_jcg_reset(void) { g_q1 = 0; }

void adc_jcg(const int *n_, const int *ndim_, const int *maxnz_, int *jcoef, double *coef,
             double *rhs, double *u, int *iwksp, const int *nw_, double *wksp, int *iparm,
             double *rparm, int *ier) {
  (void)iwksp;
  (void)wksp;
  *ier = 0;
  const int n = *n_, ndim = *ndim_, maxnz = *maxnz_, nw = *nw_;
  if (iparm[0] <= 0) return;
  const int itmax = iparm[0];
  if (n <= 0) { *ier = 11; return; }
  if (ndim < n || maxnz < 1) { *ier = 11; set_error("ndim < n or maxnz < 1"); return; }
  // structural part of scal (itpackv.F:2340-2391)
  int nsgncg = 0;
  for (int i = 1; i <= n; ++i) {
    int *jr = jcoef + (i - 1);
    double *cr = coef + (i - 1);
    if (jr[0] != i) {
      if (maxnz < 2) { *ier = 402; return; }
      for (int j = 2; j <= maxnz; ++j) {
        size_t k = (size_t)ndim * (j - 1);
        if (jr[k] == i) {
          double save = cr[k];
          cr[k] = cr[0];
          jr[k] = jr[0];
          cr[0] = save;
          jr[0] = i;
        }
      }
    }
    if (cr[0] < 0.0) {
      for (int j = 1; j <= maxnz; ++j) cr[(size_t)ndim * (j - 1)] = -cr[(size_t)ndim * (j - 1)];
      rhs[i - 1] = -rhs[i - 1];
      nsgncg++;
    } else if (cr[0] == 0.0) {
      *ier = 401;
      return;
    }
  }
  for (int j = 2; j <= maxnz; ++j)
    for (int i = 1; i <= n; ++i)
      if (jcoef[(i - 1) + (size_t)ndim * (j - 1)] <= 0) jcoef[(i - 1) + (size_t)ndim * (j - 1)] = i;
  auto restore_zeros = [&]() {
    for (int j = 2; j <= maxnz; ++j)
      for (int i = 1; i <= n; ++i)
        if (jcoef[(i - 1) + (size_t)ndim * (j - 1)] == i) jcoef[(i - 1) + (size_t)ndim * (j - 1)] = 0;
  };
  if (nsgncg > 0 && nsgncg < n) {
    // ITPACK would switch to the nonsymmetric eigenvalue routine
    // (isym = 1, eigvns/eqrt1s); that branch is not implemented.
    *ier = 903;
    restore_zeros();
    set_error("mixed-sign diagonal (ITPACK isym branch) not supported");
    return;
  }
  iparm[7] = 4 * n + 4 * itmax;
  if (nw < iparm[7]) {
    *ier = 12;
    restore_zeros();
    return;
  }
  int e = 0, in = 0;
  double stptst = 0, cme = 0, bnrm = 0, rnrm = 0;
  int rc = jcg_solve(n, ndim, maxnz, jcoef, coef, rhs, u, itmax, iparm, rparm, e, in, stptst,
                     cme, bnrm, rnrm);
  if (rc != ADC_OK) {
    *ier = 904;
    restore_zeros();
    return;
  }
  restore_zeros();
  *ier = e;
  if (e == 13 && iparm[2] == 0) rparm[0] = stptst;
  double digit1 = rparm[10], digit2 = rparm[11];
  if (iparm[11] >= 0) {
    const double srelpr = DBL_EPSILON;
    digit1 = -std::log10(std::fabs(srelpr));
    if (stptst > 0.0) digit1 = -std::log10(std::fabs(stptst));
    if (bnrm == 0.0) {
      digit2 = -std::log10(std::fabs(srelpr));
    } else {
      double temp = rnrm / bnrm;
      digit2 = (temp == 0.0) ? -std::log10(std::fabs(srelpr)) : -std::log10(std::fabs(temp)) / 2.0;
    }
  }
  iparm[7] = iparm[7] - 4 * (itmax - in);
  if (iparm[2] != 0) return;
  iparm[0] = in;
  rparm[1] = cme;
  rparm[2] = (rparm[2] == 0.0) ? -1.0 : rparm[2];
  rparm[10] = digit1;
  rparm[11] = digit2;
}

}  // extern "C"
