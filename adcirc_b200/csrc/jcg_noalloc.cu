// jcg_noalloc.cu -- the ITPACK jcg entry point for callers that must not
// allocate: all device staging lives in one file-scope __device__ array.
//
// Some hosts cannot let a library call cudaMalloc: a coupled model that
// owns every device byte through its own pool and accounts for it, or a
// process that runs under a fixed device-memory budget set when it
// started.  adc_jcg stages each solve in freshly allocated device memory,
// so those hosts cannot use it.  adc_jcg_noalloc takes the same arguments
// and performs the same solve, but carves every device buffer (matrix,
// vectors, barrier lines, ITPACK scalars) out of the static array below.
// Limits and behaviour:
//  * capacity ADC_JCG_NOALLOC_BYTES (32 MiB); a system needs about
//    n * (20 * (maxnz - 1) + 112) bytes plus 32 bytes per ITMAX, e.g.
//    n <= 80,000 at maxnz = 16; the exact layout is checked before any
//    device work, and a system that does not fit returns ier = 905 with a
//    message in adc_last_error();
//  * the array is held by every GPU that loads the library until the
//    process exits;
//  * the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress) for that device;
//  * every call shares the array and finds the previous call's contents;
//    the solver clears what must start at zero; calls whose GPU work
//    overlaps (other host threads, other streams) race on it;
//  * the call is synchronous: it copies with cudaMemcpy/cudaMemset on the
//    legacy default stream and returns once the solution is on the host;
//  * it issues no cudaMalloc, cudaFree or stream creation and no host heap
//    allocation.
#include "adc_internal.cuh"

#include <cfloat>
#include <cmath>
#include <cstring>

namespace adc {
int jcg_setup_grid(adc_ctx *c, const JcgHostSell *h);
int launch_jcg_impl(adc_ctx *c, int eta_update, int do_peror, int run_init, int defer_drift);
int jcg_q1_get();
void jcg_q1_set(int v);

constexpr size_t kNoAllocBytes = (size_t)32 << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device (host code may not use the
// symbol's host-side stand-in as a device pointer).
constexpr int kMaxDevices = 64;
static void *g_noalloc_ptr[kMaxDevices];

static int noalloc_base(void **out) {
  int dev = 0;
  ADC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) { set_error("device ordinal out of range"); return ADC_ERR_ARG; }
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return ADC_OK;
}

// Bump allocator over the static array.  A request that does not fit
// makes the carve fail for good: every later take returns nullptr too and
// `failed` stays set, so no partly carved layout reaches a kernel.
struct Carve {
  char *base;
  size_t off, cap;
  bool failed;
  template <class T>
  T *take(size_t n) {
    size_t bytes = ((std::max<size_t>(n, 1) * sizeof(T)) + 255) & ~(size_t)255;
    if (failed || off + bytes > cap) {
      failed = true;
      return nullptr;
    }
    T *p = base ? (T *)(base + off) : nullptr;
    off += bytes;
    return p;
  }
};

// Lays out every buffer of one solve, in one fixed order, over `cv`.  With
// cv.base == nullptr it only counts bytes (the size precheck).
static void noalloc_carve(Carve &cv, adc_ctx &c, int n, int nslices, size_t slots, int itmax) {
  const size_t npad = (size_t)nslices * kSlice;
  c.sl_ptr = cv.take<int>(nslices + 1);
  c.sl_w = cv.take<int>(nslices);
  c.rlen = cv.take<int>(npad);
  c.col = cv.take<int>(slots);
  c.offd = cv.take<double>(slots);
  c.soff = cv.take<double>(slots);
  c.diag = cv.take<double>(n);
  c.gwce_lv = cv.take<double>(n);
  c.etas = cv.take<double>(npad);
  c.ju1 = cv.take<double>(npad);
  c.jw = cv.take<double>(npad);
  c.jp[0] = cv.take<double4>(npad);
  c.jp[1] = cv.take<double4>(npad);
  c.jpart = cv.take<double>(4 * (size_t)c.jcg_grid);
  c.jtri = cv.take<double>(4 * (size_t)(itmax > 2 ? itmax : 2));
  c.jlines = cv.take<char>(2 * 128 * (size_t)c.jcg_rows_blocks);
  c.itp = cv.take<Itp>(1);
  c.bar = cv.take<Bar>(1);
  c.flags = cv.take<Flags>(1);
}

// Exact scratch bytes of one solve with the largest row-block count the
// solver can choose for n rows (jcg_setup_grid never uses more than
// max(1, slices/8) row blocks), or SIZE_MAX when it would not fit.
static size_t noalloc_need(int n, int maxnz, int itmax) {
  const int w = maxnz - 1;
  const int nslices = (n + kSlice - 1) / kSlice;
  const size_t slots = (size_t)nslices * kSlice * (w > 0 ? w : 1);
  adc_ctx c;
  memset((void *)&c, 0, sizeof(c));
  c.jcg_rows_blocks = std::max(1, nslices / 8);
  c.jcg_grid = c.jcg_rows_blocks + 1;
  Carve cv{nullptr, 0, kNoAllocBytes, false};
  noalloc_carve(cv, c, n, nslices, slots, itmax);
  return cv.failed ? SIZE_MAX : cv.off;
}

__global__ void k_noalloc_layout(int n, int nslices, int w, int *sl_ptr, int *sl_w, int *rlen,
                                 int *col) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= nslices) sl_ptr[t] = t * kSlice * w;
  if (t < nslices) sl_w[t] = w;
  if (t < nslices * kSlice) rlen[t] = (t < n) ? w : 0;
  // col holds jcoef (1-based) as copied from the host; rows past n are padding
  size_t tot = (size_t)nslices * kSlice * w;
  for (size_t k = t; k < tot; k += (size_t)gridDim.x * blockDim.x) {
    int lane = (int)(k % kSlice);
    int s = (int)(k / ((size_t)kSlice * w));
    int row = s * kSlice + lane;
    col[k] = (row < n) ? col[k] - 1 : 0;
  }
}

// Copies column j (0-based) of an (ndim, maxnz) Fortran array into the
// fixed-width sliced ELL slot k = j - 1, in either direction.
template <class T>
static int copy_column(T *dev, T *host, int n, int ndim, int w, int j, bool to_device) {
  const int full = n / kSlice, tail = n - full * kSlice;
  T *h = host + (size_t)ndim * j;
  T *d = dev + (size_t)(j - 1) * kSlice;
  const size_t dpitch = (size_t)kSlice * w * sizeof(T), spitch = kSlice * sizeof(T);
  if (full > 0) {
    if (to_device)
      ADC_CUDA(cudaMemcpy2D(d, dpitch, h, spitch, kSlice * sizeof(T), full, cudaMemcpyHostToDevice));
    else
      ADC_CUDA(cudaMemcpy2D(h, spitch, d, dpitch, kSlice * sizeof(T), full, cudaMemcpyDeviceToHost));
  }
  if (tail > 0) {
    if (to_device)
      ADC_CUDA(cudaMemcpy(d + full * (size_t)kSlice * w, h + (size_t)full * kSlice,
                          tail * sizeof(T), cudaMemcpyHostToDevice));
    else
      ADC_CUDA(cudaMemcpy(h + (size_t)full * kSlice, d + full * (size_t)kSlice * w,
                          tail * sizeof(T), cudaMemcpyDeviceToHost));
  }
  return ADC_OK;
}

static int noalloc_solve(int n, int ndim, int maxnz, int *jcoef, double *coef, double *rhs,
                         double *u, int itmax, const int *iparm, const double *rparm, int &ier,
                         int &in_out, double &stptst, double &cme, double &bnrm, double &rnrm) {
  void *base = nullptr;
  int rc = noalloc_base(&base);
  if (rc) return rc;
  const int w = maxnz - 1;
  const int nslices = (n + kSlice - 1) / kSlice;
  const size_t slots = (size_t)nslices * kSlice * (w > 0 ? w : 1);
  const size_t npad = (size_t)nslices * kSlice;
  adc_ctx c;
  memset((void *)&c, 0, sizeof(c));
  c.np = n;
  c.nslices = nslices;
  c.nnz_pad = (int)slots;
  c.itmax = itmax;
  c.stream = 0;   // legacy default stream: nothing is created
  rc = jcg_setup_grid(&c, nullptr);   // the direct variant: no host tables
  if (rc) return rc;
  Carve cv{(char *)base, 0, kNoAllocBytes, false};
  noalloc_carve(cv, c, n, nslices, slots, itmax);
  if (cv.failed) {
    set_error("adc_jcg_noalloc: n = %d, maxnz = %d, itmax = %d does not fit the %zu-byte "
              "static scratch", n, maxnz, itmax, kNoAllocBytes);
    return ADC_ERR_NOMEM;
  }
  // matrix: column 1 is the diagonal, columns 2..maxnz the sliced ELL
  ADC_CUDA(cudaMemcpy(c.diag, coef, n * sizeof(double), cudaMemcpyHostToDevice));
  if (w > 0) {
    ADC_CUDA(cudaMemset(c.offd, 0, slots * sizeof(double)));
    ADC_CUDA(cudaMemset(c.col, 0, slots * sizeof(int)));
    for (int j = 1; j < maxnz; ++j) {
      rc = copy_column(c.offd, coef, n, ndim, w, j, true);
      if (rc) return rc;
      rc = copy_column(c.col, jcoef, n, ndim, w, j, true);
      if (rc) return rc;
    }
  }
  k_noalloc_layout<<<nblk((long long)nslices * kSlice + 1), kThreads>>>(n, nslices, w > 0 ? w : 0,
                                                                       c.sl_ptr, c.sl_w, c.rlen,
                                                                       c.col);
  ADC_CUDA(cudaGetLastError());
  ADC_CUDA(cudaMemcpy(c.gwce_lv, rhs, n * sizeof(double), cudaMemcpyHostToDevice));
  ADC_CUDA(cudaMemset(c.etas, 0, npad * sizeof(double)));
  ADC_CUDA(cudaMemset(c.ju1, 0, npad * sizeof(double)));
  ADC_CUDA(cudaMemset(c.jp[0], 0, npad * sizeof(double4)));
  ADC_CUDA(cudaMemset(c.jp[1], 0, npad * sizeof(double4)));
  ADC_CUDA(cudaMemcpy(c.etas, u, n * sizeof(double), cudaMemcpyHostToDevice));
  Itp it;
  memset(&it, 0, sizeof(it));
  it.zeta = rparm[0];
  it.rparm1 = rparm[0];
  it.cme = rparm[1];
  it.sme = (rparm[2] == 0.0) ? -1.0 : rparm[2];
  it.itmax = itmax;
  it.adapt = (iparm[5] == 1 || iparm[5] == 3) ? 1 : 0;
  it.q1 = jcg_q1_get();
  it.srelpr = DBL_EPSILON;
  const double temp = 512.0 * DBL_EPSILON;
  if (it.zeta < temp) it.zeta = temp;
  it.rec.need_unorm = !it.q1;
  ADC_CUDA(cudaMemcpy(c.itp, &it, sizeof(it), cudaMemcpyHostToDevice));
  Bar bar = {0, 0};
  ADC_CUDA(cudaMemcpy(c.bar, &bar, sizeof(bar), cudaMemcpyHostToDevice));
  Flags fl;
  memset(&fl, 0, sizeof(fl));
  ADC_CUDA(cudaMemcpy(c.flags, &fl, sizeof(fl), cudaMemcpyHostToDevice));
  rc = launch_jcg_impl(&c, 0, iparm[11] >= 0 ? 1 : 0, 0, 0);
  if (rc) return rc;
  ADC_CUDA(cudaStreamSynchronize(0));
  ADC_CUDA(cudaMemcpy(&fl, c.flags, sizeof(fl), cudaMemcpyDeviceToHost));
  if (fl.timeout) { set_error("JCG barrier wait expired"); return ADC_ERR_TIMEOUT; }
  ADC_CUDA(cudaMemcpy(&it, c.itp, sizeof(it), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(u, c.etas, n * sizeof(double), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(rhs, c.gwce_lv, n * sizeof(double), cudaMemcpyDeviceToHost));
  ADC_CUDA(cudaMemcpy(coef, c.diag, n * sizeof(double), cudaMemcpyDeviceToHost));
  for (int j = 1; j < maxnz; ++j) {
    rc = copy_column(c.offd, coef, n, ndim, w, j, false);
    if (rc) return rc;
  }
  jcg_q1_set(it.q1);
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

void adc_jcg_noalloc(const int *n_, const int *ndim_, const int *maxnz_, int *jcoef,
                     double *coef, double *rhs, double *u, int *iwksp, const int *nw_,
                     double *wksp, int *iparm, double *rparm, int *ier) {
  (void)iwksp;
  (void)wksp;
  *ier = 0;
  const int n = *n_, ndim = *ndim_, maxnz = *maxnz_, nw = *nw_;
  if (iparm[0] <= 0) return;
  const int itmax = iparm[0];
  if (n <= 0) { *ier = 11; return; }
  if (ndim < n || maxnz < 1) { *ier = 11; set_error("ndim < n or maxnz < 1"); return; }
  if (2 * sizeof(double) * ((size_t)itmax + 1) > 48 * 1024) {
    *ier = 905;
    set_error("adc_jcg_noalloc: itmax = %d is above the JCG scalar block's limit of 3071", itmax);
    return;
  }
  const size_t need = noalloc_need(n, maxnz, itmax);
  if (need > kNoAllocBytes) {
    *ier = 905;
    set_error("adc_jcg_noalloc: n = %d, maxnz = %d, itmax = %d needs more than the %zu-byte "
              "static scratch", n, maxnz, itmax, kNoAllocBytes);
    return;
  }
  // structural part of scal (itpackv.F:2340-2391), in place on the caller's arrays
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
  int rc = noalloc_solve(n, ndim, maxnz, jcoef, coef, rhs, u, itmax, iparm, rparm, e, in, stptst,
                         cme, bnrm, rnrm);
  restore_zeros();
  if (rc != ADC_OK) {
    *ier = (rc == ADC_ERR_NOMEM) ? 905 : 904;
    return;
  }
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
